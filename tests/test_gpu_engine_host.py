"""snb_engine_md_steps_host: MD steps for a caller whose state lives in host
memory.  Thirty steps in calls that copy crd / vel in from pinned host
buffers and back out (one step per call, or ten) give, bit for bit, the
trajectory of thirty device-resident graph steps; the host buffers hold the
result when the call returns.  The velocities cross the link beside the
force phase and the first update waits for them.  Both layouts: crd and vel
apart, and side by side in one state array on each end."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from tests import gpu_helpers
    return gpu_helpers


@pytest.mark.parametrize("per_call", [1, 10])
@pytest.mark.parametrize("layout", ["apart", "state"])
def test_host_steps_equal_device_steps(g, layout, per_call):
    import torch
    from sponge_b200 import systems
    s = systems.water_box(500, seed=9)
    lib = g.capi.load()
    dt = ctypes.c_float(0.5e-3 * systems.TIME_CONVERSION)
    out = []
    for host in (False, True):
        e = g.engine_create(s, 8.0)
        g.engine_set_water_bonded(e, s)
        crd = g.dev(s.crd.reshape(-1), np.float32)
        vel = g.dev(s.vel.reshape(-1), np.float32)
        invm = g.dev((1.0 / s.mass).astype(np.float32))
        h_crd = torch.from_numpy(s.crd.reshape(-1).astype(np.float32).copy()).pin_memory()
        h_vel = torch.from_numpy(s.vel.reshape(-1).astype(np.float32).copy()).pin_memory()
        if host and layout == "state":
            d_state, h_state = torch.cat([crd, vel]), torch.cat([h_crd, h_vel]).pin_memory()
            crd, vel = d_state[:3 * s.n], d_state[3 * s.n:]
            h_crd, h_vel = h_state[:3 * s.n], h_state[3 * s.n:]
        st = torch.cuda.Stream()
        sp = ctypes.c_void_p(st.cuda_stream)
        try:
            with torch.cuda.stream(st):
                if host:
                    for k in range(0, 30, per_call):
                        g.capi.check(lib.snb_engine_md_steps_host(
                            e, g.ptr(h_crd), g.ptr(h_vel), g.ptr(crd), g.ptr(vel), g.ptr(invm),
                            dt, k, per_call, sp), "host steps")
                    out.append((h_crd.numpy().copy(), h_vel.numpy().copy()))
                else:
                    for k in range(30):
                        g.capi.check(lib.snb_engine_md_steps_graph(
                            e, g.ptr(crd), g.ptr(vel), g.ptr(invm), dt, k, 1, sp), "steps")
                    st.synchronize()
                    out.append((crd.cpu().numpy(), vel.cpu().numpy()))
        finally:
            lib.snb_engine_destroy(e)
    assert np.isfinite(out[1][0]).all()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
