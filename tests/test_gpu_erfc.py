"""The pair kernels' screened-Coulomb factors against CUDA's and against
double precision.

erfc_and_exp (sponge_b200/csrc/snb_common.cuh) forms erfc(x) for x <= 4 as a
degree-8 polynomial in t = 1/(1 + x/2) times exp(-x^2), with the hardware
exp2 and the fast division, and uses CUDA's erfcf / expf beyond 4.  In the
pair kernels x = beta r runs over [0, beta rc]: 2.79 at cutoff 8 A, 2.75 at
10 A.  Held here over [0, 6] (dense, with points on both sides of the switch
at x = 4):
  * on [0, 3], the range the pair kernels use: erfc and exp(-x^2) within
    1.5e-6 relative of double precision and of CUDA's erfcf (the budget:
    polynomial 3.3e-7, fast division 5.4e-7, hardware exp2 up to 1.2e-6 at
    x = 3 by CUDA's stated ulp bound; measured on B200: 1.01e-6, exp 8.9e-7);
  * on (3, 4]: the same within 4e-6 (the hardware exp2's error grows with
    x^2, 2 + 1.16 x^2 ulp by CUDA's documentation, and x^2 itself is rounded);
  * beyond 4: bit-equal to CUDA's erfcf and expf (they are the ones used).
"""

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_erfc_and_exp_against_cuda_and_fp64():
    import torch
    assert torch.cuda.is_available(), "GPU tests need CUDA"
    from tests import gpu_helpers as g
    lib = g.capi.load()
    x = np.concatenate([np.linspace(0.0, 6.0, 600001, dtype=np.float64),
                        4.0 + np.arange(-64, 65) * 2.0 ** -21]).astype(np.float32)
    x = np.unique(x[x >= 0])
    d_x = g.dev(x)
    out = torch.empty(4 * len(x), dtype=torch.float32, device="cuda")
    g.capi.check(lib.snb_check_erfc_exp(len(x), g.ptr(d_x), g.ptr(out), g.stream()),
                 "check_erfc_exp")
    torch.cuda.synchronize()
    o = out.cpu().numpy().reshape(-1, 4).astype(np.float64)
    ours_erfc, ours_exp, cuda_erfc, cuda_exp = o.T
    xd = x.astype(np.float64)
    true_erfc = np.array([math.erfc(v) for v in xd])
    true_exp = np.exp(-xd * xd)
    rel = lambda a, b: np.abs(a - b) / np.abs(b)  # noqa: E731
    for lo_x, hi_x, tol, tol_cuda in ((0.0, 3.0, 1.5e-6, 1.5e-6), (3.0, 4.0, 4e-6, 4e-6)):
        m = (x >= lo_x) & (x <= hi_x) if lo_x == 0.0 else (x > lo_x) & (x <= hi_x)
        errs = (rel(ours_erfc[m], true_erfc[m]).max(), rel(ours_exp[m], true_exp[m]).max(),
                rel(ours_erfc[m], cuda_erfc[m]).max(), rel(cuda_erfc[m], true_erfc[m]).max())
        print(f"[{lo_x}, {hi_x}] erfc vs fp64 {errs[0]:.2e}, exp vs fp64 {errs[1]:.2e}, "
              f"erfc vs erfcf {errs[2]:.2e} (erfcf vs fp64 {errs[3]:.2e})")
        assert errs[0] <= tol and errs[1] <= tol and errs[2] <= tol_cuda
    hi = x > 4.0
    assert hi.sum() > 1000
    assert np.array_equal(ours_erfc[hi], cuda_erfc[hi])
    assert np.array_equal(ours_exp[hi], cuda_exp[hi])
