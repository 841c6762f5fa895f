"""The reference-side adapter (oracle/ref_build/sponge_nb_adapter.*) compiled
against the reference's own headers.

adapter_signatures.cpp holds the type of every adapter member equal to the
reference member it replaces (neighbor_list.h:17-24,
Lennard_Jones_force.h:118-172, LJ_soft_core.h:238-274, PM_force.h:153-190);
these tests compile it and the adapter itself with the reference's CPU
definitions, show that a changed parameter type fails the check, and read
the built adapter library's dynamic symbols: it binds to nothing of this
library but the C ABI of include/sponge_nb.h.  They need the reference's
sources (the folder oracle's build recorded) and skip where only the
prebuilt checkers are present.
"""

import os
import re
import shutil
import subprocess

import pytest

from oracle.oracle import HERE as ORACLE_DIR
from oracle.oracle import built_reference_sources

REF = built_reference_sources()
ROOT = os.path.dirname(ORACLE_DIR)
BUILD = os.path.join(ORACLE_DIR, "ref_build")
ADAPTER_SO = os.path.join(ORACLE_DIR, "_ref", "libsponge_nb_adapter.so")
HEADER = os.path.join(ROOT, "include", "sponge_nb.h")

needs_reference = pytest.mark.skipif(REF is None, reason="reference sources absent")


def _compile(src, include_first=None):
    cmd = ["g++", "-std=c++17", "-fsyntax-only", "-DUSE_CPU", "-w"]
    if include_first:
        cmd.append(f"-I{include_first}")
    cmd += [f"-I{BUILD}", f"-I{REF}", f"-I{os.path.join(ROOT, 'include')}", src]
    return subprocess.run(cmd, capture_output=True, text=True, timeout=300)


@needs_reference
@pytest.mark.parametrize("src", ["adapter_signatures.cpp", "sponge_nb_adapter.cpp"])
def test_adapter_compiles_against_reference_headers(src):
    r = _compile(os.path.join(BUILD, src))
    assert r.returncode == 0, r.stderr[-4000:]


@needs_reference
def test_signature_check_catches_a_changed_parameter(tmp_path):
    """The check is live: the adapter header with one parameter's type
    changed (float* atom_energy -> double* in the LJ direct-force member)
    fails to compile, at the assertion naming that member."""
    with open(os.path.join(BUILD, "sponge_nb_adapter.h")) as f:
        text = f.read()
    planted = text.replace(
        "float* atom_energy, const int need_virial, LTMatrix3* atom_virial,",
        "double* atom_energy, const int need_virial, LTMatrix3* atom_virial,", 1)
    assert planted != text
    (tmp_path / "sponge_nb_adapter.h").write_text(planted)
    shutil.copy(os.path.join(BUILD, "adapter_signatures.cpp"), tmp_path)
    r = _compile(str(tmp_path / "adapter_signatures.cpp"), include_first=str(tmp_path))
    assert r.returncode != 0
    assert ("LENNARD_JONES_INFORMATION::LJ_PME_Direct_Force_With_Atom_Energy_And_Virial"
            " differs from the reference") in r.stderr


def _dynamic_symbols(path, defined):
    flag = "--defined-only" if defined else "--undefined-only"
    out = subprocess.run(["nm", "-D", flag, path], capture_output=True, text=True,
                         check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


@pytest.mark.skipif(not os.path.exists(ADAPTER_SO), reason="adapter library not built")
def test_adapter_binds_only_the_c_abi():
    with open(HEADER) as f:
        declared = set(re.findall(r"\b(snb_[a-z0-9_]+)\s*\(", f.read()))
    undefined = _dynamic_symbols(ADAPTER_SO, defined=False)
    used = {s for s in undefined if s.startswith("snb_")}
    assert used, "the adapter calls no library entry point"
    assert used <= declared, sorted(used - declared)
    # nothing else of the library: every other undefined name is the C/C++
    # runtime's or the CUDA runtime's
    other = {s.split("@")[0] for s in undefined - used}
    assert all(not s.startswith(("snb", "_ZN3snb")) for s in other), sorted(other)
    assert "adapter_force" in _dynamic_symbols(ADAPTER_SO, defined=True)
