"""C ABI checks that need no GPU: the library loads, exports every function
include/grace_b200.h declares, its structs match the ctypes mirror, and the
host-only helpers agree with the Python parameter builders."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from grace_b200 import _lib, abi, params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "grace_b200.h")


def declared_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void)\s+(grb_\w+)\s*\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    # and the Python mirror binds exactly the declared set
    assert sorted(abi.PROTOTYPES) == names


def test_library_imports_no_process_exit():
    """No code path of the library ends the caller's process: every error
    is a status code.  nvcc compiles a __device__-only helper that host code
    calls into a host stub that calls exit(1) without a diagnostic, so an
    imported exit() is that mistake."""
    out = subprocess.run(["nm", "-D", "--undefined-only", _lib.load()._name], capture_output=True, text=True,
                         check=True).stdout
    imported = {ln.split()[-1].split("@")[0] for ln in out.splitlines() if ln.strip()}
    assert not imported & {"exit", "_exit", "_Exit", "abort", "quick_exit"}


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('''#include <stdio.h>
#include <stddef.h>
#include "grace_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\\n", sizeof(grb_params), sizeof(grb_eos_params), sizeof(grb_grid),
         sizeof(grb_fields), sizeof(grb_status));
  printf("%zu %zu %zu %zu\\n", offsetof(grb_params, rho_fl), offsetof(grb_params, c2p_tol),
         offsetof(grb_params, dmp_M), offsetof(grb_params, emf));
  return 0;
}
''')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    c = [int(x) for x in out]
    py = [ctypes.sizeof(abi.Params), ctypes.sizeof(abi.EosParams), ctypes.sizeof(abi.Grid),
          ctypes.sizeof(abi.Fields), ctypes.sizeof(abi.Status),
          abi.Params.rho_fl.offset, abi.Params.c2p_tol.offset, abi.Params.dmp_M.offset,
          abi.Params.emf.offset]
    assert c == py


def test_defaults_match_python():
    lib = _lib.load()
    for kind in (abi.EOS_IDEAL_GAS, abi.EOS_HYBRID_PWPOLY):
        c = abi.Params()
        lib.grb_params_defaults(ctypes.byref(c), kind)
        p = params.defaults(kind)
        assert bytes(c) == bytes(p)


def test_pwpoly_setup_matches_python():
    lib = _lib.load()
    gammas = [1.35692, 3.005, 2.988, 2.851]
    rhos = [1.5e-4, 8.1e-4, 1.6e-3]
    e = abi.EosParams()
    g = (ctypes.c_double * 4)(*gammas)
    r = (ctypes.c_double * 3)(*rhos)
    assert lib.grb_eos_setup_pwpoly(ctypes.byref(e), 4, 0.0801, g, r) == abi.OK
    ep = abi.EosParams()
    params.setup_pwpoly(ep, 0.0801, gammas, rhos)
    for f in ("pw_kappa", "pw_gamma", "pw_rho", "pw_eps", "pw_press"):
        assert list(getattr(e, f)) == list(getattr(ep, f)), f
    # descending densities are rejected
    assert lib.grb_eos_setup_pwpoly(ctypes.byref(e), 2, 1.0, g, (ctypes.c_double * 1)(-1.0)) == abi.ERR_INVALID


def test_invalid_arguments_are_rejected_without_a_gpu():
    lib = _lib.load()
    h = ctypes.c_void_p()
    bad = params.blast()
    bad.emf = abi.EMF_UCT          # FOFC with UCT is rejected (evolve.cpp:479-481)
    assert lib.grb_create(ctypes.byref(h), ctypes.byref(bad)) == abi.ERR_INVALID
    bad = params.blast()
    bad.recon = 7
    assert lib.grb_create(ctypes.byref(h), ctypes.byref(bad)) == abi.ERR_INVALID
    assert lib.grb_advance_substep(None, None, 0.0, 0.0, 0.0, None, None, None, None) == abi.ERR_INVALID
    assert lib.grb_compute_auxiliary_quantities(None, None, None, None, None) == abi.ERR_INVALID
    assert lib.grb_destroy(None) == abi.ERR_INVALID
