"""sgb_scf_noalloc: the allocation-free single-molecule entry point, for callers that may not
allocate device memory (a host framework owning the GPU memory pool, or code that must not
allocate after start-up).  It must give what the regular stage API gives, call after call, with
its scratch in the library's static device array.  This file is collected last on purpose."""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np
import pytest

import semigpu_b200 as sg

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
with open(os.path.join(GOLDEN, "reference_cases.json")) as _fh:
    CASES = json.load(_fh)["cases"]

TOL_E = 1e-6  # eV, the energy tolerance of the other parity tests


def _noalloc(Z, xyz, tol=1e-6, max_iter=100):
    Z = np.ascontiguousarray(Z, np.int32)
    xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1)
    eel, ecc = ctypes.c_double(), ctypes.c_double()
    it, cv, st = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    rc = sg.lib().sgb_scf_noalloc(len(Z), Z.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                  xyz.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), tol,
                                  max_iter, None, ctypes.byref(eel), ctypes.byref(ecc),
                                  ctypes.byref(it), ctypes.byref(cv), ctypes.byref(st))
    return rc, eel.value, ecc.value, it.value, bool(cv.value), st.value


def test_noalloc_two_calls_match_stage_api():
    """Two different molecules back to back (the second reuses the scratch the first left)."""
    keys = ["fixture/04_pyridine@1e-06", "fixture/03_formaldehyde@1e-06"]
    got = []
    for key in keys:  # the allocation-free calls come first: a fresh process sets up here
        c = CASES[key]
        got.append(_noalloc(c["Z"], c["xyz"], tol=c["tol"]))
    with sg.Context(0) as ctx:
        for key, (rc, eel, ecc, it, cv, st) in zip(keys, got):
            c = CASES[key]
            ref = sg.Molecule(ctx, np.array(c["Z"], np.int32), np.array(c["xyz"])).run(tol=c["tol"])
            assert rc == 0 and st == 0 and cv
            assert it == ref["n_iter"] == c["n_iter"]
            assert abs(eel - ref["E_el"]) < TOL_E
            assert abs(ecc - ref["E_cc"]) < TOL_E
            assert abs(eel + ecc - c["E_tot"]) < TOL_E


def test_noalloc_rejects_oversize_molecule():
    Z = np.full(40, 6, np.int32)  # 160 AOs > 128
    xyz = np.arange(120, dtype=np.float64) * 1.5
    rc = _noalloc(Z, xyz)[0]
    assert rc == sg.E_UNSUPPORTED
