"""sgb_scf_noalloc: the allocation-free single-molecule entry point.

It exists for callers that may not allocate device memory: code running inside a host framework
that owns the GPU's memory through its own pool and forbids other allocations, or code that must
not allocate once it has started.  It must give what the regular stage API gives, call after
call, with its scratch in the library's static device array.

The file name sorts last so that pytest collects it after every other test.  When it runs after
them, earlier tests have already set up the device (contexts, constant tables), so the per-device
first-call set-up inside sgb_scf_noalloc is covered by a fresh child process in
test_noalloc_first_call_in_fresh_process."""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import semigpu_b200 as sg

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
with open(os.path.join(GOLDEN, "reference_cases.json")) as _fh:
    CASES = json.load(_fh)["cases"]

TOL_E = 1e-6      # eV, the energy tolerance of the other parity tests
TOL_MIXED = 1e-4  # eV, the mixed-precision form against the reference

# one molecule per size class the static scratch serves: nao <= 32, 33-64, 65-96, 97-128 (the
# last at the entry point's 128-AO limit region: C20H42, 122 AOs, ~0.7 MB of scratch)
CLASS_CASES = ["fixture/04_pyridine@1e-06", "batch/02_C9H20@1e-06", "batch/03_C13H28@1e-06",
               "alkane/C20H42@1e-06"]


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


def _stage_api(ctx, c):
    return sg.Molecule(ctx, np.array(c["Z"], np.int32), np.array(c["xyz"])).run(tol=c["tol"])


def test_noalloc_two_calls_match_stage_api():
    """Two different molecules back to back (the second reuses the scratch the first left)."""
    keys = ["fixture/04_pyridine@1e-06", "fixture/03_formaldehyde@1e-06"]
    got = [_noalloc(CASES[k]["Z"], CASES[k]["xyz"], tol=CASES[k]["tol"]) for k in keys]
    with sg.Context(0) as ctx:
        for key, (rc, eel, ecc, it, cv, st) in zip(keys, got):
            c = CASES[key]
            ref = _stage_api(ctx, c)
            assert rc == 0 and st == 0 and cv
            assert it == ref["n_iter"] == c["n_iter"]
            assert abs(eel - ref["E_el"]) < TOL_E
            assert abs(ecc - ref["E_cc"]) < TOL_E
            assert abs(eel + ecc - c["E_tot"]) < TOL_E


def test_noalloc_every_size_class_twice():
    """Each CTA-size instance (128, 256, 512 threads) through the static scratch, up to the
    ~0.7 MB a 122-AO molecule needs; every molecule twice, in two rounds, against the stage API
    and the reference's energy."""
    rounds = [[_noalloc(CASES[k]["Z"], CASES[k]["xyz"]) for k in CLASS_CASES] for _ in range(2)]
    with sg.Context(0) as ctx:
        for i, key in enumerate(CLASS_CASES):
            c = CASES[key]
            ref = _stage_api(ctx, c)
            for got in rounds:
                rc, eel, ecc, it, cv, st = got[i]
                assert rc == 0 and st == 0 and cv, key
                assert it == ref["n_iter"] == c["n_iter"], key
                assert abs(eel - ref["E_el"]) < TOL_E, key
                assert abs(ecc - ref["E_cc"]) < TOL_E, key
                assert abs(eel + ecc - c["E_tot"]) < TOL_E, key


def test_noalloc_mixed_precision_at_the_ao_limit(monkeypatch):
    """The 122-AO alkane with SGB_DENSITY_SOLVER=mixed (TF32 tensor-core products): within the
    mixed-precision tolerance of the reference's energy, twice in a row."""
    monkeypatch.setenv("SGB_DENSITY_SOLVER", "mixed")
    c = CASES["alkane/C20H42@1e-06"]
    for _ in range(2):
        rc, eel, ecc, it, cv, st = _noalloc(c["Z"], c["xyz"])
        assert rc == 0 and st == 0 and cv
        assert abs(eel + ecc - c["E_tot"]) < TOL_MIXED


def test_noalloc_allocates_no_device_memory():
    """After one warm-up call per molecule (which may load kernel code lazily), further calls
    leave the device's free memory unchanged."""
    import torch

    for k in CLASS_CASES:
        assert _noalloc(CASES[k]["Z"], CASES[k]["xyz"])[0] == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(2):
        for k in CLASS_CASES:
            assert _noalloc(CASES[k]["Z"], CASES[k]["xyz"])[0] == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0


_CHILD = r"""
import ctypes, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import semigpu_b200 as sg
c = json.loads(sys.argv[2])
Z = np.ascontiguousarray(c["Z"], np.int32)
xyz = np.ascontiguousarray(c["xyz"], np.float64)
out = []
for _ in range(2):
    eel, ecc = ctypes.c_double(), ctypes.c_double()
    it, cv, st = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    rc = sg.lib().sgb_scf_noalloc(len(Z), Z.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                  xyz.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1e-6, 100,
                                  None, ctypes.byref(eel), ctypes.byref(ecc), ctypes.byref(it),
                                  ctypes.byref(cv), ctypes.byref(st))
    out.append([rc, eel.value, ecc.value, it.value, cv.value, st.value])
print(json.dumps(out))
"""


def test_noalloc_first_call_in_fresh_process():
    """The per-device set-up of the first call (constant tables, the scratch's device address),
    in a process that has made no other CUDA call before it."""
    c = CASES["batch/03_C13H28@1e-06"]
    arg = json.dumps({"Z": c["Z"], "xyz": c["xyz"]})
    r = subprocess.run([sys.executable, "-c", _CHILD, ROOT, arg], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    for rc, eel, ecc, it, cv, st in json.loads(r.stdout.strip().splitlines()[-1]):
        assert rc == 0 and st == 0 and cv
        assert it == c["n_iter"]
        assert abs(eel + ecc - c["E_tot"]) < TOL_E


def test_noalloc_rejects_oversize_molecule():
    Z = np.full(40, 6, np.int32)  # 160 AOs > 128
    xyz = np.arange(120, dtype=np.float64) * 1.5
    rc = _noalloc(Z, xyz)[0]
    assert rc == sg.E_UNSUPPORTED
