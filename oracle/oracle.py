"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracle.

Two checkers live here:
  * ``liboracle_mndo.so``  — the C restatement (mndo_oracle.c), callable in-process;
  * ``_ref/ref_driver``    — the unmodified reference (LuisAlfredoNu/semiGPU) built by
    oracle/Makefile, run as a subprocess that prints one JSON object.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
The product library never does.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_mndo.so")
REF_DRIVER = os.path.join(HERE, "_ref", "ref_driver")
REF_CLI = os.path.join(HERE, "_ref", "semiGPU")

_lib = None
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def build(quiet: bool = True) -> None:
    """Compile the restatement (and the reference when its tree is present)."""
    subprocess.run(["make", "-C", HERE, "all"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_nao.argtypes = [ctypes.c_int, _I]
        L.oracle_nocc.argtypes = [ctypes.c_int, _I]
        L.oracle_block_count.argtypes = [ctypes.c_int, _I]
        L.oracle_block_count.restype = ctypes.c_long
        L.oracle_integrals.argtypes = [ctypes.c_int, _I, _D, _D]
        L.oracle_hcore.argtypes = [ctypes.c_int, _I, _D, _D, _D]
        L.oracle_overlap.argtypes = [ctypes.c_int, _I, _D, _D]
        L.oracle_fock.argtypes = [ctypes.c_int, _I, _D, _D, _D, _D, ctypes.c_int]
        L.oracle_energy.argtypes = [ctypes.c_int, _D, _D, _D]
        L.oracle_energy.restype = ctypes.c_double
        L.oracle_core_core.argtypes = [ctypes.c_int, _I, _D, _D]
        L.oracle_core_core.restype = ctypes.c_double
        L.oracle_density.argtypes = [ctypes.c_int, ctypes.c_int, _D, _D]
        L.oracle_scf.argtypes = [ctypes.c_int, _I, _D, ctypes.c_double, ctypes.c_int, _D, _I, _I,
                                 _D, _D, _D, _D, _D, _D, ctypes.c_int]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_D)


def _i(a):
    return a.ctypes.data_as(_I)


def _arrs(Z, xyz):
    Z = np.ascontiguousarray(Z, np.int32)
    xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1)
    return Z, xyz


def nao(Z):
    Z = np.ascontiguousarray(Z, np.int32)
    return lib().oracle_nao(len(Z), _i(Z))


def integrals(Z, xyz):
    """Ragged pair blocks in the reference's [A][B<=A] order, flattened (eV)."""
    Z, xyz = _arrs(Z, xyz)
    out = np.zeros(lib().oracle_block_count(len(Z), _i(Z)))
    rc = lib().oracle_integrals(len(Z), _i(Z), _d(xyz), _d(out))
    if rc:
        raise ValueError(f"oracle_integrals rc={rc}")
    return out


def hcore(Z, xyz, blocks):
    Z, xyz = _arrs(Z, xyz)
    n = nao(Z)
    H = np.zeros(n * (n + 1) // 2)
    rc = lib().oracle_hcore(len(Z), _i(Z), _d(xyz), _d(np.ascontiguousarray(blocks)), _d(H))
    if rc:
        raise ValueError(f"oracle_hcore rc={rc}")
    return H


def overlap(Z, xyz):
    Z, xyz = _arrs(Z, xyz)
    n = nao(Z)
    S = np.zeros(n * (n + 1) // 2)
    lib().oracle_overlap(len(Z), _i(Z), _d(xyz), _d(S))
    return S


def fock(Z, blocks, H, P, literal=False):
    Z = np.ascontiguousarray(Z, np.int32)
    F = np.zeros_like(H)
    rc = lib().oracle_fock(len(Z), _i(Z), _d(np.ascontiguousarray(blocks)),
                           _d(np.ascontiguousarray(H)), _d(np.ascontiguousarray(P)), _d(F),
                           int(literal))
    if rc:
        raise ValueError(f"oracle_fock rc={rc}")
    return F


def energy(H, F, P):
    n = int((np.sqrt(8 * len(H) + 1) - 1) / 2)
    return lib().oracle_energy(n, _d(np.ascontiguousarray(H)), _d(np.ascontiguousarray(F)),
                               _d(np.ascontiguousarray(P)))


def core_core(Z, xyz, blocks):
    Z, xyz = _arrs(Z, xyz)
    return lib().oracle_core_core(len(Z), _i(Z), _d(xyz), _d(np.ascontiguousarray(blocks)))


def scf(Z, xyz, tol=1e-6, max_iter=100, literal_fock=False):
    """Full SCF; dict with energies, n_iter, converged, E_el, E_cc, E_tot, H, F, P, eig."""
    Z, xyz = _arrs(Z, xyz)
    n = nao(Z)
    if n < 0:
        raise ValueError("unsupported element")
    npk = n * (n + 1) // 2
    en = np.zeros(max_iter + 1)
    it, cv = ctypes.c_int(0), ctypes.c_int(0)
    eel, ecc = ctypes.c_double(0), ctypes.c_double(0)
    H, F, P, w = np.zeros(npk), np.zeros(npk), np.zeros(npk), np.zeros(n)
    rc = lib().oracle_scf(len(Z), _i(Z), _d(xyz), tol, max_iter, _d(en), ctypes.byref(it),
                          ctypes.byref(cv), ctypes.byref(eel), ctypes.byref(ecc), _d(H), _d(F),
                          _d(P), _d(w), int(literal_fock))
    if rc:
        raise RuntimeError(f"oracle_scf rc={rc}")
    return {"energies": en[: it.value + 1], "n_iter": it.value, "converged": bool(cv.value),
            "E_el": eel.value, "E_cc": ecc.value, "E_tot": eel.value + ecc.value,
            "H": H, "F": F, "P": P, "eig": w}


def reference_available() -> bool:
    return os.path.exists(REF_DRIVER)


def run_reference(Z, xyz, tol=1e-6, max_iter=100, matrices=True, timeout=None) -> dict:
    """Run the unmodified reference through ref_driver on a temporary XYZ file."""
    from semigpu_b200.geometry import Molecule, format_xyz

    Z, xyz = _arrs(Z, xyz)
    with tempfile.NamedTemporaryFile("w", suffix=".xyz", delete=False) as fh:
        fh.write(format_xyz(Molecule(Z, xyz.reshape(-1, 3)), comment="oracle"))
        path = fh.name
    try:
        cmd = [REF_DRIVER, path, "--tol", repr(tol), "--max-iter", str(max_iter)]
        if not matrices:
            cmd.append("--no-matrices")
        out = subprocess.run(cmd, check=True, capture_output=True, text=True, timeout=timeout,
                             env=dict(os.environ, OPENBLAS_NUM_THREADS="1"))
        return json.loads(out.stdout)
    finally:
        os.unlink(path)
