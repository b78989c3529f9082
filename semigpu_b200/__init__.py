"""semigpu_b200: MNDO SCF engine for NVIDIA B200, Python access to its C ABI.

The compute path is the CUDA library ``libsemigpu_b200.so`` built in-tree for sm_100a
(``python -m semigpu_b200.build``).  This module only marshals arrays through ctypes; there is
no CPU implementation behind it.  If the library is missing, every entry point raises.

Reference interface mirrored (LuisAlfredoNu/semiGPU, src/common): the stage API of
``src/App/semiGPU.cc:29-104`` — two-center integrals, Hcore, SCF, core-core repulsion — on one
molecule (:class:`Molecule`), plus a batched path for many molecules (:class:`Batch`,
:func:`run_molecules`).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import geometry

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsemigpu_b200.so")

OK, E_ARG, E_ELEMENT, E_CUDA, E_NOMEM, E_STATE, E_UNSUPPORTED, E_EIG, E_NAN, E_NOCONV = (
    0, -1, -2, -3, -4, -5, -6, 1, 2, 3)
BLOCKS, HCORE, FOCK, DENSITY, EIGVAL, EIGVEC = range(6)
PATH_AUTO, PATH_CTA, PATH_GRID = range(3)
SOLVER_PURIFY, SOLVER_JACOBI, SOLVER_PURIFY_MIXED = range(3)

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_VP = ctypes.c_void_p

# name -> (restype, argtypes); the exported C ABI of include/semigpu_b200.h
SIGNATURES = {
    "sgb_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_size_t, ctypes.POINTER(_VP)]),
    "sgb_ctx_destroy": (ctypes.c_int, [_VP]),
    "sgb_ctx_synchronize": (ctypes.c_int, [_VP]),
    "sgb_last_error": (ctypes.c_char_p, [_VP]),
    "sgb_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "sgb_ctx_bytes_in_use": (ctypes.c_size_t, [_VP]),
    "sgb_ctx_reserve": (ctypes.c_int, [_VP, ctypes.c_size_t]),
    "sgb_ctx_set_density_solver": (ctypes.c_int, [_VP, ctypes.c_int]),
    "sgb_ctx_set_sm_share": (ctypes.c_int, [_VP, ctypes.c_double]),
    "sgb_ctx_set_diis": (ctypes.c_int, [_VP, ctypes.c_int]),
    "sgb_ctx_set_damping": (ctypes.c_int, [_VP, ctypes.c_double]),
    "sgb_grid_configs": (ctypes.c_int, [_I, _I, _I, _I, _I, ctypes.c_int]),
    "sgb_ctx_set_grid_config": (ctypes.c_int, [_VP, ctypes.c_int]),
    "sgb_ctx_set_limits": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_longlong]),
    "sgb_diag_barrier_timeout": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int,
                                                ctypes.c_longlong, _I]),
    "sgb_size_classes": (ctypes.c_int, [_I, _I, _I, ctypes.c_int]),
    "sgb_ctx_set_class_threads": (ctypes.c_int, [_VP, ctypes.c_int, _I]),
    "sgb_mndo_parameters": (ctypes.c_int, [ctypes.c_int, _D]),
    "sgb_heat_of_formation": (ctypes.c_int, [ctypes.c_int, _I, ctypes.c_double, _D]),
    "sgb_mol_create": (ctypes.c_int, [_VP, ctypes.c_int, _I, _D, ctypes.POINTER(_VP)]),
    "sgb_mol_destroy": (ctypes.c_int, [_VP]),
    "sgb_mol_info": (ctypes.c_int, [_VP, _I, _I, _I, ctypes.POINTER(ctypes.c_longlong)]),
    "sgb_mol_set_path": (ctypes.c_int, [_VP, ctypes.c_int]),
    "sgb_two_center": (ctypes.c_int, [_VP, _VP]),
    "sgb_hcore": (ctypes.c_int, [_VP, _VP]),
    "sgb_scf": (ctypes.c_int, [_VP, _VP, ctypes.c_double, ctypes.c_int, _VP, _D]),
    "sgb_core_core": (ctypes.c_int, [_VP, _VP, _D]),
    "sgb_fock": (ctypes.c_int, [_VP, _VP, _D, _D, _D]),
    "sgb_get": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _D, ctypes.c_size_t]),
    "sgb_electronic_energy": (ctypes.c_int, [_VP, ctypes.c_int, _D, _D, _D, _D]),
    "sgb_batch_create": (ctypes.c_int, [_VP, ctypes.c_int, _I, _I, _D, ctypes.POINTER(_VP)]),
    "sgb_batch_destroy": (ctypes.c_int, [_VP]),
    "sgb_batch_set_coordinates": (ctypes.c_int, [_VP, _VP, _D]),
    "sgb_batch_run": (ctypes.c_int, [_VP, _VP, ctypes.c_double, ctypes.c_int]),
    "sgb_batch_results": (ctypes.c_int, [_VP, _VP, _D, _D, _I, _I, _I]),
    "sgb_run_molecules": (ctypes.c_int, [_VP, ctypes.c_int, _I, _I, _D, ctypes.c_double,
                                         ctypes.c_int, _D, _D, _I, _I, _I]),
    "sgb_batch_last_ms": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_float)]),
    "sgb_ctx_set_priority": (ctypes.c_int, [_VP, ctypes.c_int]),
    "sgb_gradient": (ctypes.c_int, [_VP, ctypes.c_int, _I, _D, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_double, _D, _D]),
    "sgb_batch_launches": (ctypes.c_int, [_VP, _I]),
    "sgb_scf_noalloc": (ctypes.c_int, [ctypes.c_int, _I, _D, ctypes.c_double, ctypes.c_int, _VP,
                                       _D, _D, _I, _I, _I]),
    "sgb_batch_device_coordinates": (ctypes.c_int, [_VP, ctypes.POINTER(_VP)]),
    "sgb_batch_timestamps": (ctypes.c_int, [_VP, _VP, ctypes.POINTER(ctypes.c_ulonglong),
                                            ctypes.POINTER(ctypes.c_ulonglong)]),
    "sgb_batch_set_profiling": (ctypes.c_int, [_VP, ctypes.c_int]),
    "sgb_batch_stage_cycles": (ctypes.c_int, [_VP, _VP, ctypes.POINTER(ctypes.c_ulonglong)]),
}

_lib = None


class SGBError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def lib() -> ctypes.CDLL:
    """The CUDA library; raises if it has not been built (there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m semigpu_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_D)


def _i(a):
    return a.ctypes.data_as(_I)


def heat_of_formation(Z, e_tot: float) -> float:
    """kcal/mol from the total energy in eV (MOPAC convention, atomic eisol / heat data)."""
    Z = np.ascontiguousarray(Z, np.int32)
    out = ctypes.c_double()
    rc = lib().sgb_heat_of_formation(len(Z), _i(Z), float(e_tot), ctypes.byref(out))
    if rc:
        raise SGBError(rc, lib().sgb_status_string(rc).decode())
    return out.value


def size_classes() -> list[tuple[int, int]]:
    """(largest nao, default CTA threads) of each size class of the batched launch."""
    cnt = ctypes.c_int()
    lib().sgb_size_classes(ctypes.byref(cnt), None, None, 0)
    nmax = np.zeros(cnt.value, np.int32)
    thr = np.zeros(cnt.value, np.int32)
    lib().sgb_size_classes(ctypes.byref(cnt), _i(nmax), _i(thr), cnt.value)
    return [(int(a), int(b)) for a, b in zip(nmax, thr)]


def grid_configs() -> list[dict]:
    """Tile configurations of the whole-GPU purification: tile rows, warps, k-blocks per ring
    stage, stages (index = the value for Context.set_grid_config)."""
    n = ctypes.c_int()
    lib().sgb_grid_configs(ctypes.byref(n), None, None, None, None, 0)
    a = [np.zeros(n.value, np.int32) for _ in range(4)]
    lib().sgb_grid_configs(ctypes.byref(n), *(_i(x) for x in a), n.value)
    return [{"bm": int(a[0][k]), "warps": int(a[1][k]), "kblocks": int(a[2][k]),
             "stages": int(a[3][k])} for k in range(n.value)]


def mndo_parameters(z: int) -> np.ndarray:
    """The engine's MNDO parameters of element z (order of the SGB_P_* indices)."""
    out = np.zeros(18)
    rc = lib().sgb_mndo_parameters(int(z), _d(out))
    if rc:
        raise SGBError(rc, lib().sgb_status_string(rc).decode())
    return out


class _ScfResult(ctypes.Structure):
    _fields_ = [("e_el", ctypes.c_double), ("n_iter", ctypes.c_int),
                ("converged", ctypes.c_int), ("status", ctypes.c_int)]


class Context:
    """One device, one stream (sgb_ctx)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        h = _VP()
        rc = lib().sgb_ctx_create(device, hbm_budget, ctypes.byref(h))
        if rc:
            raise SGBError(rc, f"sgb_ctx_create(device={device}) failed: "
                               f"{lib().sgb_status_string(rc).decode()}")
        self.h = h

    def check(self, rc: int, what: str = ""):
        if rc < 0:
            raise SGBError(rc, f"{what}: {lib().sgb_last_error(self.h).decode()}")
        return rc

    def synchronize(self):
        self.check(lib().sgb_ctx_synchronize(self.h), "synchronize")

    def set_density_solver(self, solver: int):
        """SOLVER_PURIFY (default), SOLVER_JACOBI or SOLVER_PURIFY_MIXED for the SCF steps of
        later calls."""
        self.check(lib().sgb_ctx_set_density_solver(self.h, int(solver)), "set_density_solver")

    def set_class_threads(self, threads):
        """CTA size per size class for this context's batched launches (see size_classes)."""
        t = np.ascontiguousarray(threads, np.int32)
        self.check(lib().sgb_ctx_set_class_threads(self.h, len(t), _i(t)), "set_class_threads")

    def set_priority(self, high: bool = True):
        """Launches of this context at the device's greatest stream priority (or the default):
        its blocks go to freed SMs before other contexts' waiting blocks."""
        self.check(lib().sgb_ctx_set_priority(self.h, int(bool(high))), "sgb_ctx_set_priority")

    def set_diis(self, depth: int):
        """Pulay DIIS of this depth (2..8; 0 = off) for this context's SCF runs (batched
        launches and single molecules alike); step counts then differ from the reference's."""
        self.check(lib().sgb_ctx_set_diis(self.h, int(depth)), "set_diis")

    def electronic_energy(self, H, F, P) -> float:
        """E_el = 1/2 sum P (H + F) of packed matrices (ElectronicEnergy::ComputeEnergy),
        reduced on the device."""
        H, F, P = (np.ascontiguousarray(x, np.float64) for x in (H, F, P))
        n = int((np.sqrt(8 * len(H) + 1) - 1) / 2)
        if not (len(H) == len(F) == len(P) == n * (n + 1) // 2):
            raise ValueError("H, F, P must be packed triangles of one order")
        e = ctypes.c_double()
        self.check(lib().sgb_electronic_energy(self.h, n, _d(H), _d(F), _d(P), ctypes.byref(e)),
                   "sgb_electronic_energy")
        return e.value

    def set_grid_config(self, config: int):
        """Tile configuration of the whole-GPU purification (index into grid_configs(); -1 =
        chosen by size)."""
        self.check(lib().sgb_ctx_set_grid_config(self.h, int(config)), "set_grid_config")

    def set_damping(self, factor: float):
        """Density damping 0 <= factor < 1 (0 = off): P = (1 - f) P_new + f P_old each step."""
        self.check(lib().sgb_ctx_set_damping(self.h, float(factor)), "set_damping")

    def set_limits(self, max_sweeps: int = 0, wait_spins: int = -1):
        """Jacobi sweeps per eigensolve (0 = default) and polls of each bounded device wait
        (< 0 = default); small values exercise the failure paths."""
        self.check(lib().sgb_ctx_set_limits(self.h, int(max_sweeps), int(wait_spins)),
                   "set_limits")

    def barrier_timeout_probe(self, blocks: int, extra: int, spins: int) -> bool:
        """Launches a grid barrier that expects `extra` more blocks than it has; True when it
        reported its timeout (see sgb_diag_barrier_timeout)."""
        out = ctypes.c_int()
        self.check(lib().sgb_diag_barrier_timeout(self.h, int(blocks), int(extra), int(spins),
                                                  ctypes.byref(out)), "barrier probe")
        return bool(out.value)

    def set_sm_share(self, share: float):
        """Batched launches of this context use at most this fraction of the SMs."""
        self.check(lib().sgb_ctx_set_sm_share(self.h, float(share)), "set_sm_share")

    def reserve(self, nbytes: int):
        """Reusable device arena for batches of up to `nbytes` (see sgb_ctx_reserve)."""
        self.check(lib().sgb_ctx_reserve(self.h, int(nbytes)), "sgb_ctx_reserve")

    @property
    def bytes_in_use(self) -> int:
        return int(lib().sgb_ctx_bytes_in_use(self.h))

    def close(self):
        if getattr(self, "h", None):
            lib().sgb_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Molecule:
    """One molecule on the device, driven stage by stage like the reference CLI."""

    def __init__(self, ctx: Context, Z, xyz):
        self.ctx = ctx
        self.Z = np.ascontiguousarray(Z, np.int32)
        self.xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1)
        h = _VP()
        ctx.check(lib().sgb_mol_create(ctx.h, len(self.Z), _i(self.Z), _d(self.xyz),
                                       ctypes.byref(h)), "sgb_mol_create")
        self.h = h
        na, nao, nocc, nb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        lib().sgb_mol_info(h, ctypes.byref(na), ctypes.byref(nao), ctypes.byref(nocc),
                           ctypes.byref(nb))
        self.natoms, self.nao, self.nocc, self.nblocks = na.value, nao.value, nocc.value, nb.value

    @classmethod
    def from_geometry(cls, ctx: Context, mol: geometry.Molecule) -> "Molecule":
        return cls(ctx, mol.Z, mol.xyz)

    def set_path(self, path: int):
        """PATH_AUTO, PATH_CTA (one CTA per molecule, nao <= 1024) or PATH_GRID (whole GPU)."""
        self.ctx.check(lib().sgb_mol_set_path(self.h, path), "sgb_mol_set_path")

    def two_center(self):
        self.ctx.check(lib().sgb_two_center(self.ctx.h, self.h), "sgb_two_center")

    def hcore(self):
        self.ctx.check(lib().sgb_hcore(self.ctx.h, self.h), "sgb_hcore")

    def scf(self, tol: float = 5e-3, max_iter: int = 100) -> dict:
        r = _ScfResult()
        en = np.zeros(max_iter + 1)
        rc = lib().sgb_scf(self.ctx.h, self.h, tol, max_iter, ctypes.byref(r), _d(en))
        self.ctx.check(rc, "sgb_scf")
        return {"E_el": r.e_el, "n_iter": r.n_iter, "converged": bool(r.converged),
                "status": r.status, "energies": en[: r.n_iter + 1]}

    def core_core(self) -> float:
        e = ctypes.c_double()
        self.ctx.check(lib().sgb_core_core(self.ctx.h, self.h, ctypes.byref(e)), "sgb_core_core")
        return e.value

    def fock(self, P):
        P = np.ascontiguousarray(P, np.float64)
        F = np.zeros(self.nao * (self.nao + 1) // 2)
        e = ctypes.c_double()
        self.ctx.check(lib().sgb_fock(self.ctx.h, self.h, _d(P), _d(F), ctypes.byref(e)), "sgb_fock")
        return F, e.value

    def get(self, which: int) -> np.ndarray:
        n = self.nao
        size = {BLOCKS: self.nblocks, HCORE: n * (n + 1) // 2, FOCK: n * (n + 1) // 2,
                DENSITY: n * (n + 1) // 2, EIGVAL: n, EIGVEC: n * n}[which]
        out = np.zeros(size)
        self.ctx.check(lib().sgb_get(self.ctx.h, self.h, which, _d(out), size), "sgb_get")
        return out

    def run(self, tol: float = 5e-3, max_iter: int = 100) -> dict:
        """All stages in the reference CLI's order (semiGPU.cc:58-95)."""
        self.two_center()
        self.hcore()
        r = self.scf(tol, max_iter)
        r["E_cc"] = self.core_core()
        r["E_tot"] = r["E_el"] + r["E_cc"]
        r["dHf_kcal"] = heat_of_formation(self.Z, r["E_tot"])
        return r

    def close(self):
        if getattr(self, "h", None):
            lib().sgb_mol_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _concat(mols):
    """natoms, Z and xyz of all molecules as flat arrays (one gather per array: the host-side
    cost of a 4096-molecule call is about 2 ms)."""
    zs = [m.Z for m in mols]
    natoms = np.fromiter(map(len, zs), np.int32, count=len(zs))
    Z = np.ascontiguousarray(np.concatenate(zs), np.int32)
    xyz = np.ascontiguousarray(np.concatenate([m.xyz for m in mols]), np.float64).reshape(-1)
    return natoms, Z, xyz


class Batch:
    """Many molecules resident on the device, run by one persistent launch."""

    def __init__(self, ctx: Context, mols):
        self.ctx = ctx
        self.natoms, self.Z, self.xyz = _concat(mols)
        self.nmol = len(mols)
        h = _VP()
        ctx.check(lib().sgb_batch_create(ctx.h, self.nmol, _i(self.natoms), _i(self.Z),
                                         _d(self.xyz), ctypes.byref(h)), "sgb_batch_create")
        self.h = h

    def set_coordinates(self, xyz):
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1)
        self.ctx.check(lib().sgb_batch_set_coordinates(self.ctx.h, self.h, _d(xyz)), "set_coordinates")

    def run(self, tol: float = 1e-6, max_iter: int = 100):
        self.ctx.check(lib().sgb_batch_run(self.ctx.h, self.h, tol, max_iter), "sgb_batch_run")

    def results(self) -> dict:
        n = self.nmol
        eel, ecc = np.zeros(n), np.zeros(n)
        it, cv, st = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n, np.int32)
        self.ctx.check(lib().sgb_batch_results(self.ctx.h, self.h, _d(eel), _d(ecc), _i(it),
                                               _i(cv), _i(st)), "sgb_batch_results")
        return {"E_el": eel, "E_cc": ecc, "E_tot": eel + ecc, "n_iter": it,
                "converged": cv.astype(bool), "status": st}

    def launches(self) -> int:
        """Kernel launches per run (one persistent launch per occupied size class)."""
        n = ctypes.c_int()
        lib().sgb_batch_launches(self.h, ctypes.byref(n))
        return n.value

    def last_ms(self) -> float:
        ms = ctypes.c_float()
        lib().sgb_batch_last_ms(self.h, ctypes.byref(ms))
        return ms.value

    def timestamps(self):
        """(t_begin, t_end) per molecule in ns of the device clock, last run."""
        tb = np.zeros(self.nmol, np.uint64)
        te = np.zeros(self.nmol, np.uint64)
        P = ctypes.POINTER(ctypes.c_ulonglong)
        self.ctx.check(lib().sgb_batch_timestamps(self.ctx.h, self.h, tb.ctypes.data_as(P),
                                                  te.ctypes.data_as(P)), "timestamps")
        return tb, te

    STAGES = ("integrals", "hcore", "fock", "warm_gemm", "jacobi", "eigval_sort", "density",
              "core_core", "purify", "sweeps", "bipartite_solves", "full_solves",
              "purify_products")
    TIMED_STAGES = 9  # the first nine are SM cycles, the rest counts

    def set_profiling(self, on: bool = True):
        lib().sgb_batch_set_profiling(self.h, int(on))

    def stage_cycles(self) -> np.ndarray:
        """(nmol, 13): per-stage SM cycles of the last run (the first TIMED_STAGES columns),
        then counts (Jacobi sweeps, occupied-virtual eigensolves, full eigensolves,
        purification products)."""
        out = np.zeros((self.nmol, len(self.STAGES)), np.uint64)
        self.ctx.check(lib().sgb_batch_stage_cycles(
            self.ctx.h, self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_ulonglong))),
            "stage_cycles")
        return out

    def device_coordinates(self) -> int:
        p = _VP()
        lib().sgb_batch_device_coordinates(self.h, ctypes.byref(p))
        return p.value

    def close(self):
        if getattr(self, "h", None):
            lib().sgb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_molecules(ctx: Context, mols, tol: float = 1e-6, max_iter: int = 100) -> dict:
    """Host arrays in, per-molecule results out (sgb_run_molecules)."""
    natoms, Z, xyz = _concat(mols)
    n = len(mols)
    eel, ecc = np.zeros(n), np.zeros(n)
    it, cv, st = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n, np.int32)
    ctx.check(lib().sgb_run_molecules(ctx.h, n, _i(natoms), _i(Z), _d(xyz), tol, max_iter,
                                      _d(eel), _d(ecc), _i(it), _i(cv), _i(st)), "sgb_run_molecules")
    return {"E_el": eel, "E_cc": ecc, "E_tot": eel + ecc, "n_iter": it,
            "converged": cv.astype(bool), "status": st}


def gradient(ctx: Context, mol, tol: float = 1e-9, max_iter: int = 200, step: float = 1e-4):
    """(E_tot, dE_tot/dxyz in eV/Angstrom, shape (natoms, 3)) by central differences, the 6N
    displaced geometries in one batched launch (sgb_gradient)."""
    Z = np.ascontiguousarray(mol.Z, np.int32)
    xyz = np.ascontiguousarray(mol.xyz, np.float64).reshape(-1)
    g = np.zeros_like(xyz)
    e = ctypes.c_double()
    rc = lib().sgb_gradient(ctx.h, len(Z), _i(Z), _d(xyz), tol, max_iter, step, ctypes.byref(e),
                            _d(g))
    if rc != 0:  # the SCF statuses (a geometry that stopped or did not converge) are positive
        raise SGBError(rc, f"sgb_gradient: {lib().sgb_status_string(rc).decode()}: "
                           f"{lib().sgb_last_error(ctx.h).decode()}")
    return e.value, g.reshape(-1, 3)


def optimize(ctx, mol, gtol: float = 0.02, max_steps: int = 50, tol: float = 1e-9,
             step: float = 1e-4, max_move: float = 0.2, energy_gradient=None):
    """Geometry optimisation (BFGS on the Cartesian coordinates, moves capped at max_move
    Angstrom, backtracking when the energy rises) with the finite-difference gradients of
    `gradient`; stops when every gradient component is below gtol eV/Angstrom.  A caller may
    pass energy_gradient(molecule) -> (E_tot, gradient) instead of a context.  Returns
    (optimised geometry, E_tot, max |gradient|, steps)."""
    x = np.ascontiguousarray(mol.xyz, np.float64).reshape(-1).copy()
    n = x.size
    if energy_gradient is None:
        def energy_gradient(m):
            return gradient(ctx, m, tol=tol, step=step)

    def eg(xx):
        return energy_gradient(geometry.Molecule(mol.Z, xx.reshape(-1, 3)))

    e, g = eg(x)
    g = g.reshape(-1)
    Hinv = np.eye(n) / 50.0  # eV / Angstrom^2 scale of bond stretches
    it = 0
    for it in range(1, max_steps + 1):
        if np.max(np.abs(g)) < gtol:
            it -= 1
            break
        p = -Hinv @ g
        big = np.max(np.abs(p))
        if big > max_move:
            p *= max_move / big
        alpha = 1.0
        while True:
            xn = x + alpha * p
            en, gn = eg(xn)
            gn = gn.reshape(-1)
            if en <= e + 1e-4 * alpha * float(g @ p) or alpha < 1e-3:
                break
            alpha *= 0.5
        s_, y = xn - x, gn - g
        sy = float(s_ @ y)
        if sy > 1e-10:  # BFGS update of the inverse Hessian
            rho = 1.0 / sy
            I = np.eye(n)
            Hinv = (I - rho * np.outer(s_, y)) @ Hinv @ (I - rho * np.outer(y, s_)) + rho * np.outer(s_, s_)
        x, e, g = xn, en, gn
    return geometry.Molecule(mol.Z, x.reshape(-1, 3)), e, float(np.max(np.abs(g))), it
