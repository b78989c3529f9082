"""Molecule-level data parallelism across GPUs (one process per GPU).

The MNDO path has no exchange step between molecules, so a multi-GPU run is a partition of the
molecule list over ranks plus a gather of per-molecule scalars at the end; no collective touches
the data path.  Partitioning is longest-processing-time-first on an estimated cost (the SCF's
O(nao^3) eigensolves dominate), which keeps ranks within one large molecule of each other.
"""
from __future__ import annotations

import heapq

import numpy as np


def estimated_cost(mol) -> float:
    """Relative cost of one molecule's SCF: ~nao^3 eigensolve work plus the O(natoms^2) pair work."""
    n = mol.nao
    return float(n) ** 3 + 50.0 * mol.natoms ** 2


def partition(mols, world: int) -> list[list[int]]:
    """Molecule indices per rank, greedy longest-first onto the least-loaded rank.  Every rank
    computes the same partition from the same list (deterministic, no communication)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(mols)), key=lambda i: (-estimated_cost(mols[i]), i))
    heap = [(0.0, r) for r in range(world)]
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + estimated_cost(mols[i]), r))
    for p in parts:
        p.sort()
    return parts


# dtypes of the per-molecule results run_sharded gathers (fixed, so that a rank with no
# molecules sends arrays of the same types as the others)
RESULT_DTYPES = {"E_el": np.float64, "E_cc": np.float64, "n_iter": np.int32,
                 "converged": np.bool_, "status": np.int32}


def gather_results(local: dict, indices, total: int, group=None, dtypes=None) -> dict:
    """Collects per-molecule result arrays from every rank into full-length arrays on every rank
    (torch.distributed all_gather_object of the small per-molecule scalars).

    The output dtype of each key is dtypes[key] when given, else that of the first rank whose
    array for it is non-empty (a rank without molecules sends empty lists, whose own dtype
    would be float64)."""
    import torch.distributed as dist

    payload = {"idx": list(indices),
               **{k: {"dtype": np.asarray(v).dtype.str, "v": np.asarray(v).tolist()}
                  for k, v in local.items()}}
    if dist.is_available() and dist.is_initialized():
        out = [None] * dist.get_world_size(group)
        dist.all_gather_object(out, payload, group=group)
    else:
        out = [payload]
    keys = [k for k in local]
    full = {}
    for k in keys:
        dt = (dtypes or {}).get(k)
        if dt is None:
            dt = next((np.dtype(p[k]["dtype"]) for p in out if p[k]["v"]),
                      np.asarray(local[k]).dtype)
        full[k] = np.zeros(total, dtype=dt)
    for p in out:
        for k in keys:
            if p["idx"]:
                full[k][p["idx"]] = p[k]["v"]
    return full


def run_sharded(ctx, mols, tol: float = 1e-6, max_iter: int = 100, group=None,
                runner=None) -> dict:
    """This rank's share of `mols` through the batched path, gathered on every rank.

    runner(ctx, mols, tol=, max_iter=) -> dict of per-molecule arrays (E_el, E_cc, n_iter,
    converged, status); the default is the CUDA batch (semigpu_b200.run_molecules).  Tests on
    CPU pass a host stand-in so the partition -> run -> gather path runs without a GPU."""
    import torch.distributed as dist

    if runner is None:
        from . import run_molecules as runner

    world = dist.get_world_size(group) if dist.is_available() and dist.is_initialized() else 1
    rank = dist.get_rank(group) if world > 1 else 0
    mine = partition(mols, world)[rank]
    if mine:
        local = runner(ctx, [mols[i] for i in mine], tol=tol, max_iter=max_iter)
        keep = {k: np.asarray(local[k], RESULT_DTYPES[k]) for k in RESULT_DTYPES}
    else:
        keep = {k: np.zeros(0, dt) for k, dt in RESULT_DTYPES.items()}
    return gather_results(keep, mine, len(mols), group=group, dtypes=RESULT_DTYPES)
