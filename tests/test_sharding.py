"""Molecule sharding over ranks (host logic), including a 2-rank gloo run on CPU."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from semigpu_b200 import geometry as geo
from semigpu_b200 import sharding


def test_partition_covers_every_molecule_once():
    mols = geo.batch_c3(300, seed=4)
    for world in (1, 2, 3, 8):
        parts = sharding.partition(mols, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(mols)))
        loads = [sum(sharding.estimated_cost(mols[i]) for i in p) for p in parts]
        biggest = max(sharding.estimated_cost(m) for m in mols)
        assert max(loads) - min(loads) <= biggest + 1e-9  # LPT bound


def test_partition_is_deterministic():
    mols = geo.batch_c3(64, seed=9)
    assert sharding.partition(mols, 4) == sharding.partition(mols, 4)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mols = geo.batch_c3(40, seed=1)
        mine = sharding.partition(mols, world)[rank]
        # stand-in per-molecule results computed on the host: nao and a rank tag
        local = {"nao": np.array([mols[i].nao for i in mine], np.int64),
                 "who": np.full(len(mine), rank, np.int64)}
        full = sharding.gather_results(local, mine, len(mols))
        out[rank] = (full["nao"].tolist(), full["who"].tolist())
    finally:
        dist.destroy_process_group()


def _oracle_runner(ctx, mols, tol=1e-6, max_iter=100):
    """CPU stand-in for the CUDA batch: the C restatement of the reference's SCF."""
    import oracle

    out = {k: [] for k in ("E_el", "E_cc", "n_iter", "converged", "status")}
    for m in mols:
        r = oracle.scf(m.Z, m.xyz, tol=tol, max_iter=max_iter)
        out["E_el"].append(r["E_el"])
        out["E_cc"].append(r["E_cc"])
        out["n_iter"].append(r["n_iter"])
        out["converged"].append(r["converged"])
        out["status"].append(0)
    return out


def _sharded_worker(rank, world, port, nmol, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mols = geo.batch_c3(nmol, seed=2)
        full = sharding.run_sharded(None, mols, tol=1e-6, runner=_oracle_runner)
        out[rank] = {k: (v.dtype.str, v.tolist()) for k, v in full.items()}
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nmol", [6, 1])
def test_two_rank_run_sharded_gloo(oracle_mod, nmol):
    """partition -> run -> gather over 2 gloo ranks with the oracle as the runner; with one
    molecule, rank 1 has none and must still gather the same dtypes."""
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_sharded_worker, args=(world, _free_port(), nmol, out), nprocs=world, join=True)
    mols = geo.batch_c3(nmol, seed=2)
    ref = _oracle_runner(None, mols)
    for r in range(world):
        got = out[r]
        assert got == out[0]  # every rank holds the same gathered arrays
        assert got["n_iter"][0] == np.dtype(np.int32).str
        assert got["status"][0] == np.dtype(np.int32).str
        assert got["converged"][0] == np.dtype(np.bool_).str
        assert got["n_iter"][1] == ref["n_iter"]
        np.testing.assert_array_equal(got["E_el"][1], ref["E_el"])
        assert all(got["converged"][1])


def test_two_rank_gather_gloo():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    mols = geo.batch_c3(40, seed=1)
    parts = sharding.partition(mols, world)
    for r in range(world):
        nao, who = out[r]
        assert nao == [m.nao for m in mols]
        for rr, p in enumerate(parts):
            assert all(who[i] == rr for i in p)
