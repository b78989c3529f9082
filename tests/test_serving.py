"""Serving scheduler (host logic) with a stand-in engine, and the real engine on the GPU."""
from __future__ import annotations

import threading
import time

import numpy as np
import pytest

from semigpu_b200 import geometry as geo
from semigpu_b200 import serving


def _fake_engine(delay=0.002, log=None):
    lock = threading.Lock()

    def run(ctx, mols, tol, max_iter):
        with lock:
            if log is not None:
                log.append(len(mols))
        time.sleep(delay)
        n = len(mols)
        return {"E_el": np.array([-float(m.nao) for m in mols]), "E_cc": np.zeros(n),
                "E_tot": np.array([-float(m.nao) for m in mols]), "n_iter": np.ones(n, np.int32),
                "converged": np.ones(n, bool), "status": np.zeros(n, np.int32)}
    return run


def test_every_request_answered_once_with_its_own_result():
    log = []
    srv = serving.Server(slots=3, engine=_fake_engine(log=log))
    try:
        mols = geo.batch_c3(300, seed=2)
        ids = [srv.submit(m) for m in mols]
        done = srv.drain(timeout=60)
    finally:
        srv.close()
    assert [r.rid for r in done] == ids
    for r, m in zip(done, mols):
        assert r.result["E_el"] == -float(m.nao)
        assert r.t_done >= r.t_arrival
    assert sum(log) == 300
    assert len(log) < 300  # requests were batched


def test_small_and_large_molecules_never_share_a_batch():
    """Molecules above nao 160 have their own queue and worker: a small request is never held
    in a batch with a large one."""
    batches = []
    lock = threading.Lock()
    inner = _fake_engine(delay=0.003)

    def engine(ctx, mols, tol, max_iter):
        with lock:
            batches.append([m.nao for m in mols])
        return inner(ctx, mols, tol, max_iter)

    rng = np.random.default_rng(4)
    mols = geo.batch_c3(120, seed=6) + [geo.alkane(int(k), rng) for k in (30, 45, 60, 80)]
    order = rng.permutation(len(mols))
    srv = serving.Server(slots=3, big_slots=1, engine=engine)
    try:
        for i in order:
            srv.submit(mols[i])
        done = srv.drain(timeout=60)
    finally:
        srv.close()
    assert len(done) == len(mols)
    for b in batches:
        assert all(n > serving.SMEM_MAX_NAO for n in b) or all(n <= serving.SMEM_MAX_NAO for n in b)
    assert any(all(n > serving.SMEM_MAX_NAO for n in b) for b in batches)


def test_whole_sm_molecules_have_their_own_queue():
    """With mid_slots, molecules of nao 129-160 (whole-SM CTAs) go to their own worker: no
    batch mixes them with smaller or larger molecules."""
    batches = []
    lock = threading.Lock()
    inner = _fake_engine(delay=0.003)

    def engine(ctx, mols, tol, max_iter):
        with lock:
            batches.append([m.nao for m in mols])
        return inner(ctx, mols, tol, max_iter)

    rng = np.random.default_rng(8)
    mid = [geo.alkane(int(k), rng) for k in (22, 24, 26)]  # nao 134, 146, 158
    assert all(serving.WHOLE_SM_NAO < m.nao <= serving.SMEM_MAX_NAO for m in mid)
    mols = geo.batch_c3(90, seed=7) + mid + [geo.alkane(int(k), rng) for k in (30, 45)]
    order = rng.permutation(len(mols))
    srv = serving.Server(slots=4, big_slots=1, mid_slots=1, engine=engine)
    try:
        for i in order:
            srv.submit(mols[i])
        done = srv.drain(timeout=60)
    finally:
        srv.close()
    assert len(done) == len(mols)

    def kind(n):
        return 1 if n > serving.SMEM_MAX_NAO else 2 if n > serving.WHOLE_SM_NAO else 0

    for b in batches:
        assert len({kind(n) for n in b}) == 1, b
    assert any(kind(b[0]) == 2 for b in batches)


def test_admission_respects_hbm_share():
    log = []
    mols = geo.batch_c3(50, seed=3)
    biggest = max(serving.device_bytes(m) for m in mols)
    srv = serving.Server(slots=1, hbm_budget=3 * biggest, engine=_fake_engine(delay=0.01, log=log))
    try:
        for m in mols:
            srv.submit(m)
        srv.drain(timeout=60)
    finally:
        srv.close()
    assert max(log) <= 50 and len(log) > 1


def test_open_loop_replay_and_stats():
    srv = serving.Server(slots=2, engine=_fake_engine(delay=0.001))
    try:
        arrivals = serving_arrivals = [(0.001 * i, m) for i, m in enumerate(geo.batch_c3(60, seed=5))]
        done = srv.replay(serving_arrivals)
    finally:
        srv.close()
    s = serving.stats(done)
    assert s["requests"] == 60 and s["p99_ms"] >= s["p50_ms"] > 0 and s["all_converged"]


@pytest.mark.gpu
def test_served_results_equal_alone():
    """Each molecule gives the same energy served in a mixed stream as computed alone."""
    import semigpu_b200 as sg

    mols = geo.batch_c3(96, seed=21)
    srv = serving.Server(slots=3, hbm_budget=2 << 30)
    try:
        arrivals = [(0.0005 * i, m) for i, m in enumerate(mols)]
        done = srv.replay(arrivals)
    finally:
        srv.close()
    assert len(done) == 96 and all(r.result["status"] == 0 for r in done)
    with sg.Context(0) as ctx:
        for i in (0, 13, 50, 95):
            alone = sg.Molecule.from_geometry(ctx, mols[i]).run(tol=1e-6)
            assert done[i].result["n_iter"] == alone["n_iter"]
            assert abs(done[i].result["E_tot"] - alone["E_tot"]) < 1e-9
    s = serving.stats(done)
    assert s["all_converged"] and s["p99_ms"] > 0


@pytest.mark.gpu
def test_served_mixed_precision_within_tolerance_of_fp64():
    """Serving in mixed precision (TF32 tensor-core products, FP64 finish): each result equals
    the same molecule run alone in mixed precision, and is within 1e-4 eV of FP64."""
    import semigpu_b200 as sg

    mols = geo.batch_c3(96, seed=22)
    srv = serving.Server(slots=3, hbm_budget=2 << 30, solver=sg.SOLVER_PURIFY_MIXED)
    try:
        done = srv.replay([(0.0005 * i, m) for i, m in enumerate(mols)])
    finally:
        srv.close()
    assert len(done) == 96 and all(r.result["status"] == 0 for r in done)
    assert serving.stats(done)["all_converged"]
    with sg.Context(0) as c64:
        fp64 = sg.run_molecules(c64, mols, tol=1e-6)
    e = np.array([r.result["E_tot"] for r in done])
    np.testing.assert_allclose(e, fp64["E_tot"], rtol=0, atol=1e-4)
    big = [i for i, m in enumerate(mols) if 64 < m.nao <= 160][:4]
    assert big  # the tensor-core form is exercised
    with sg.Context(0) as ctx:
        ctx.set_density_solver(sg.SOLVER_PURIFY_MIXED)
        for i in big:
            alone = sg.Molecule.from_geometry(ctx, mols[i]).run(tol=1e-6)
            assert done[i].result["n_iter"] == alone["n_iter"]
            assert abs(done[i].result["E_tot"] - alone["E_tot"]) < 1e-9


def test_stats_latency_by_arrival_quarter():
    """A backlog that grows shows as rising per-quarter p50; the drain is last result minus
    last arrival."""
    from semigpu_b200 import serving
    from semigpu_b200.geometry import Molecule

    m = Molecule([1, 1], [[0, 0, 0], [0.74, 0, 0]])
    reqs = []
    for i in range(40):
        r = serving.Request(i, m, t_arrival=0.1 * i)
        r.t_done = r.t_arrival + 0.01 * (1 + i // 10)  # 10, 20, 30, 40 ms by quarter
        r.result = {"converged": True}
        reqs.append(r)
    st = serving.stats(reqs)
    assert [round(v) for v in st["p50_ms_by_arrival_quarter"]] == [10, 20, 30, 40]
    assert abs(st["drain_ms"] - 40.0) < 1e-6
    assert st["requests"] == 40 and st["all_converged"]
