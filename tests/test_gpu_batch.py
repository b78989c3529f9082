"""Batched persistent path: same results as the single-molecule path and the references."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

import semigpu_b200 as sg
from semigpu_b200 import geometry as geo

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
with open(os.path.join(GOLDEN, "reference_cases.json")) as _fh:
    CASES = json.load(_fh)["cases"]


def test_batch_matches_golden(gpu_ctx):
    keys = sorted(k for k, v in CASES.items() if v["nao"] <= 160)
    mols = [geo.Molecule(CASES[k]["Z"], CASES[k]["xyz"]) for k in keys]
    tols = {CASES[k]["tol"] for k in keys}
    for tol in sorted(tols):
        sel = [i for i, k in enumerate(keys) if CASES[k]["tol"] == tol]
        r = sg.run_molecules(gpu_ctx, [mols[i] for i in sel], tol=tol, max_iter=100)
        for j, i in enumerate(sel):
            c = CASES[keys[i]]
            assert r["status"][j] == 0, keys[i]
            assert r["n_iter"][j] == c["n_iter"], keys[i]
            assert abs(r["E_el"][j] - c["E_el"]) < 1e-6, keys[i]
            assert abs(r["E_cc"][j] - c["E_cc"]) < 1e-6, keys[i]


def test_alone_equals_in_mix(gpu_ctx):
    """Each molecule's result is the same alone and inside a mixed batch."""
    mols = geo.batch_c3(48, seed=3)
    mix = sg.run_molecules(gpu_ctx, mols, tol=1e-6)
    for i in (0, 7, 19, 47):
        alone = sg.Molecule.from_geometry(gpu_ctx, mols[i]).run(tol=1e-6)
        assert alone["n_iter"] == mix["n_iter"][i]
        assert abs(alone["E_tot"] - mix["E_tot"][i]) < 1e-9


def test_batch_against_oracle(gpu_ctx, oracle_mod):
    mols = geo.batch_c3(256, seed=11)
    r = sg.run_molecules(gpu_ctx, mols, tol=1e-6)
    assert np.all(r["status"] == 0) and np.all(r["converged"])
    for i in range(0, 256, 8):
        o = oracle_mod.scf(mols[i].Z, mols[i].xyz, tol=1e-6)
        assert r["n_iter"][i] == o["n_iter"]
        assert abs(r["E_el"][i] - o["E_el"]) < 1e-6
        assert abs(r["E_cc"][i] - o["E_cc"]) < 1e-6


def test_batch_rerun_new_coordinates(gpu_ctx, oracle_mod):
    mols = geo.batch_c3(16, seed=5)
    b = sg.Batch(gpu_ctx, mols)
    b.run(1e-6)
    r1 = b.results()
    rng = np.random.default_rng(0)  # a random displacement (a uniform shift would not change E)
    moved = [geo.Molecule(m.Z, m.xyz + rng.normal(0.0, 0.02, m.xyz.shape)) for m in mols]
    b.set_coordinates(np.concatenate([m.xyz.reshape(-1) for m in moved]))
    b.run(1e-6)
    r2 = b.results()
    for i in (0, 9):
        o = oracle_mod.scf(moved[i].Z, moved[i].xyz, tol=1e-6)
        assert abs(r2["E_tot"][i] - o["E_tot"]) < 1e-6
    assert not np.allclose(r1["E_tot"], r2["E_tot"])
    assert b.last_ms() > 0


def test_high_priority_context_same_results(gpu_ctx):
    """sgb_ctx_set_priority replaces the context's streams; a batch on the high-priority streams
    (and again after going back to the default) gives the default context's results."""
    mols = geo.batch_c3(64, seed=5)
    ref = sg.run_molecules(gpu_ctx, mols, tol=1e-6)
    with sg.Context(0) as ctx:
        ctx.set_priority(True)
        hi = sg.run_molecules(ctx, mols, tol=1e-6)
        ctx.set_priority(False)
        lo = sg.run_molecules(ctx, mols, tol=1e-6)
    for r in (hi, lo):
        assert np.array_equal(r["n_iter"], ref["n_iter"])
        assert np.max(np.abs(r["E_tot"] - ref["E_tot"])) == 0.0
