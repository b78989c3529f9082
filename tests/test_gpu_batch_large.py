"""Batched path above nao 160: one CTA per molecule with its eigensolver columns streamed from
global memory, in the same launch as the small molecules."""
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


def test_c60_in_batch_matches_golden(gpu_ctx):
    """nao 240 inside a batch, reference at its 5e-3 default."""
    c = CASES["fixture/C60-Ih@0.005"]
    small = [geo.Molecule(CASES[k]["Z"], CASES[k]["xyz"])
             for k in sorted(CASES) if CASES[k]["tol"] == c["tol"] and CASES[k]["nao"] <= 60][:6]
    mols = small + [geo.Molecule(c["Z"], c["xyz"])]
    r = sg.run_molecules(gpu_ctx, mols, tol=c["tol"], max_iter=100)
    assert r["status"][-1] == 0
    assert r["n_iter"][-1] == c["n_iter"]
    assert abs(r["E_el"][-1] - c["E_el"]) < 1e-6
    assert abs(r["E_cc"][-1] - c["E_cc"]) < 1e-6


def test_large_in_mix_against_oracle(gpu_ctx, oracle_mod):
    rng = np.random.default_rng(7)
    large = [geo.alkane(27, rng), geo.polyene(40, rng), geo.alkane(50, rng)]
    assert [m.nao for m in large] == [164, 202, 302]
    mols = geo.batch_c3(40, seed=9) + large
    r = sg.run_molecules(gpu_ctx, mols, tol=1e-6)
    assert np.all(r["status"] == 0) and np.all(r["converged"])
    for i in range(len(mols) - 3, len(mols)):
        o = oracle_mod.scf(mols[i].Z, mols[i].xyz, tol=1e-6)
        assert r["n_iter"][i] == o["n_iter"], mols[i].nao
        assert abs(r["E_el"][i] - o["E_el"]) < 1e-6
        assert abs(r["E_cc"][i] - o["E_cc"]) < 1e-6


def test_large_batch_equals_grid_path(gpu_ctx):
    """The same molecule through the batch (one CTA) and the grid path (whole GPU)."""
    mol = geo.alkane(36, np.random.default_rng(4))  # nao 218
    r = sg.run_molecules(gpu_ctx, [mol], tol=1e-6)
    g = sg.Molecule.from_geometry(gpu_ctx, mol)
    g.set_path(sg.PATH_GRID)
    rg = g.run(tol=1e-6)
    assert r["n_iter"][0] == rg["n_iter"]
    assert abs(r["E_tot"][0] - rg["E_tot"]) < 1e-8


def test_single_molecule_cta_path_above_160(gpu_ctx):
    """PATH_CTA forced above nao 160 runs the streamed one-CTA eigensolver; matrices agree with
    the grid path."""
    mol = geo.polyene(44, np.random.default_rng(5))  # nao 222
    a = sg.Molecule.from_geometry(gpu_ctx, mol)
    a.set_path(sg.PATH_CTA)
    b = sg.Molecule.from_geometry(gpu_ctx, mol)
    b.set_path(sg.PATH_GRID)
    ra, rb = a.run(tol=1e-6), b.run(tol=1e-6)
    assert ra["n_iter"] == rb["n_iter"]
    assert abs(ra["E_tot"] - rb["E_tot"]) < 1e-8
    np.testing.assert_allclose(a.get(sg.DENSITY), b.get(sg.DENSITY), rtol=0, atol=1e-8)
    np.testing.assert_allclose(a.get(sg.EIGVAL), b.get(sg.EIGVAL), rtol=0, atol=1e-7)


def test_c100h202_in_batch_against_oracle(gpu_ctx, oracle_mod):
    """C100H202 (602 AOs) through the batched path."""
    mol = geo.alkane_c2(0)
    r = sg.run_molecules(gpu_ctx, [mol, geo.ring_c1()], tol=1e-6)
    o = oracle_mod.scf(mol.Z, mol.xyz, tol=1e-6)
    assert r["status"][0] == 0 and r["converged"][0]
    assert r["n_iter"][0] == o["n_iter"]
    assert abs(r["E_el"][0] - o["E_el"]) < 1e-6
    assert abs(r["E_cc"][0] - o["E_cc"]) < 1e-6


def test_large_fp64_tiles_without_fallback(oracle_mod):
    """FP64 above nao 160 in the batch through both tile shapes of the TMA-staged loop (64 x 64
    for nao 164 and 302, 128 x 128 for 202 and 452): the reference's energies and step counts,
    with every step's density from purification (a failed purification would fall back to the
    Jacobi eigensolve, which gives the same energies)."""
    rng = np.random.default_rng(19)
    mols = [geo.alkane(27, rng), geo.polyene(40, rng), geo.alkane(50, rng), geo.polyene(90, rng)]
    assert [m.nao for m in mols] == [164, 202, 302, 452]
    ctx = sg.Context(0)
    try:
        b = sg.Batch(ctx, mols)
        b.set_profiling(True)
        b.run(1e-6)
        r = b.results()
        sc = b.stage_cycles()
        b.close()
    finally:
        ctx.close()
    assert np.all(r["status"] == 0) and np.all(r["converged"])
    assert np.all(sc[:, sg.Batch.STAGES.index("full_solves")] == 0)
    for i, m in enumerate(mols):
        o = oracle_mod.scf(m.Z, m.xyz, tol=1e-6)
        assert r["n_iter"][i] == o["n_iter"], m.nao
        assert abs(r["E_tot"][i] - o["E_tot"]) < 1e-6, (m.nao, r["E_tot"][i] - o["E_tot"])


def test_large_mixed_tensor_core_against_oracle(oracle_mod):
    """Mixed form above nao 160 in the batch (one CTA per molecule): the TF32 tensor-core phase
    on TMA-staged hi / lo panels, then the FP64 tile loop; every molecule within 1e-4 eV of the
    FP64 oracle, with no Jacobi fallback."""
    rng = np.random.default_rng(19)
    mols = [geo.alkane(27, rng), geo.polyene(40, rng), geo.alkane(50, rng), geo.polyene(90, rng)]
    assert [m.nao for m in mols] == [164, 202, 302, 452]
    ctx = sg.Context(0)
    try:
        ctx.set_density_solver(sg.SOLVER_PURIFY_MIXED)
        b = sg.Batch(ctx, mols)
        b.set_profiling(True)
        b.run(1e-6)
        r = b.results()
        sc = b.stage_cycles()
        b.close()
    finally:
        ctx.close()
    assert np.all(r["status"] == 0) and np.all(r["converged"])
    assert np.all(sc[:, sg.Batch.STAGES.index("full_solves")] == 0)
    for i, m in enumerate(mols):
        o = oracle_mod.scf(m.Z, m.xyz, tol=1e-6)
        assert abs(r["E_tot"][i] - o["E_tot"]) <= 1e-4, (m.nao, r["E_tot"][i] - o["E_tot"])
        assert abs(r["n_iter"][i] - o["n_iter"]) <= 1
