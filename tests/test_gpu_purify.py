"""Density by purification (default solver) against the Jacobi eigensolver and the goldens."""
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


@pytest.fixture
def jacobi_ctx():
    ctx = sg.Context(0)
    ctx.set_density_solver(sg.SOLVER_JACOBI)
    yield ctx
    ctx.close()


def test_solvers_agree_on_mixed_batch(gpu_ctx, jacobi_ctx):
    mols = geo.batch_c3(192, seed=21)
    a = sg.run_molecules(gpu_ctx, mols, tol=1e-6)
    b = sg.run_molecules(jacobi_ctx, mols, tol=1e-6)
    assert np.all(a["status"] == 0) and np.all(b["status"] == 0)
    np.testing.assert_array_equal(a["n_iter"], b["n_iter"])
    np.testing.assert_allclose(a["E_el"], b["E_el"], rtol=0, atol=1e-9)
    np.testing.assert_array_equal(a["E_cc"], b["E_cc"])


def test_purified_density_and_eigenpairs_match_golden(gpu_ctx):
    """Single-molecule path: the density comes from purification, the eigenvalues from one
    Jacobi at the end; both equal the reference's."""
    m_npz = np.load(os.path.join(GOLDEN, "reference_matrices.npz"))
    keys = sorted({k.rsplit("/", 1)[0] for k in m_npz.files})[::5]
    for key in keys:
        c = CASES[key]
        m = sg.Molecule(gpu_ctx, np.array(c["Z"], np.int32), np.array(c["xyz"]))
        m.set_path(sg.PATH_CTA)
        m.two_center()
        m.hcore()
        r = m.scf(tol=c["tol"], max_iter=100)
        assert r["n_iter"] == c["n_iter"], key
        np.testing.assert_allclose(m.get(sg.DENSITY), m_npz[f"{key}/P"], rtol=0, atol=1e-8)
        np.testing.assert_allclose(m.get(sg.EIGVAL), m_npz[f"{key}/eig"], rtol=0, atol=1e-8)


def test_every_size_class_purifies(gpu_ctx):
    """Padded orders 16 .. 160 (one to four super-tiles per warp, 128- to 512-thread CTAs) all
    converge by purification."""
    rng = np.random.default_rng(3)
    mols = [geo.alkane(k, rng) for k in (1, 2, 5, 7, 10, 12, 15, 20, 24, 26)]
    mols += [geo.polyene(k, rng) for k in (10, 20, 26, 30)]
    assert sorted({(m.nao + 15) // 16 * 16 for m in mols}) == list(range(16, 161, 16))
    b = sg.Batch(gpu_ctx, mols)
    b.set_profiling(True)
    b.run(1e-6)
    r = b.results()
    sc = b.stage_cycles()
    st = sg.Batch.STAGES
    assert np.all(r["status"] == 0) and np.all(r["converged"])
    assert np.all(sc[:, st.index("full_solves")] == 0)  # no Jacobi fallback
    assert np.all(sc[:, st.index("purify_products")] >= 10 * r["n_iter"])


def test_zero_gap_falls_back_to_jacobi(gpu_ctx):
    """Square cyclobutadiene: the degenerate pair of pi orbitals holds two electrons, so the
    HOMO-LUMO gap is zero by symmetry.  Purification cannot converge there; the step falls back
    to a Jacobi eigensolve and the run still completes."""
    a, ch = 1.45, 1.08
    ring = np.array([[a / 2, a / 2, 0], [-a / 2, a / 2, 0], [-a / 2, -a / 2, 0], [a / 2, -a / 2, 0]])
    out = ring / np.linalg.norm(ring, axis=1, keepdims=True)
    xyz = np.vstack([ring, ring + ch * out])
    mol = geo.Molecule([6, 6, 6, 6, 1, 1, 1, 1], xyz)
    b = sg.Batch(gpu_ctx, [mol])
    b.set_profiling(True)
    b.run(1e-6, max_iter=30)
    r = b.results()
    sc = b.stage_cycles()
    assert r["status"][0] == 0
    assert np.isfinite(r["E_el"][0])
    assert sc[0, sg.Batch.STAGES.index("full_solves")] >= 1


def test_grid_path_purification_matches_jacobi(gpu_ctx, jacobi_ctx):
    """One large molecule on the whole GPU: purification (DSYRK products) against the Jacobi
    eigensolver, then its eigenpairs (computed when first read) against the Jacobi ones."""
    mol = geo.alkane(40, np.random.default_rng(8))  # nao 242
    a = sg.Molecule.from_geometry(gpu_ctx, mol)
    b = sg.Molecule.from_geometry(jacobi_ctx, mol)
    ra, rb = a.run(tol=1e-6), b.run(tol=1e-6)
    assert ra["n_iter"] == rb["n_iter"]
    assert abs(ra["E_tot"] - rb["E_tot"]) < 1e-8
    np.testing.assert_allclose(a.get(sg.DENSITY), b.get(sg.DENSITY), rtol=0, atol=1e-9)
    np.testing.assert_allclose(a.get(sg.EIGVAL), b.get(sg.EIGVAL), rtol=0, atol=1e-8)


def test_mixed_precision_within_tolerance(gpu_ctx, oracle_mod):
    """Mixed form (FP32 products, FP64 finish) on C100H202 against the FP64 oracle:
    |dE_total| <= 1e-4 eV (the stated tolerance of the mixed form)."""
    mol = geo.alkane_c2(0)
    ctx = sg.Context(0)
    ctx.set_density_solver(sg.SOLVER_PURIFY_MIXED)
    try:
        r = sg.Molecule.from_geometry(ctx, mol).run(tol=1e-6)
    finally:
        ctx.close()
    o = oracle_mod.scf(mol.Z, mol.xyz, tol=1e-6)
    assert r["converged"] and r["status"] == 0
    assert abs(r["E_tot"] - o["E_tot"]) <= TOL_MIXED
    assert abs(r["n_iter"] - o["n_iter"]) <= 1


def test_diis_converges_to_the_same_energy_in_no_more_steps():
    """Optional DIIS on the grid path: same converged energy as the reference's plain loop
    (within its tolerance), and no more steps."""
    mol = geo.polyene(60, np.random.default_rng(12))  # nao 302, conjugated: slow plain SCF
    ctx = sg.Context(0)
    try:
        plain = sg.Molecule.from_geometry(ctx, mol).run(tol=1e-6, max_iter=100)
        ctx.set_diis(6)
        diis = sg.Molecule.from_geometry(ctx, mol).run(tol=1e-6, max_iter=100)
    finally:
        ctx.close()
    assert plain["converged"] and diis["converged"]
    assert diis["n_iter"] <= plain["n_iter"]
    assert abs(diis["E_tot"] - plain["E_tot"]) < 1e-5


TOL_MIXED = 1e-4  # eV: |E_tot(mixed) - E_tot(FP64 oracle)| per molecule


def _oracle_energies(oracle_mod, mols, tol=1e-6):
    """E_tot and step counts of the FP64 oracle (the C restatement of the reference)."""
    out = [oracle_mod.scf(m.Z, m.xyz, tol=tol) for m in mols]
    return np.array([o["E_tot"] for o in out]), np.array([o["n_iter"] for o in out])


def test_mixed_tensor_core_products_in_batch(gpu_ctx, oracle_mod):
    """Mixed form in the batch: nao 65-128 (one 128-row tile) purify with TF32 tcgen05 products
    (3xTF32) and an FP64 finish; every molecule converges within 1e-4 eV of the FP64 oracle,
    without a fallback."""
    rng = np.random.default_rng(17)
    mols = [geo.alkane(k, rng) for k in (11, 13, 15, 17, 19, 21)]  # nao 68 .. 128
    mols += [geo.polyene(k, rng) for k in (14, 18, 22, 24)]           # nao 72 .. 122
    assert all(64 < m.nao <= 128 for m in mols)
    ref_e, _ = _oracle_energies(oracle_mod, mols)
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
    np.testing.assert_allclose(r["E_tot"], ref_e, rtol=0, atol=TOL_MIXED)


def test_mixed_tensor_core_products_two_accumulators(gpu_ctx, oracle_mod):
    """nao 129-160 (n16 144 and 160): X taller than one 128-row tile, products from two
    tensor-memory accumulators plus symmetry; same bar as the single-tile form."""
    rng = np.random.default_rng(23)
    mols = [geo.alkane(k, rng) for k in (22, 23, 24, 25, 26)]  # nao 134 .. 158
    mols += [geo.polyene(k, rng) for k in (26, 28, 30)]         # nao 132 .. 152
    assert {(m.nao + 15) // 16 * 16 for m in mols} == {144, 160}
    ref_e, ref_it = _oracle_energies(oracle_mod, mols)
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
    np.testing.assert_allclose(r["E_tot"], ref_e, rtol=0, atol=TOL_MIXED)
    assert np.all(np.abs(r["n_iter"] - ref_it) <= 1)


def test_batched_diis_same_energies_in_fewer_steps(gpu_ctx):
    """Pulay DIIS in the batched launch (each CTA extrapolates its molecule's F): every molecule
    converges to the energy of the reference's plain loop (within its tolerance) and the batch
    needs fewer SCF steps; single molecules on one CTA take the same path."""
    mols = geo.batch_c3(160, seed=31)
    ref = sg.run_molecules(gpu_ctx, mols, tol=1e-6)
    ctx = sg.Context(0)
    try:
        ctx.set_diis(6)
        r = sg.run_molecules(ctx, mols, tol=1e-6)
        one = sg.Molecule.from_geometry(ctx, mols[7])
        one.set_path(sg.PATH_CTA)
        r1 = one.run(tol=1e-6)
        one.close()
    finally:
        ctx.close()
    assert np.all(r["status"] == 0) and np.all(r["converged"])
    np.testing.assert_allclose(r["E_tot"], ref["E_tot"], rtol=0, atol=1e-5)
    assert r["n_iter"].sum() < ref["n_iter"].sum()
    assert r1["converged"] and abs(r1["E_tot"] - ref["E_tot"][7]) < 1e-5
    assert r1["n_iter"] == r["n_iter"][7]


def test_mixed_precision_with_batched_diis(gpu_ctx, oracle_mod):
    """Both options at once (tensor-core products and DIIS in the same kernel instances):
    converged, within the mixed form's 1e-4 eV of the FP64 oracle's plain loop."""
    mols = geo.batch_c3(96, seed=41)
    assert any(64 < m.nao <= 160 for m in mols)
    ref = sg.run_molecules(gpu_ctx, mols, tol=1e-6)
    ref_e, _ = _oracle_energies(oracle_mod, mols)
    ctx = sg.Context(0)
    try:
        ctx.set_density_solver(sg.SOLVER_PURIFY_MIXED)
        ctx.set_diis(6)
        r = sg.run_molecules(ctx, mols, tol=1e-6)
    finally:
        ctx.close()
    assert np.all(r["status"] == 0) and np.all(r["converged"])
    np.testing.assert_allclose(r["E_tot"], ref_e, rtol=0, atol=TOL_MIXED)
    assert r["n_iter"].sum() < ref["n_iter"].sum()


def test_mixed_batch_composition_against_oracle(oracle_mod):
    """The bench batch's composition (every size class) in the mixed form: each molecule's
    E_tot within 1e-4 eV of the FP64 oracle, the error reported per molecule."""
    mols = geo.batch_c3(256, seed=0)
    ref_e, ref_it = _oracle_energies(oracle_mod, mols)
    ctx = sg.Context(0)
    try:
        ctx.set_density_solver(sg.SOLVER_PURIFY_MIXED)
        r = sg.run_molecules(ctx, mols, tol=1e-6)
    finally:
        ctx.close()
    assert np.all(r["status"] == 0) and np.all(r["converged"])
    err = np.abs(r["E_tot"] - ref_e)
    assert err.max() <= TOL_MIXED, (int(err.argmax()), float(err.max()))
    assert np.all(np.abs(r["n_iter"] - ref_it) <= 1)
