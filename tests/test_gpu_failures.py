"""Failure paths, exercised without faulting, trapping or hanging the GPU.

The reference reports two failures: LAPACK's info > 0 (print and break,
src/common/scfcalculation.cpp:87-93) and an SCF that does not converge within its step cap
(energyConverge = false, :78).  Here: a Jacobi sweep cap that runs out (SGB_E_EIG), a step cap
(converged == 0 with status OK), a non-finite input (SGB_E_NAN), and the bounded device waits --
a grid barrier that can never complete, and a tensor-core MMA wait with no polls -- which end
with an error status or a fallback instead of a hang.  Density damping (the SCF-loop option
next to DIIS) is checked here too: same converged energy as the plain loop."""
from __future__ import annotations

import numpy as np
import pytest

import semigpu_b200 as sg
from semigpu_b200 import geometry as geo

pytestmark = pytest.mark.gpu


@pytest.fixture()
def ctx():
    c = sg.Context(0)
    yield c
    c.close()


def _alkane(n, seed=3):
    return geo.alkane(n, np.random.default_rng(seed))


def test_grid_barrier_times_out_and_returns(ctx):
    """A barrier expecting one block more than the grid has: every block gives up after its
    poll limit and the launch ends; the same barrier with the right count completes."""
    assert ctx.barrier_timeout_probe(blocks=8, extra=1, spins=2000) is True
    assert ctx.barrier_timeout_probe(blocks=8, extra=0, spins=2000) is False
    # the context is still usable afterwards
    r = sg.Molecule.from_geometry(ctx, geo.ring_c1()).run(tol=1e-6)
    assert r["status"] == sg.OK and r["converged"]


@pytest.mark.parametrize("path", [sg.PATH_CTA, sg.PATH_GRID])
def test_nan_coordinate_reports_nan(ctx, path):
    m = geo.ring_c1()
    xyz = m.xyz.copy()
    xyz[3, 1] = np.nan
    mol = sg.Molecule(ctx, m.Z, xyz)
    mol.set_path(path)
    mol.two_center()
    mol.hcore()
    r = mol.scf(tol=1e-6, max_iter=50)
    assert r["status"] == sg.E_NAN
    assert not r["converged"] and r["n_iter"] == 0


def test_nan_coordinate_in_a_batch_stops_only_that_molecule(ctx):
    mols = geo.batch_c3(12, seed=5)
    bad = geo.Molecule(mols[4].Z, mols[4].xyz.copy())
    bad.xyz[0, 0] = np.nan
    mols[4] = bad
    r = sg.run_molecules(ctx, mols, tol=1e-6)
    assert r["status"][4] == sg.E_NAN and not r["converged"][4]
    others = [i for i in range(12) if i != 4]
    assert (r["status"][others] == sg.OK).all() and r["converged"][others].all()


@pytest.mark.parametrize("path", [sg.PATH_CTA, sg.PATH_GRID])
def test_step_cap_reports_not_converged(ctx, path):
    """max_iter = 2: two SCF steps, converged == 0, status OK (the reference's
    energyConverge = false)."""
    mol = sg.Molecule.from_geometry(ctx, geo.ring_c1())
    mol.set_path(path)
    mol.two_center()
    mol.hcore()
    r = mol.scf(tol=1e-6, max_iter=2)
    assert r["status"] == sg.OK
    assert not r["converged"] and r["n_iter"] == 2
    assert len(r["energies"]) == 3 and np.isfinite(r["energies"]).all()


@pytest.mark.parametrize("path", [sg.PATH_CTA, sg.PATH_GRID])
def test_jacobi_sweep_cap_reports_eig_failure(ctx, path):
    """One Jacobi sweep per eigensolve cannot converge a cold start: SGB_E_EIG, as the
    reference stops on LAPACK info > 0."""
    ctx.set_density_solver(sg.SOLVER_JACOBI)
    ctx.set_limits(max_sweeps=1)
    mol = sg.Molecule.from_geometry(ctx, _alkane(6))
    mol.set_path(path)
    mol.two_center()
    mol.hcore()
    r = mol.scf(tol=1e-6, max_iter=20)
    assert r["status"] == sg.E_EIG
    assert not r["converged"]
    ctx.set_limits()  # defaults again: the same molecule converges
    mol2 = sg.Molecule.from_geometry(ctx, _alkane(6))
    mol2.set_path(path)
    r2 = mol2.run(tol=1e-6)
    assert r2["status"] == sg.OK and r2["converged"]


def test_tensor_wait_without_polls_falls_back_to_jacobi(ctx):
    """Mixed precision on nao 65-160 waits for tcgen05 MMAs through an mbarrier.  With zero
    polls every wait gives up at once: the step's purification is abandoned (after a second,
    full-length wait for the MMAs in flight, before the tensor memory is freed) and the step is
    diagonalised instead.  The energies are then the FP64 Jacobi ones."""
    mols = [_alkane(20, 1), _alkane(26, 2)]  # 122 and 158 AOs: both tensor-core forms
    assert all(65 <= m.nao <= 160 for m in mols)
    ref = sg.run_molecules(ctx, mols, tol=1e-6)
    ctx.set_density_solver(sg.SOLVER_PURIFY_MIXED)
    ctx.set_limits(wait_spins=0)
    b = sg.Batch(ctx, mols)
    b.set_profiling(True)
    b.run(1e-6)
    r = b.results()
    cyc = b.stage_cycles()
    b.close()
    ctx.set_limits()
    ctx.set_density_solver(sg.SOLVER_PURIFY)
    assert (r["status"] == sg.OK).all() and r["converged"].all()
    np.testing.assert_allclose(r["E_tot"], ref["E_tot"], rtol=0, atol=1e-6)
    # no purification finished (products count only for accepted purifications); every step
    # took a full Jacobi eigensolve
    full_jacobi = cyc[:, 11]
    assert (full_jacobi >= r["n_iter"]).all()


@pytest.mark.parametrize("path", [sg.PATH_CTA, sg.PATH_GRID])
def test_damping_reaches_the_same_energy(ctx, path):
    m = _alkane(8)
    plain = sg.Molecule.from_geometry(ctx, m)
    plain.set_path(path)
    r0 = plain.run(tol=1e-8)
    ctx.set_damping(0.3)
    damped = sg.Molecule.from_geometry(ctx, m)
    damped.set_path(path)
    r1 = damped.run(tol=1e-8)
    ctx.set_damping(0.0)
    assert r1["status"] == sg.OK and r1["converged"]
    assert abs(r1["E_tot"] - r0["E_tot"]) < 1e-6
    # the first step's density is mixed with the guess, so the trajectories differ
    assert abs(r1["energies"][1] - r0["energies"][1]) > 1e-3


def test_damping_in_a_batch(ctx):
    mols = geo.batch_c3(64, seed=8)
    r0 = sg.run_molecules(ctx, mols, tol=1e-8)
    ctx.set_damping(0.25)
    r1 = sg.run_molecules(ctx, mols, tol=1e-8)
    ctx.set_damping(0.0)
    assert r1["converged"].all()
    np.testing.assert_allclose(r1["E_tot"], r0["E_tot"], rtol=0, atol=1e-6)
