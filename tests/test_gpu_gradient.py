"""Finite-difference geometry gradients on the device (sgb_gradient: the molecule and its 6N
displaced copies as one batch) against the oracle's central differences at the same step.
Tolerance: 2e-3 eV/Angstrom per component -- each energy agrees with the oracle to about the
SCF tolerance (1e-9 eV here), divided by the 2e-4 Angstrom of the difference quotient."""
from __future__ import annotations

import numpy as np
import pytest

import semigpu_b200 as sg
from semigpu_b200 import geometry as geo

from test_optimizer import fd_gradient

pytestmark = pytest.mark.gpu


@pytest.fixture()
def ctx():
    c = sg.Context(0)
    yield c
    c.close()


CASES = {
    "formaldehyde": geo.Molecule([6, 8, 1, 1], [[0, 0, 0], [1.25, 0.05, 0], [-0.55, 0.95, 0.02],
                                                [-0.5, -0.9, -0.05]]),
    "hexane": geo.alkane(6, np.random.default_rng(5), jitter=0.05),
    "aza": geo.aza_ring((0, 2), np.random.default_rng(2), jitter=0.05),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_gradient_matches_oracle(ctx, oracle_mod, name):
    mol = CASES[name]
    e, g = sg.gradient(ctx, mol, tol=1e-9, step=1e-4)
    e_ref, g_ref = fd_gradient(oracle_mod, mol, step=1e-4, tol=1e-10)
    assert abs(e - e_ref) < 1e-6
    assert g.shape == (mol.natoms, 3)
    np.testing.assert_allclose(g, g_ref, atol=2e-3, rtol=0)
    assert np.max(np.abs(g_ref)) > 0.05  # a displaced geometry, not a minimum
    np.testing.assert_allclose(g.sum(axis=0), 0, atol=5e-3)


def test_gradient_mixed_solver_close_to_fp64(ctx):
    """The mixed-precision density solver (TF32 products, FP64 finish) gives the same forces
    (step 1e-3 Angstrom, so that energy differences of 1e-6 eV move a component by 5e-4)."""
    mol = geo.alkane(40, np.random.default_rng(1), jitter=0.03)  # nao 242: TF32 phase active
    e64, g64 = sg.gradient(ctx, mol, tol=1e-9, step=1e-3)
    ctx.set_density_solver(sg.SOLVER_PURIFY_MIXED)
    e32, g32 = sg.gradient(ctx, mol, tol=1e-9, step=1e-3)
    assert abs(e32 - e64) < 1e-4
    np.testing.assert_allclose(g32, g64, atol=5e-3, rtol=0)


def test_gradient_argument_errors(ctx):
    mol = CASES["formaldehyde"]
    with pytest.raises(sg.SGBError):
        sg.gradient(ctx, mol, step=0.0)
    with pytest.raises(sg.SGBError):
        sg.gradient(ctx, mol, tol=-1.0)
    with pytest.raises(sg.SGBError):
        sg.gradient(ctx, mol, max_iter=0)


def test_gradient_reports_scf_failures(ctx):
    """A displaced geometry whose SCF reaches the step cap (SGB_E_NOCONV), or a non-finite
    coordinate (SGB_E_NAN), fails the call instead of returning a gradient."""
    mol = CASES["hexane"]
    with pytest.raises(sg.SGBError) as info:
        sg.gradient(ctx, mol, max_iter=2)
    assert info.value.code == sg.E_NOCONV
    bad = geo.Molecule(mol.Z, np.where(np.arange(mol.xyz.size).reshape(-1, 3) == 4, np.nan,
                                       mol.xyz))
    with pytest.raises(sg.SGBError) as info:
        sg.gradient(ctx, bad)
    assert info.value.code == sg.E_NAN
    e, _ = sg.gradient(ctx, mol)  # the context is still usable
    assert np.isfinite(e)


def test_optimizer_on_device_lowers_the_energy(ctx):
    mol = CASES["formaldehyde"]
    e0, _ = sg.gradient(ctx, mol)
    opt, e, gmax, steps = sg.optimize(ctx, mol, gtol=1e-2, max_steps=60)
    assert gmax < 1e-2 and steps < 60
    assert e < e0 - 0.05
    # C=O of MNDO formaldehyde: 1.217 Angstrom
    assert abs(np.linalg.norm(opt.xyz[1] - opt.xyz[0]) - 1.217) < 0.01
