"""The geometry optimiser's host logic (BFGS with capped, backtracked moves) on CPU, driven by
the oracle's energies through central differences -- the same differences sgb_gradient takes on
the device.  Water relaxes to MNDO's minimum (O-H 0.943 Angstrom, H-O-H 106.8 degrees in the
published MNDO parametrisation), and the gradient there vanishes."""
from __future__ import annotations

import numpy as np

import semigpu_b200 as sg
from semigpu_b200 import geometry as geo


def fd_gradient(oracle, mol, step=1e-4, tol=1e-10):
    x = mol.xyz.reshape(-1)
    e0 = oracle.scf(mol.Z, mol.xyz, tol=tol, max_iter=300)["E_tot"]
    g = np.zeros_like(x)
    for c in range(x.size):
        e = []
        for s in (step, -step):
            xx = x.copy()
            xx[c] += s
            e.append(oracle.scf(mol.Z, xx.reshape(-1, 3), tol=tol, max_iter=300)["E_tot"])
        g[c] = (e[0] - e[1]) / (2 * step)
    return e0, g.reshape(-1, 3)


def test_water_relaxes_to_the_mndo_minimum(oracle_mod):
    water = geo.Molecule([8, 1, 1], [[0, 0, 0], [1.05, 0, 0], [-0.15, 0.9, 0.1]])
    e_start, g_start = fd_gradient(oracle_mod, water)
    assert np.max(np.abs(g_start)) > 1.0
    mol, e, gmax, steps = sg.optimize(None, water, gtol=5e-3, max_steps=60,
                                      energy_gradient=lambda m: fd_gradient(oracle_mod, m))
    assert gmax < 5e-3 and steps < 60
    assert e < e_start - 0.1
    oh1 = np.linalg.norm(mol.xyz[1] - mol.xyz[0])
    oh2 = np.linalg.norm(mol.xyz[2] - mol.xyz[0])
    cosang = (mol.xyz[1] - mol.xyz[0]) @ (mol.xyz[2] - mol.xyz[0]) / (oh1 * oh2)
    ang = np.degrees(np.arccos(cosang))
    assert abs(oh1 - oh2) < 2e-3
    assert abs(oh1 - 0.943) < 0.01, oh1
    assert abs(ang - 106.8) < 1.5, ang


def test_translation_and_rotation_leave_the_gradient_sum_zero(oracle_mod):
    """Sum of forces and of torques vanish for any geometry (energy invariant under rigid
    motions) -- checks the difference quotient's indexing."""
    mol = geo.Molecule([6, 8, 1, 1], [[0, 0, 0], [1.25, 0.05, 0], [-0.55, 0.95, 0.02],
                                      [-0.5, -0.9, -0.05]])
    _, g = fd_gradient(oracle_mod, mol)
    assert np.max(np.abs(g)) > 0.1
    np.testing.assert_allclose(g.sum(axis=0), 0, atol=1e-4)
    np.testing.assert_allclose(np.cross(mol.xyz, g).sum(axis=0), 0, atol=1e-4)
