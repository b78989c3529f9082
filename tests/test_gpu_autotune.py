"""Per-class CTA sizes: validation, results unchanged by the choice, and the autotuner."""
from __future__ import annotations

import numpy as np
import pytest

import semigpu_b200 as sg
from semigpu_b200 import autotune
from semigpu_b200 import geometry as geo

pytestmark = pytest.mark.gpu


def test_invalid_class_threads_rejected(gpu_ctx):
    n = len(sg.size_classes())
    with pytest.raises(sg.SGBError):
        gpu_ctx.set_class_threads([128] * n)  # 128-thread CTAs only for nao <= 64


def test_results_do_not_depend_on_cta_size(gpu_ctx):
    mols = geo.batch_c3(96, seed=13)
    ref = sg.run_molecules(gpu_ctx, mols, tol=1e-6)
    classes = sg.size_classes()
    alt = [512 if nmax <= 160 else t for nmax, t in classes]  # every class at 512 threads
    gpu_ctx.set_class_threads(alt)
    try:
        r = sg.run_molecules(gpu_ctx, mols, tol=1e-6)
    finally:
        gpu_ctx.set_class_threads([t for _, t in classes])
    np.testing.assert_array_equal(r["n_iter"], ref["n_iter"])
    np.testing.assert_allclose(r["E_tot"], ref["E_tot"], rtol=0, atol=1e-9)


def test_autotuner_returns_a_valid_choice():
    ctx = sg.Context(0)
    try:
        res = autotune.tune(ctx, geo.batch_c3(256, seed=2), repeats=1)
        assert res["ms"] <= res["default_ms"]
        assert len(res["class_threads"]) == len(sg.size_classes())
        r = sg.run_molecules(ctx, geo.batch_c3(32, seed=3), tol=1e-6)
        assert np.all(r["converged"])
    finally:
        ctx.close()


def test_every_grid_config_gives_the_same_scf():
    """One molecule on the whole GPU with each tile configuration of the purification loop:
    the same steps and energy (the products differ only in summation order)."""
    mol = geo.alkane(50, np.random.default_rng(6))  # nao 302
    ctx = sg.Context(0)
    try:
        out = []
        for k in [-1] + list(range(len(sg.grid_configs()))):
            ctx.set_grid_config(k)
            out.append(sg.Molecule.from_geometry(ctx, mol).run(tol=1e-6))
        with pytest.raises(sg.SGBError):
            ctx.set_grid_config(len(sg.grid_configs()))
    finally:
        ctx.close()
    for r in out[1:]:
        assert r["status"] == 0 and r["n_iter"] == out[0]["n_iter"]
        assert abs(r["E_tot"] - out[0]["E_tot"]) < 1e-8


def test_grid_autotuner_returns_a_valid_choice():
    mol = geo.alkane(60, np.random.default_rng(7))  # nao 362
    ctx = sg.Context(0)
    try:
        res = autotune.tune_grid(ctx, mol, repeats=1)
        assert res["config"] in [-1] + list(range(len(sg.grid_configs())))
        assert res["ms"] <= res["auto_ms"]
        r = sg.Molecule.from_geometry(ctx, mol).run(tol=1e-6)
        assert r["converged"] and r["status"] == 0
    finally:
        ctx.close()
