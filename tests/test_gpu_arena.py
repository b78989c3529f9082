"""Device arenas of destroyed molecules and batches are kept by the context and reused: results
do not depend on what an arena held before, the held bytes stay bounded, and a budget still
admits what fits once the spare arenas are given back."""
from __future__ import annotations

import numpy as np
import pytest

import semigpu_b200 as sg
from semigpu_b200 import geometry as geo

pytestmark = pytest.mark.gpu


def _energies(ctx, mols):
    out = []
    for m in mols:
        one = sg.Molecule.from_geometry(ctx, m)
        r = one.run(tol=1e-6)
        one.close()
        out.append((r["E_tot"], r["n_iter"]))
    return out


def test_reused_arenas_give_the_same_results():
    rng = np.random.default_rng(31)
    mols = [geo.alkane(k, rng) for k in (12, 3, 20, 1, 7)] + [geo.polyene(k, rng) for k in (24, 6)]
    fresh = []
    for m in mols:
        c = sg.Context(0)
        fresh += _energies(c, [m])
        c.close()
    ctx = sg.Context(0)
    try:
        again = _energies(ctx, mols) + _energies(ctx, mols[::-1])
        held = ctx.bytes_in_use
        for _ in range(3):
            _energies(ctx, mols)
        assert ctx.bytes_in_use == held  # steady state: nothing new is allocated
    finally:
        ctx.close()
    assert again == fresh + fresh[::-1]


def test_batch_arena_reused_by_molecules_and_batches():
    mols = geo.batch_c3(64, seed=5)
    ctx = sg.Context(0)
    try:
        b = sg.Batch(ctx, mols)
        b.run(1e-6)
        ref = b.results()
        b.close()
        b = sg.Batch(ctx, mols[::-1])  # the same arena, other order
        b.run(1e-6)
        r = b.results()
        b.close()
    finally:
        ctx.close()
    np.testing.assert_array_equal(r["E_tot"][::-1], ref["E_tot"])
    np.testing.assert_array_equal(r["n_iter"][::-1], ref["n_iter"])


def test_budget_reclaims_spare_arenas():
    rng = np.random.default_rng(2)
    small, big = geo.alkane(10, rng), geo.alkane(20, rng)
    probe = sg.Context(0)
    m = sg.Molecule.from_geometry(probe, big)
    need = probe.bytes_in_use
    m.close()
    probe.close()
    # room for the big molecule's arena but not for it beside a spare small one
    ctx = sg.Context(0, hbm_budget=need + (need // 8))
    try:
        (e_small, _), = _energies(ctx, [small])
        assert ctx.bytes_in_use > 0  # the small arena is kept
        (e_big, _), = _energies(ctx, [big])
        assert ctx.bytes_in_use <= need + need // 8
    finally:
        ctx.close()
    assert np.isfinite(e_small) and np.isfinite(e_big)


def test_context_closed_before_its_molecules_and_batches():
    """Closing a context first (a `with` block around objects collected later) releases their
    device memory; destroying them afterwards touches only their host parts."""
    ctx = sg.Context(0)
    m = sg.Molecule.from_geometry(ctx, geo.ring_c1())
    r = m.run(tol=1e-6)
    b = sg.Batch(ctx, geo.batch_c3(8, seed=1))
    b.run(1e-6)
    b.results()
    ctx.close()
    m.close()
    b.close()
    assert r["converged"]
    with sg.Context(0) as c2:
        r2 = sg.run_molecules(c2, geo.batch_c3(4, seed=2), tol=1e-6)
    assert np.all(r2["status"] == 0)
