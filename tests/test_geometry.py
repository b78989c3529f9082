"""XYZ input (against the reference reader's own parse of its 45 fixtures) and the seeded
workload generators."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from semigpu_b200 import geometry as geo

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
with open(os.path.join(GOLDEN, "reference_cases.json")) as _fh:
    READER = json.load(_fh)["xyz_reader_fixtures"]


@pytest.mark.parametrize("name", sorted(READER))
def test_reader_matches_reference_reader(name):
    fx = READER[name]
    Z_ref, xyz_ref = np.array(fx["Z"]), np.array(fx["xyz"]).reshape(-1, 3)
    if any(int(z) not in (1, 6, 7, 8) for z in Z_ref):
        with pytest.raises(geo.UnsupportedElement):
            geo.parse_xyz(fx["text"])
        return
    m = geo.parse_xyz(fx["text"])
    assert m.Z.tolist() == Z_ref.tolist()
    np.testing.assert_array_equal(m.xyz, xyz_ref)


def test_reader_errors():
    with pytest.raises(ValueError):
        geo.parse_xyz("")
    with pytest.raises(ValueError):
        geo.parse_xyz("0\n\n")
    with pytest.raises(ValueError):
        geo.parse_xyz("3\ncomment\nH 0 0 0\n")
    with pytest.raises(geo.UnsupportedElement):
        geo.parse_xyz("2\nx\nH 0 0 0\nCl 0 0 1.3\n")
    with pytest.raises(geo.UnsupportedElement):
        geo.parse_xyz("1\nx\nXx 0 0 0\n")


def test_multi_frame_roundtrip(tmp_path):
    mols = geo.batch_c3(7, seed=3)
    path = tmp_path / "ens.xyz"
    geo.write_xyz(str(path), mols)
    back = geo.read_xyz_frames(str(path))
    assert len(back) == 7
    for a, b in zip(mols, back):
        assert a.Z.tolist() == b.Z.tolist()
        np.testing.assert_array_equal(a.xyz, b.xyz)


def test_named_workloads():
    c1 = geo.ring_c1()
    assert (c1.natoms, c1.nao, c1.nocc) == (11, 29, 15)
    ring = c1.xyz[:6]
    d = np.linalg.norm(ring - np.roll(ring, 1, axis=0), axis=1)
    np.testing.assert_allclose(d, 1.39, atol=1e-12)
    c2 = geo.alkane_c2(0)
    assert (c2.natoms, c2.nao, c2.nocc) == (302, 602, 301)
    c4 = geo.polyene_c4(0)
    assert (c4.natoms, c4.nao, c4.nocc) == (4002, 10002, 5001)


def test_batch_composition():
    mols = geo.batch_c3(4096, seed=0)
    kinds = [m.meta["kind"] for m in mols]
    frac = {k: kinds.count(k) / len(kinds) for k in ("alkane", "polyene", "ring")}
    assert abs(frac["alkane"] - 0.5) < 0.03 and abs(frac["polyene"] - 0.3) < 0.03
    nao = np.array([m.nao for m in mols])
    assert nao.min() == 8 and nao.max() == 152
    assert all(m.nocc * 2 == sum(int(z) if z < 2 else int(z) - 2 for z in m.Z) for m in mols)
    again = geo.batch_c3(4096, seed=0)
    assert all(np.array_equal(a.xyz, b.xyz) for a, b in zip(mols[:50], again[:50]))


def test_bond_geometry():
    a = geo.alkane(6, rng=None)
    cc = np.linalg.norm(np.diff(a.xyz[:6], axis=0), axis=1)
    np.testing.assert_allclose(cc, 1.54, atol=1e-12)
    p = geo.polyene(6, rng=None)
    bonds = np.linalg.norm(np.diff(p.xyz[:6], axis=0), axis=1)
    np.testing.assert_allclose(bonds, [1.34, 1.46, 1.34, 1.46, 1.34], atol=1e-12)
    for m in (a, p):  # every H 1.08-1.09 A from its nearest carbon
        C, H = m.xyz[m.Z == 6], m.xyz[m.Z == 1]
        dmin = np.min(np.linalg.norm(H[:, None] - C[None], axis=2), axis=1)
        assert np.all((dmin > 1.07) & (dmin < 1.10))


def test_cli_frames_rejects_a_truncated_frame(tmp_path):
    """The CLI's multi-frame reader (C++ façade) stops at a frame with fewer atom lines than its
    count, before any device work."""
    import subprocess

    cli = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "semigpu_b200", "semiGPU")
    if not os.path.exists(cli):
        pytest.skip("CLI not built")
    p = tmp_path / "bad.xyz"
    p.write_text("3\nwater\nO 0 0 0\nH 0.96 0 0\nH -0.24 0.93 0\n\n2\ncut\nH 0 0 0\n")
    r = subprocess.run([cli, "--frames", str(p)], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0
    assert "frame 1" in r.stdout and "ends after 1 of 2 atoms" in r.stdout
