"""The `semiGPU geometry.xyz` CLI (C++ façade with the reference's class names over the C ABI)
prints what the reference CLI prints, apart from paths and timings."""
from __future__ import annotations

import json
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "semigpu_b200", "semiGPU")
with open(os.path.join(ROOT, "tests", "golden", "reference_cli.json")) as _fh:
    GOLD = json.load(_fh)


def _normalise(text: str):
    out = []
    for line in text.splitlines():
        if line.startswith("XYZ file :") or line.startswith("Time taken"):
            continue
        line = re.sub(r"\s+LapackTime = .*$", "", line)  # per-stage timings differ by design
        out.append(line)
    return out


@pytest.mark.parametrize("name", sorted(GOLD))
def test_cli_printout_matches_reference(tmp_path, name):
    xyz = tmp_path / f"{name}.xyz"
    xyz.write_text(GOLD[name]["xyz"])
    r = subprocess.run([CLI, str(xyz)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert _normalise(r.stdout) == _normalise(GOLD[name]["stdout"])


def test_cli_tolerance_flag(tmp_path):
    xyz = tmp_path / "pyridine.xyz"
    xyz.write_text(GOLD["04_pyridine"]["xyz"])
    r = subprocess.run([CLI, "--tol", "1e-6", str(xyz)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    steps = [l for l in r.stdout.splitlines() if l.startswith("SCF step :")]
    assert len(steps) == 15  # step 0 + 14 steps at 1e-6 eV (reference oracle driver)


def test_cli_rejects_unsupported_element(tmp_path):
    xyz = tmp_path / "hf.xyz"
    xyz.write_text("2\nHF\nH 0 0 0\nF 0 0 0.92\n")
    r = subprocess.run([CLI, str(xyz)], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "MNDO parameters" in r.stdout + r.stderr


def test_cli_frames_one_batch_against_oracle(tmp_path, oracle_mod):
    """--frames --json: every frame of a multi-frame file (the golden CLI molecules, blank lines
    between some frames) in one batched launch; each frame's energies and step count as the
    oracle's."""
    names = sorted(GOLD)
    text = "\n".join(GOLD[n]["xyz"].strip() + ("\n" if i % 2 else "") for i, n in enumerate(names))
    xyz = tmp_path / "ensemble.xyz"
    xyz.write_text(text + "\n")
    r = subprocess.run([CLI, "--tol", "1e-6", "--frames", "--json", "--heat", str(xyz)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    rows = [json.loads(line) for line in r.stdout.splitlines()]
    assert [row["frame"] for row in rows] == list(range(len(names)))
    from semigpu_b200 import geometry as geo

    for row, n in zip(rows, names):
        mol = geo.parse_xyz(GOLD[n]["xyz"])
        o = oracle_mod.scf(mol.Z, mol.xyz, tol=1e-6)
        assert row["natoms"] == mol.natoms and row["status"] == 0 and row["converged"]
        assert row["n_iter"] == o["n_iter"], n
        assert abs(row["E_tot"] - o["E_tot"]) < 1e-6, n
        assert "heat_of_formation_kcal_mol" in row
