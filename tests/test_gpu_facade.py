"""The C++ host API with the reference's class names, driven the way the reference's own
drivers drive it: ElectronicEnergy::ComputeEnergy and the integral lookup
TwoCenterIntegral::GetValueFromArray (through the reference's literal Fock sum) against the
device results and the reference's golden energies."""
from __future__ import annotations

import json
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "semigpu_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
with open(os.path.join(GOLDEN, "reference_cases.json")) as _fh:
    CASES = json.load(_fh)["cases"]


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    from semigpu_b200 import build

    build.build()
    exe = str(tmp_path_factory.mktemp("facade") / "facade_stages")
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{os.path.join(ROOT, 'include')}",
                    f"-I{os.path.join(PKG, 'host')}",
                    os.path.join(ROOT, "tests", "cpp", "facade_stages.cc"), f"-L{PKG}",
                    "-lsemigpu_host", "-lsemigpu_b200", f"-Wl,-rpath,{PKG}", "-o", exe],
                   check=True)
    return exe


@pytest.mark.parametrize("key", ["fixture/04_pyridine@1e-06", "fixture/03_formaldehyde@1e-06",
                                 "batch/09_C4H4N2@1e-06"])
def test_facade_energy_and_integral_lookup(program, tmp_path, key):
    from semigpu_b200 import geometry as geo

    c = CASES[key]
    path = tmp_path / "m.xyz"
    path.write_text(geo.format_xyz(geo.Molecule(np.array(c["Z"]), np.array(c["xyz"]).reshape(-1, 3))))
    r = subprocess.run([program, str(path), repr(c["tol"])], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["steps"] == c["n_iter"] and out["converged"] == 1
    assert abs(out["final_energy"] - c["E_el"]) < 1e-6
    assert abs(out["energy_recomputed"] - out["final_energy"]) < 1e-9
    assert abs(out["e_cc"] - c["E_cc"]) < 1e-6
    assert out["max_abs_dF_lookup"] < 1e-8


def test_electronic_energy_entry_point(gpu_ctx, golden_mats):
    """sgb_electronic_energy on the reference's own final H, F, P gives its E_el."""
    import semigpu_b200 as sg

    for key in ("fixture/04_pyridine@1e-06", "config/ring_C5H5N@1e-06"):
        H, F, P = (golden_mats[f"{key}/{k}"] for k in ("H", "F", "P"))
        e = gpu_ctx.electronic_energy(H, F, P)
        assert abs(e - CASES[key]["E_el"]) < 1e-8
