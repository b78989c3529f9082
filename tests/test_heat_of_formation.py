"""Heat of formation: host arithmetic of the C ABI (no GPU needed), checked against the formula
on oracle energies and, loosely, against published MNDO values (which are quoted at MNDO-optimised
geometries, not at these fixture geometries)."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

import semigpu_b200 as sg

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
with open(os.path.join(GOLDEN, "reference_cases.json")) as _fh:
    CASES = json.load(_fh)["cases"]

# Dewar & Thiel, J. Am. Chem. Soc. 99, 4899 (1977), kcal/mol
PUBLISHED = {"02_methane": -11.9, "03_h2o": -60.9, "02_benzene": 21.2, "02_ethylene": 15.4,
             "03_formaldehyde": -33.0, "02_ethane": -19.7}


@pytest.mark.parametrize("name", sorted(PUBLISHED))
def test_heat_of_formation(name):
    c = CASES[f"fixture/{name}@1e-06"]
    dhf = sg.heat_of_formation(c["Z"], c["E_tot"])
    eisol = sum(sg.mndo_parameters(z)[17] for z in c["Z"])
    heat = sum(sg.mndo_parameters(z)[16] for z in c["Z"])
    assert dhf == pytest.approx((c["E_tot"] - eisol) * 23.060548 + heat, abs=1e-9)
    assert abs(dhf - PUBLISHED[name]) < 2.5


def test_parameters_match_reference_table():
    c = sg.mndo_parameters(6)
    assert c[0] == -52.279745 and c[3] == -18.985044 and c[12] == 0.68515777
    with pytest.raises(sg.SGBError):
        sg.mndo_parameters(9)
