"""The C ABI library loads without a GPU and exports every entry point declared in
include/semigpu_b200.h; no compute call is made here."""
from __future__ import annotations

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "semigpu_b200.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sgb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared()
    assert "sgb_scf" in names and "sgb_batch_run" in names and len(names) >= 20


def test_library_exports_every_symbol():
    import semigpu_b200 as sg

    if not os.path.exists(sg.LIB_PATH):
        from semigpu_b200 import build as _b

        _b.build()
    L = ctypes.CDLL(sg.LIB_PATH)
    missing = [n for n in declared() if not hasattr(L, n)]
    assert not missing, missing
    assert set(sg.SIGNATURES) == set(declared())


def test_status_strings_without_gpu():
    import semigpu_b200 as sg

    L = sg.lib()
    assert L.sgb_status_string(0) == b"ok"
    assert L.sgb_status_string(-2).startswith(b"element")


def test_size_classes_cover_the_batched_range():
    """The batched launch's size classes: increasing nao bounds up to the single-CTA limit of
    1024 (then the grid-path class), default CTA sizes 128/256/512."""
    import semigpu_b200 as sg

    cls = sg.size_classes()
    bounds = [n for n, _ in cls]
    assert bounds == sorted(bounds) and bounds[0] == 32 and 1024 in bounds
    assert {t for _, t in cls} <= {128, 256, 512}


def test_grid_configs_without_gpu():
    """The whole-GPU purification's tile configurations, listed without a device: the default
    (index 0) is the 128 x 128 tile; every tile is a whole number of 8 x 8 DMMA fragments."""
    import semigpu_b200 as sg

    cfgs = sg.grid_configs()
    assert len(cfgs) == 5 and cfgs[0]["bm"] == 128
    assert {c["bm"] for c in cfgs} == {32, 64, 128}
    assert all(c["bm"] % 8 == 0 and 1 <= c["stages"] <= 8 and c["warps"] in (4, 8, 16) for c in cfgs)
