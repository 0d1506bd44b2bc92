"""Shared pytest configuration: the ``gpu`` marker and golden-fixture helpers."""

from __future__ import annotations

import json
import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_golden(name: str):
    """Return (arrays, optics_dict, grid_dict) of one golden fixture."""
    d = np.load(GOLDEN / f"{name}.npz", allow_pickle=False)
    meta = json.loads(str(d["meta"]))
    arrays = {k: d[k] for k in d.files if k != "meta"}
    return arrays, meta.get("optics"), meta.get("grid")


def ns_optics(od: dict) -> SimpleNamespace:
    """Duck-typed optics object from a fixture's JSON dict (for the oracle)."""
    od = dict(od)
    od["zernike_coeffs"] = {int(k): v for k, v in (od.get("zernike_coeffs") or {}).items()}
    o = SimpleNamespace(**od)
    o.image_index = od["n_immersion"] if od.get("n_image") is None else od["n_image"]
    return o


def ns_grid(gd: dict) -> SimpleNamespace:
    return SimpleNamespace(**gd)


@pytest.fixture
def golden():
    return load_golden
