"""Golden vectors produced by the reference's own Python code (see
make_golden.py) and a loader."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def load(name: str):
    p = HERE / name
    if name.endswith(".json"):
        return json.loads(p.read_text())
    return np.load(p)
