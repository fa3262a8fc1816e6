"""Shared helpers for the test-suite (not part of the product)."""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def digest(*arrays) -> str:
    """SHA-256 over the little-endian int64 bytes of the given arrays."""
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(np.asarray(a), dtype="<i8").tobytes())
    return h.hexdigest()


def load_golden() -> dict:
    with open(os.path.join(GOLDEN_DIR, "golden.json")) as f:
        return json.load(f)


def load_small():
    return np.load(os.path.join(GOLDEN_DIR, "small.npz"))
