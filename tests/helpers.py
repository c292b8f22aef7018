"""Shared test helpers: golden fixtures and parameter construction."""
from __future__ import annotations

import glob
import json
import os

import numpy as np

from pfc_b200 import params as P

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    meta = json.loads(str(z["meta"]))
    return meta, z


def params_of(meta):
    return P.make_params(meta["params"], meta["c"], meta["dt"])


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)
