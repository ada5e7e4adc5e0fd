"""Loader for the committed golden fixtures (made by tests/golden/make_golden.py)."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def summary():
    with open(os.path.join(GOLDEN, "golden.json")) as fh:
        return json.load(fh)


def arrays(prec):
    return dict(np.load(os.path.join(GOLDEN, f"golden_{prec}.npz")))


def cases():
    return summary()["cases"]
