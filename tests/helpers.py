"""Shared helpers of the test suite."""
import os

import numpy as np

from adventure_fullwave_b200 import meshgen

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(name: str):
    import make_golden

    z = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    params = make_golden.params_of(z)
    return z, params, make_golden.build_model(params)


def rel_l2(a, b) -> float:
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
