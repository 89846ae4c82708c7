"""Loading of the golden fixtures (tests/golden/*.npz)."""
import os
import sys

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)

from make_golden import load_scenario  # noqa: E402

CASES = ["argon_small", "argon_default_cells", "dpd_small", "lattice_small", "lattice_break", "morse2_small",
         "lattice_noisy"]


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return z, load_scenario(z)


def ref_tasks(z):
    t = z["force_tasks"]
    return t[(t[:, 0] == 1) | (t[:, 0] == 2)]


def rel_rms(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.sqrt((b ** 2).sum())
    return np.sqrt(((a - b) ** 2).sum()) / (den if den > 0 else 1.0)
