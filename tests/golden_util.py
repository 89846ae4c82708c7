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


def fp64_total(scn, xrel, vel, cell, z, bond_flags=None, virial=False):
    """FP64 oracle of a whole force pass: tier B's nonbonded forces and energy plus the
    bonded restatement (bonds selected by bond_flags), on the configuration (xrel, cell)
    of the fixture's cell grid. With virial=True also the virial (pair + bonded)."""
    from oracle import restatement as R
    n = len(scn["t"])
    f, ep, W = np.zeros((n, 3)), 0.0, np.zeros((3, 3))
    if scn.get("pots"):
        out = R.nonbond(scn, xrel, vel, cell, ref_tasks(z), z["force_cdim"], precision=64, virial=virial)
        f, ep = out[0], out[1]
        if virial:
            W = out[3]
    if any(k in scn and len(scn[k]) for k in ("bi", "ai", "di", "ex_i")):
        origins = R.cell_origins(scn["dim"], z["force_cdim"])
        xabs = origins[np.asarray(cell)] + np.asarray(xrel, dtype=np.float64)
        out = R.bonded(scn, xabs, bond_flags, virial=virial)
        f, ep = f + out[0], ep + out[1]
        if virial:
            W = W + out[2]
    return (f, ep, W) if virial else (f, ep)
