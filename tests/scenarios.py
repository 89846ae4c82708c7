"""Test-side alias of the seeded workloads (mechanica_b200/workloads.py)."""
from mechanica_b200.workloads import *  # noqa: F401,F403
from mechanica_b200.workloads import _reject_close, argon, build_gpu, chains, dpd, large, lattice, make_potential, morse2, species, walls  # noqa: F401
