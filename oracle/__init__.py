"""CPU oracles for the force-and-step path. TEST INFRASTRUCTURE ONLY.

- refengine: the reference's own engine sources compiled in place (tier A).
- restatement: an independent C++ restatement in FP32 and FP64 (tier B).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use these.
"""
