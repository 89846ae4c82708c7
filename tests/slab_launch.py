"""Launches the ranks of tests/slab_worker.py as subprocesses on 127.0.0.1 (gloo) and waits
for all of them, each bounded by a timeout."""
import os
import socket
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(world, args, timeout=600):
    """Runs slab_worker.py with args on `world` ranks; returns their exit codes and the tail of
    each rank's output."""
    port = free_port()
    procs = []
    for r in range(world):
        env = dict(os.environ, RANK=str(r), WORLD_SIZE=str(world), LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "slab_worker.py")] + [str(a) for a in args],
                                      env=env, stdout=subprocess.PIPE, stderr=subprocess.STDOUT))
    out = []
    try:
        for p in procs:
            o, _ = p.communicate(timeout=timeout)
            out.append((p.returncode, o.decode(errors="replace")[-2000:]))
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
                p.wait()
    return out
