#!/usr/bin/env python
"""Benchmark of the force-and-step path on B200: particle-steps/s.

Default workload (N=1): the DPD fluid with a body force -- 200,000 particles in a
40x20x20 box, periodic in x/y, no-slip walls in z, DPD a=25, gamma=4.5,
sigma=3, cutoff 1, constant force 0.02 in +x, dt=0.01 -- seeded synthetic
positions (uniform) and velocities (Maxwell-Boltzmann, kT=1).

One step = one engine_step: nonbonded forces, integrator, re-binning (three
kernels replayed from a CUDA graph). value = particles x timed steps / device
time (per-step CUDA events on the engine stream, L2 flushed between steps with
a 256 MiB write). e2e = the same metric through the C ABI in the reference's
data format with host buffers: every step engine_load's the absolute positions
and velocities by particle id from pinned host memory, steps, and
engine_unload's them back (host clock; the median of five blocks of round
trips, each block's mean); the raw slot-order state copy is reported beside
it. roofline: the force kernel against the FP32 pipe (and, as
hbm_view, against the measured copy bandwidth); rebin_view: the integrator and
the re-binning scatter against the measured copy bandwidth.

--impl reference times the reference's own CPU engine (compiled in place from
the reference sources, oracle/_ref) on this host's cores for the same workload.
With torchrun (N > 1) each rank runs an independent replica (weak scaling); the
reported time is the max over ranks.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s (1 B200) plain vs batched/adjoint; force rel-err <=1e-5"
WORKLOAD = ("DPD fluid with body force: 200,000 particles, 40x20x20 box, periodic x/y, no-slip z; "
            "DPD a=25 gamma=4.5 sigma=3 rc=1 kT=1; constant force 0.02 +x; FP32, dt=0.01")
# counters of one force launch of the 200,000-particle DPD workload from an ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum, smsp__inst_executed.sum), with the hash of the
# kernel sources they were captured on; used only while that hash matches the current sources
COUNTERS = os.path.join(ROOT, "profiles", "force_kernel_dpd200k.counters.txt")
# algorithmic FP32 operations per candidate pair and per interacting DPD pair
# (counted from the reference's scalar pair loop and dpd_eval)
F_CAND = 9
F_INT_DPD = 40
F_INT_TABLE = 44


# the sources that decide what a force launch does: its kernels and device structures, the host
# engine that builds its work items, tables and launch configuration, and the build flags
FORCE_SOURCES = ("mechanica_b200/csrc/mxg_kernels.cu", "mechanica_b200/csrc/mxg_kernels.h",
                 "mechanica_b200/csrc/mxg_device.cuh", "mechanica_b200/csrc/mxg_engine.cpp",
                 "mechanica_b200/csrc/potential_table.cpp", "mechanica_b200/csrc/potential_table.h",
                 "mechanica_b200/build.py")


def sources_sha16():
    """Hash of the sources that decide what a force launch does: identifies the build whose
    launches a capture measured."""
    import hashlib
    h = hashlib.sha256()
    for path in (os.path.join(ROOT, f) for f in FORCE_SOURCES):
        h.update(os.path.basename(path).encode())
        with open(path, "rb") as f:
            h.update(f.read())
    return h.hexdigest()[:16]


def captured_counters():
    """(counters dict, note): the force launch's captured counters when they were taken on the
    current sources, else (None, why not)."""
    if not os.path.exists(COUNTERS):
        return None, "no capture recorded"
    rec = {}
    with open(COUNTERS) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 2 and not line.startswith("#"):
                rec[parts[0]] = parts[1]
    want = sources_sha16()
    if rec.get("sources_sha16") != want:
        return None, f"capture of sources {rec.get('sources_sha16')} is stale (current {want})"
    return {k: int(v) for k, v in rec.items() if k != "sources_sha16" and v.isdigit()}, "captured on these sources"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=200000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-forms", action="store_true", help="skip the other configurations (batched, LJ, lattice)")
    ap.add_argument("--record-counters", metavar="CSV",
                    help="write the force-launch counters file from an ncu --csv capture of one force launch "
                         "(dram__bytes_read.sum, dram__bytes_write.sum, smsp__inst_executed.sum) and exit")
    return ap.parse_args()


def record_counters(csv_path):
    """Writes COUNTERS from an ncu CSV capture of one force launch of the default workload, with
    the hash of the current sources (the capture must have run these sources)."""
    import csv
    vals = {}
    kernel = None
    with open(csv_path) as f:
        rows = [r for r in csv.reader(f)]
    hdr = next(i for i, r in enumerate(rows) if "Metric Name" in r)
    cols = rows[hdr]
    for r in rows[hdr + 1:]:
        if len(r) != len(cols):
            continue
        d = dict(zip(cols, r))
        if "force_kernel" not in d["Kernel Name"]:
            continue
        if kernel is None:
            kernel = (d["ID"], d["Kernel Name"])
        if (d["ID"], d["Kernel Name"]) != kernel:
            continue
        vals[d["Metric Name"]] = int(float(d["Metric Value"].replace(",", "")))
    need = ("dram__bytes_read.sum", "dram__bytes_write.sum", "smsp__inst_executed.sum")
    missing = [k for k in need if k not in vals]
    if missing:
        raise SystemExit(f"{csv_path}: no {missing} for a force_kernel launch")
    with open(COUNTERS, "w") as f:
        f.write(f"# one force launch of the default workload (ncu capture {os.path.basename(csv_path)}: "
                f"{kernel[1].split('(')[0]})\n")
        f.write(f"sources_sha16 {sources_sha16()}\n")
        f.write(f"dram_bytes_per_launch {vals['dram__bytes_read.sum'] + vals['dram__bytes_write.sum']}\n")
        f.write(f"dram_bytes_read {vals['dram__bytes_read.sum']}\n")
        f.write(f"dram_bytes_write {vals['dram__bytes_write.sum']}\n")
        f.write(f"warp_instructions_per_launch {vals['smsp__inst_executed.sum']}\n")
    print(open(COUNTERS).read(), end="")


def max_over_ranks(x, world, device=None):
    """The largest of a per-rank float over all ranks (a MAX all-reduce in FP64). Every
    rank calls it at the same point; with one rank it returns x."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, n, steps, ms):
    """Whole-job particle-steps/s: each of `world` ranks advances its own n-particle
    replica `steps` times, and the job lasts as long as its slowest rank (`ms`, the max
    over ranks of the device-timed milliseconds)."""
    return world * n * steps / (ms / 1e3)


def workload(n):
    from mechanica_b200 import workloads as W
    scale = (n / 200000.0) ** (1.0 / 3.0)
    dims = (40.0 * scale, 20.0 * scale, 20.0 * scale) if n != 200000 else (40.0, 20.0, 20.0)
    return W.dpd(n=n, dims=dims, seed=2)


class Clocks:
    """Samples the SM clock and the clock-event (throttle) reasons during a timed region:
    NVML polled every half millisecond in a thread (a 20-step region lasts a few
    milliseconds), else nvidia-smi every 200 ms. Reads only; changes no setting."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.f = None
        self.thread = None
        self.samples = []
        self.max_mhz = None

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            bits = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}
            self.stop_flag = threading.Event()

            def poll():
                while not self.stop_flag.is_set():
                    mhz = float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                    r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((mhz, [n for n, bit in bits.items() if r & bit]))
                    time.sleep(0.0005)

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        try:
            self.f = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join()
            sm = [m for m, _ in self.samples]
            reasons = sorted({n for _, rs in self.samples for n in rs})
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz, "reasons": reasons,
                    "samples": len(sm), "source": "NVML, 0.5 ms period"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no clock source"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, name in enumerate(self.NAMES):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(name)
            except Exception:
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi, 200 ms period"}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


def cpu_baseline(scn, seconds):
    """The reference's own CPU engine on this host, a bounded sample of the workload."""
    from oracle import refengine
    if not refengine.available():
        return None, None
    cores = os.cpu_count() or 1
    probe = refengine.run(dict(scn, action="steps", nsteps=2, warmup=1, runners=cores))
    per = max(float(probe["seconds"]) / 2, 1e-4)
    nsteps = int(max(3, min(500, seconds / per)))
    r = refengine.run(dict(scn, action="steps", nsteps=nsteps, warmup=1, runners=cores))
    n = len(scn["t"])
    val = n * nsteps / float(r["seconds"])
    return {"value": val, "unit": "particle-steps/s", "cores": cores, "kind": "reference",
            "sample": f"{nsteps} engine_step calls of the full {n}-particle workload after 1 warm-up step, "
                      f"nr_runners = {cores} pthreads (reference engine compiled from its own sources)"}, r


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    scn = workload(args.n)
    from oracle import refengine
    if not refengine.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference engine library (oracle/_ref) not built"}))
        return
    cores = os.cpu_count() or 1
    n = len(scn["t"])
    probe = refengine.run(dict(scn, action="steps", nsteps=1, warmup=0, runners=cores))
    per = max(float(probe["seconds"]), 1e-4)
    budget = 120.0
    steps = int(max(1, min(args.steps, budget / per)))
    r = refengine.run(dict(scn, action="steps", nsteps=steps, warmup=args.warmup if args.warmup <= 5 else 3,
                           runners=cores))
    secs = float(r["seconds"])
    val = n * steps / secs
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "particle-steps/s", "n_gpus": 0,
            "steps": steps, "warmup": min(args.warmup, 5), "ms_per_step": 1e3 * secs / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded uniform positions, Maxwell-Boltzmann velocities)",
            "config": {"workload": WORKLOAD, "steps_requested": args.steps},
            "cpu_baseline": {"value": val, "unit": "particle-steps/s", "cores": cores, "kind": "reference",
                             "sample": f"{steps} of {args.steps} requested engine_step calls (bounded to ~{budget:.0f} s), "
                                       f"nr_runners = {cores}"},
            "e2e": {"value": val, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def _time_steps(L, e, K, stream, flush):
    """Device time (ms) of K single steps of engine e, L2 flushed between steps
    outside the per-step events."""
    import torch
    a = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    b = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    with torch.cuda.stream(stream):
        for k in range(K):
            flush.zero_()
            a[k].record(stream)
            L.mxg_engine_step(e, 1)
            b[k].record(stream)
    torch.cuda.synchronize()
    return sum(x.elapsed_time(y) for x, y in zip(a, b))


def _plain(u, stream):
    """Moves a universe built by the workload helpers onto the bench stream."""
    u.stream = stream.cuda_stream
    u._dirty = True
    u._ensure()
    return u._e


def forms_and_configs(args, stream, flush):
    """The other configurations on the same GPU: the LJ argon fluid and the
    bonded lattice (plain engine), and the batched ensemble of 256 cell-sorting
    replicas against the same replicas run one after another."""
    import mechanica_b200 as m
    from mechanica_b200 import workloads as W
    from mechanica_b200._native import lib, check
    L = lib()
    out = {}
    K = max(10, min(args.steps, 200))
    for name, build in (("lj_argon_10k", lambda: W.argon(n=10000, L=10.0, cells=10, seed=21)),
                        ("lattice_32k", lambda: W.lattice(nx=32, seed=23))):
        scn = build()
        W.build_gpu(scn)
        e = _plain(m.universe, stream)
        with torch_stream(stream):
            check(L.mxg_engine_step(e, 3), "warm-up")
        ms = _time_steps(L, e, K, stream, flush)
        check(L.mxg_engine_status(e), name)
        n = len(scn["t"])
        out[name] = {"value": n * K / (ms / 1e3), "unit": "particle-steps/s", "particles": n, "steps": K,
                     "ms_per_step": ms / K}
        m.universe.close()
        if not args.no_cpu_baseline:
            # the reference engine on the host cores, a bounded sample of the same workload
            try:
                from oracle import refengine
                if refengine.available():
                    cores = os.cpu_count() or 1
                    # the window the GPU form times: K steps after 3 warm-up steps (the lattice
                    # loses its bonds in the first ten steps and clumps, so early steps are cheaper)
                    r = refengine.run(dict(scn, action="steps", nsteps=K, warmup=3, runners=cores))
                    ref = n * K / float(r["seconds"])
                    out[name]["cpu_reference"] = {"value": ref, "unit": "particle-steps/s", "cores": cores,
                                                  "kind": "reference",
                                                  "sample": f"{K} engine_step calls after 3 warm-up steps, "
                                                            "the same step window as the GPU form"}
                    out[name]["speedup_vs_cpu_reference"] = out[name]["value"] / ref
            except Exception as exc:
                out[name]["cpu_reference"] = {"error": str(exc)[:200]}

    # batched ensemble: all replicas in one engine, one set of launches per step
    specs = W.cell_sorting_specs(nrep=256, seed=5)
    ntot = sum(len(sc["t"]) for sc in specs)
    Kb = max(5, min(args.steps, 50))
    u = W.build_gpu_batch(specs, stream=stream.cuda_stream)
    u._ensure()
    per_sm = u.autotune()
    e = u._e
    with torch_stream(stream):
        check(L.mxg_engine_step(e, 3), "warm-up")
    ms_b = _time_steps(L, e, Kb, stream, flush)
    check(L.mxg_engine_status(e), "batched")
    batched_roofline = force_roofline(L, e, flush, F_INT_TABLE, "Morse tables over all replicas")
    u.close()
    # the same replicas, one plain engine each, run one after another
    ms_s = 0.0
    for sc in specs:
        W.build_gpu(sc)
        e = _plain(m.universe, stream)
        with torch_stream(stream):
            check(L.mxg_engine_step(e, 3), "warm-up")
        ms_s += _time_steps(L, e, Kb, stream, flush)
        check(L.mxg_engine_status(e), "sequential")
        m.universe.close()
    out["adjoint_32k"] = adjoint_form(stream)
    out["adjoint_bonded_32k"] = adjoint_bonded_form(stream)
    out["batched_256"] = {"value": ntot * Kb / (ms_b / 1e3), "unit": "particle-steps/s", "replicas": len(specs),
                          "particles": ntot, "steps": Kb, "ms_per_step": ms_b / Kb,
                          "force_ctas_per_sm": per_sm,
                          "sequential_plain_value": ntot * Kb / (ms_s / 1e3),
                          "speedup_vs_sequential": ms_s / ms_b, "roofline": batched_roofline}
    return out


def fp32_peak_tflops():
    """Nominal FP32 pipe of the current device (MEASURED_PEAKS.json holds no FP32 figure):
    SMs x 128 lanes x 2 FLOP x the measured maximum SM clock."""
    import torch
    sm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = (measured_peaks() or {}).get("sm_max_mhz", 1965.0)
    return sm * 128 * 2 * mhz * 1e6 / 1e12, f"nominal FP32 pipe: {sm} SMs x 128 lanes x 2 x {mhz:.0f} MHz"


def force_roofline(L, e, flush, f_int, what, reps=20):
    """The engine's force launch against the FP32 pipe: algorithmic FLOPs (F_CAND per
    candidate pair of the reference's task lists, f_int per interacting pair, counted on the
    current state) over the median CUDA-event time of reps launches, L2 flushed before each."""
    from mechanica_b200._native import check
    cand, inter = ctypes.c_longlong(), ctypes.c_longlong()
    check(L.mxg_engine_pair_counts(e, ctypes.byref(cand), ctypes.byref(inter)), "pair_counts")
    per = np.zeros(reps)
    check(L.mxg_engine_time_force_launches(e, reps, ctypes.c_void_p(flush.data_ptr()), flush.numel(),
                                           per.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "time_force")
    ms = float(np.median(per))
    flops = F_CAND * cand.value + f_int * inter.value
    peak, src = fp32_peak_tflops()
    achieved = flops / (ms / 1e3) / 1e12
    return {"bound": "fp32", "kernel": f"force_kernel ({what})", "achieved": achieved, "peak": peak,
            "unit": "TFLOP/s", "frac": achieved / peak, "peak_source": src, "force_ms_per_launch": ms,
            "algorithmic_flops_per_launch": flops, "candidate_pairs": cand.value, "interacting_pairs": inter.value,
            "flops_per_pair": {"candidate": F_CAND, "interacting": f_int}}


def adjoint_form(stream, nsteps=200, every=20):
    """The adjoint workload: 32,768-particle two-type Morse mixture with a summed
    DPD thermostat (Philox), 200 steps, snapshots every 20, RDF loss; gradients of
    the loss with respect to the ten potential parameters and the initial state.
    Timed with CUDA events on the engine's stream around forward + loss +
    backward (segment recompute included)."""
    import torch
    import mechanica_b200 as m
    from mechanica_b200 import adjoint as A
    from mechanica_b200 import workloads as W
    spec = W.adjoint_spec(n=32768, seed=7)
    with torch.cuda.stream(stream):
        u, P = W.build_adjoint(spec, stream=stream.cuda_stream)
        sim = A.Simulation(u, P, nsteps=nsteps, checkpoint_every=every, step0=0)
        tgt = torch.tensor(W.rdf_target(), dtype=torch.float64, device="cuda")
        theta = torch.tensor(P.theta(), dtype=torch.float64, requires_grad=True)
        x0 = torch.tensor(spec["x"], dtype=torch.float64, requires_grad=True)
        v0 = torch.tensor(spec["v"], dtype=torch.float64, requires_grad=True)
        # warm-up (builds the engine, derivative tables and graphs)
        x4 = A.trajectory(theta, x0, v0, A.Simulation(u, P, nsteps=every, checkpoint_every=every, step0=0))
        A.rdf_loss(x4, tgt, spec["dim"], 0, 1)[0].backward()
        theta.grad = None
        torch.cuda.synchronize()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        x4 = A.trajectory(theta, x0, v0, sim)
        loss, _ = A.rdf_loss(x4, tgt, spec["dim"], 0, 1)
        e1.record(stream)
        loss.backward()
        e2.record(stream)
        torch.cuda.synchronize()
    fwd, tot = e0.elapsed_time(e1), e0.elapsed_time(e2)
    n = len(spec["t"])
    out = {"value": n * nsteps / (tot / 1e3), "unit": "particle-steps/s (forward + backward)", "particles": n,
           "steps": nsteps, "checkpoint_every": every, "ms_forward": fwd, "ms_forward_backward": tot,
           "forward_value": n * nsteps / (fwd / 1e3), "loss": float(loss.item()),
           "grad_theta": [float(g) for g in theta.grad.numpy()],
           "params": "Morse (d, a, r0) of AA, AB, BB; DPD gamma shared",
           "check": "gradients vs FP64 central differences: tests/test_gpu_adjoint.py (512 particles; a = 8 over "
                    "12 steps; the workload's own a = 5 over 4 steps with h = 1e-4, where Morse r0's difference "
                    "spreads by ~1e-3 over h as its table edge crosses pairs at the cutoff)",
           "roofline": adjoint_roofline(u._e, tot, nsteps, F_INT_TABLE + F_INT_DPD)}
    u.close()
    return out


# the VJP of a pair term is counted as twice its forward arithmetic (the polynomial's value
# and derivative for each term of the force and of its parameters)
F_VJP_FACTOR = 2


def adjoint_roofline(e, ms_total, nsteps, f_int):
    """Forward + backward against the FP32 pipe. Algorithmic FLOPs per step: the forward force
    pass and its recompute in the backward sweep (F_CAND per candidate, f_int per interacting
    pair each) and the VJP (F_CAND per candidate, F_VJP_FACTOR x f_int per interacting pair);
    pairs counted on the starting state (the density is constant), steps x that over the
    CUDA-event time of forward + loss + backward."""
    from mechanica_b200._native import check, lib
    cand, inter = ctypes.c_longlong(), ctypes.c_longlong()
    check(lib().mxg_engine_pair_counts(e, ctypes.byref(cand), ctypes.byref(inter)), "pair_counts")
    per_step = 2 * (F_CAND * cand.value + f_int * inter.value) + F_CAND * cand.value + F_VJP_FACTOR * f_int * inter.value
    flops = nsteps * per_step
    peak, src = fp32_peak_tflops()
    achieved = flops / (ms_total / 1e3) / 1e12
    return {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "peak_source": src, "algorithmic_flops": flops, "candidate_pairs": cand.value,
            "interacting_pairs": inter.value,
            "flops_per_step": "2 x (9 cand + f_int int) + (9 cand + 2 f_int int)", "f_int": f_int}


def adjoint_bonded_form(stream, nsteps=200, every=20):
    """The adjoint through bonds: a 32^3 harmonic-bonded block (98,304 bonds, k = 20,
    r0 = 0.5, starting stretched at 0.51) with a weak Morse term, overdamped, dt = 0.002;
    200 steps, snapshots every 20; loss = a seeded linear functional of the final positions;
    gradients with respect to harmonic k and r0 and Morse d and a (the FD-checked model of
    tests/test_gpu_adjoint_bonds.py, scaled up)."""
    import torch
    from mechanica_b200 import adjoint as A
    from mechanica_b200 import workloads as W
    spec = W.bonded_block(nx=32)
    n = len(spec["t"])
    with torch.cuda.stream(stream):
        u, P = W.build_bonded_adjoint(spec, stream=stream.cuda_stream)
        c = torch.tensor(np.random.default_rng(3).normal(size=(n, 3)), dtype=torch.float64, device="cuda")
        theta = torch.tensor(P.theta(), dtype=torch.float64, requires_grad=True)
        x0 = torch.tensor(spec["x"], dtype=torch.float64, requires_grad=True)
        v0 = torch.zeros_like(x0)
        x4 = A.trajectory(theta, x0, v0, A.Simulation(u, P, nsteps=every, checkpoint_every=every, step0=0))
        (x4[:, :3].double() * c).sum().backward()
        theta.grad = None
        sim = A.Simulation(u, P, nsteps=nsteps, checkpoint_every=every, step0=0)
        torch.cuda.synchronize()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        x4 = A.trajectory(theta, x0, v0, sim)
        loss = (x4[:, :3].double() * c).sum()
        e1.record(stream)
        loss.backward()
        e2.record(stream)
        torch.cuda.synchronize()
    fwd, tot = e0.elapsed_time(e1), e0.elapsed_time(e2)
    out = {"value": n * nsteps / (tot / 1e3), "unit": "particle-steps/s (forward + backward)", "particles": n,
           "bonds": int(len(spec["bi"])), "steps": nsteps, "checkpoint_every": every, "ms_forward": fwd,
           "ms_forward_backward": tot, "forward_value": n * nsteps / (fwd / 1e3),
           "grad_theta": [float(g) for g in theta.grad.numpy()], "params": "harmonic k, r0; Morse d, a",
           "check": "bond-k, r0, Morse and position gradients vs FP64 central differences: "
                    "tests/test_gpu_adjoint_bonds.py (6^3 block, 10 steps)",
           "roofline": adjoint_roofline(u._e, tot, nsteps, F_INT_TABLE)}
    u.close()
    return out


class torch_stream:
    def __init__(self, stream):
        import torch
        self.ctx = torch.cuda.stream(stream)

    def __enter__(self):
        return self.ctx.__enter__()

    def __exit__(self, *a):
        return self.ctx.__exit__(*a)


def main():
    args = parse()
    if args.record_counters:
        record_counters(args.record_counters)
        return
    if args.impl == "reference":
        reference_arm(args)
        return
    import torch
    import torch.distributed as dist

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)

    import mechanica_b200 as m
    from mechanica_b200 import workloads as W
    from mechanica_b200._native import lib, check

    scn = workload(args.n)
    n = len(scn["t"])
    stream = torch.cuda.Stream(device=dev)
    # build through the public API on our stream
    bc = {"x": scn["bc"][0], "y": scn["bc"][1], "z": scn["bc"][2]}
    W.build_gpu(scn)
    u = m.universe
    u.stream = stream.cuda_stream
    u._dirty = True
    u._ensure()
    e = u._e
    L = lib()

    # accuracy on the initial configuration: GPU force pass (the reference leg
    # below compares it against the reference engine)
    check(L.mxg_engine_force(e), "force")
    x0, v0, f_gpu, c0, xr0 = u.state()
    cand = ctypes.c_longlong()
    inter = ctypes.c_longlong()
    check(L.mxg_engine_pair_counts(e, ctypes.byref(cand), ctypes.byref(inter)), "pair_counts")

    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    def barrier():
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # ---- warm-up ----
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            check(L.mxg_engine_step(e, 1), "step")
    barrier()
    check(L.mxg_engine_status(e), "warmup status")

    # ---- timed region: device-resident ----
    K = args.steps
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(K)]
    clk = Clocks(local)
    clk.start()
    barrier()
    t_wall = time.perf_counter()
    with torch.cuda.stream(stream):
        for k in range(K):
            starts[k].record(stream)
            L.mxg_engine_step(e, 1)
            ends[k].record(stream)
            flush.zero_()
    barrier()
    t_wall = time.perf_counter() - t_wall
    clocks = clk.stop()
    rc = L.mxg_engine_status(e)
    if rc < 0:
        raise RuntimeError(f"engine status {rc} after the timed steps")
    ms = max_over_ranks(sum(s.elapsed_time(t) for s, t in zip(starts, ends)), world, dev)
    value = job_rate(world, n, K, ms)

    # ---- e2e through the C ABI with pinned host buffers ----
    hpos = torch.empty(n * 16, dtype=torch.uint8, pin_memory=True)
    hvel = torch.empty(n * 16, dtype=torch.uint8, pin_memory=True)
    hen = torch.zeros(2, dtype=torch.float64, pin_memory=True)
    pe = ctypes.c_void_p(hpos.data_ptr())
    ve = ctypes.c_void_p(hvel.data_ptr())
    ee = ctypes.cast(ctypes.c_void_p(hen.data_ptr()), ctypes.POINTER(ctypes.c_double))
    check(L.mxg_engine_copy_state(e, pe, ve, 0), "copy_state")
    with torch.cuda.stream(stream):  # warm-up of this path (untimed)
        for _ in range(3):
            L.mxg_engine_copy_state(e, pe, ve, 1)
            L.mxg_engine_step(e, 1)
            L.mxg_engine_copy_state(e, pe, ve, 0)
            L.mxg_engine_energy_async(e, ee)
    Ke = max(100, min(K, 500))
    s2 = [torch.cuda.Event(enable_timing=True) for _ in range(Ke)]
    e2 = [torch.cuda.Event(enable_timing=True) for _ in range(Ke)]
    barrier()
    with torch.cuda.stream(stream):
        for k in range(Ke):
            s2[k].record(stream)
            L.mxg_engine_copy_state(e, pe, ve, 1)
            L.mxg_engine_step(e, 1)
            L.mxg_engine_copy_state(e, pe, ve, 0)
            L.mxg_engine_energy_async(e, ee)
            e2[k].record(stream)
            flush.zero_()
    barrier()
    ms_e2e = max_over_ranks(sum(s.elapsed_time(t) for s, t in zip(s2, e2)), world, dev)
    e2e_raw = job_rate(world, n, Ke, ms_e2e)

    # ---- e2e through the reference's own data format: engine_load (absolute positions and
    # velocities by particle id, from pinned host memory), engine_step, engine_unload (the same
    # arrays back), on the host's clock around the synchronised calls ----
    hx = torch.empty((n, 3), dtype=torch.float64, pin_memory=True)
    hv = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
    xp = ctypes.cast(ctypes.c_void_p(hx.data_ptr()), ctypes.POINTER(ctypes.c_double))
    vp = ctypes.cast(ctypes.c_void_p(hv.data_ptr()), ctypes.POINTER(ctypes.c_float))
    check(L.mxg_engine_unload(e, n, xp, vp, None, None, None), "unload")
    # warm-up of this path (untimed): the first load allocates the engine's staging buffers
    for _ in range(3):
        check(L.mxg_engine_load(e, n, xp, vp), "load")
        check(L.mxg_engine_step(e, 1), "step")
        check(L.mxg_engine_unload(e, n, xp, vp, None, None, None), "unload")
    # five blocks of round trips, each timed on the host clock as a whole (its mean per round
    # trip); the figure is the median block, so that one stall of the host (another process
    # scheduled on the core for some milliseconds) does not set it
    NB, KB = 5, max(20, min(K, 40))
    Kl = NB * KB
    blocks = []
    barrier()
    for b in range(NB):
        t_l = time.perf_counter()
        for k in range(KB):
            check(L.mxg_engine_load(e, n, xp, vp), "load")
            check(L.mxg_engine_step(e, 1), "step")
            check(L.mxg_engine_unload(e, n, xp, vp, None, None, None), "unload")
        torch.cuda.synchronize(dev)
        blocks.append(1e3 * (time.perf_counter() - t_l) / KB)
    ms_l = max_over_ranks(float(np.median(blocks)), world, dev)
    barrier()
    check(L.mxg_engine_status(e), "e2e status")
    e2e = job_rate(world, n, 1, ms_l)

    # ---- roofline of the dominant kernel (nonbonded forces) ----
    # the force kernel alone, per launch, L2 flushed before each launch; the median
    R = 50
    per = np.zeros(R)
    barrier()
    check(L.mxg_engine_time_force_launches(e, R, ctypes.c_void_p(flush.data_ptr()), flush.numel(),
                                           per.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "time_force")
    barrier()
    force_ms = float(np.median(per))
    flops = F_CAND * cand.value + F_INT_DPD * inter.value
    peaks = measured_peaks()
    sm_count = torch.cuda.get_device_properties(dev).multi_processor_count
    max_mhz = (peaks or {}).get("sm_max_mhz", 1965.0)
    fp32_peak = sm_count * 128 * 2 * max_mhz * 1e6 / 1e12  # TFLOP/s, nominal (no measured FP32 figure)
    achieved = flops / (force_ms / 1e3) / 1e12
    roofline = {"bound": "fp32", "kernel": "force_kernel (nonbonded cell-pair forces)", "achieved": achieved,
                "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                "peak_source": f"nominal FP32 pipe: {sm_count} SMs x 128 lanes x 2 x {max_mhz:.0f} MHz "
                               "(MEASURED_PEAKS.json holds no FP32 figure)",
                "algorithmic_flops_per_launch": flops, "candidate_pairs": cand.value,
                "interacting_pairs": inter.value,
                "flops_per_pair": {"candidate": F_CAND, "interacting_dpd": F_INT_DPD},
                "force_ms_per_launch": force_ms}
    counters, counters_note = captured_counters() if n == 200000 else (None, "no capture of this size")
    traffic = counters.get("dram_bytes_per_launch") if counters else None
    roofline.update({"traffic": traffic, "traffic_unit": "bytes per launch", "traffic_source": counters_note,
                     "sources_sha16": sources_sha16()})
    # the same launch against the measured HBM copy bandwidth: compulsory state bytes (position and
    # velocity read, force written, 16 B each per particle) over the launch time, and the captured
    # DRAM traffic over the same time; both far below the bound, so HBM does not limit this kernel
    hbm_peak = (peaks or {}).get("hbm_gbs")
    if hbm_peak:
        state_bytes = 48 * n
        roofline["hbm_view"] = {
            "peak": hbm_peak, "unit": "GB/s", "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)",
            "algorithmic_bytes_per_launch": state_bytes,
            "achieved": state_bytes / (force_ms / 1e3) / 1e9,
            "frac": state_bytes / (force_ms / 1e3) / 1e9 / hbm_peak,
            "traffic_rate": (traffic / (force_ms / 1e3) / 1e9) if traffic else None}
    if counters and counters.get("warp_instructions_per_launch"):
        # the limiter the counters show: instruction issue (one warp instruction per scheduler
        # per clock, four schedulers per SM), from the capture of these sources
        wi = counters["warp_instructions_per_launch"]
        issue_peak = sm_count * 4 * max_mhz * 1e6 / 1e9
        issue = wi / (force_ms / 1e3) / 1e9
        roofline["issue_view"] = {
            "warp_instructions_per_launch": wi, "achieved": issue, "peak": issue_peak,
            "unit": "G warp-instructions/s", "frac": issue / issue_peak,
            "peak_source": f"{sm_count} SMs x 4 schedulers x {max_mhz:.0f} MHz (nominal issue rate)"}

    # ---- re-binning against the measured HBM bandwidth: the integrator (advance + mover counts)
    # and the scatter (re-binning + next key bounds), each timed with CUDA events at the phase
    # boundaries of whole steps (kernel by kernel, no L2 flush: the integrator reads the received
    # planes the force pass just wrote); algorithmic bytes 88 per particle for each (integrate:
    # pos, vel, force, type read, pos, vel, cell written; scatter: key, pos, vel, id, type read
    # and written) ----
    tm = (ctypes.c_double * 16)()
    Kt = 20
    barrier()
    check(L.mxg_engine_step_timed(e, Kt, tm, 16), "step_timed")
    barrier()
    if hbm_peak:
        rb = {"peak": hbm_peak, "unit": "GB/s", "bytes_per_particle": 88,
              "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)", "steps": Kt}
        for name, slot in (("integrate_kernel", 11), ("scatter_kernel", 14)):
            t = tm[slot] / Kt
            rate = 88 * n / (t / 1e3) / 1e9
            rb[name] = {"ms_per_launch": t, "achieved": rate, "frac": rate / hbm_peak}
        roofline["rebin_view"] = rb

    # ---- CPU baseline and accuracy (reference engine, rank 0, N=1 only) ----
    cpu = None
    accuracy = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            from oracle import refengine
            if refengine.available():
                ref = refengine.run(dict(scn, action="force", runners=os.cpu_count() or 1))
                d = f_gpu.astype(np.float64) - ref["f"]
                accuracy = {"force_rel_rms_vs_reference": float(np.sqrt((d ** 2).sum() / (ref["f"].astype(np.float64) ** 2).sum())),
                            "cells_equal": bool(np.array_equal(c0, ref["cell"])), "tolerance": 1e-5}
                cpu, _ = cpu_baseline(scn, args.cpu_seconds)
        except Exception as exc:  # the baseline is reported, not required
            cpu = {"error": str(exc)[:300]}

    m.universe.close()
    forms = None
    if rank == 0 and world == 1 and not args.no_forms:
        forms = forms_and_configs(args, stream, flush)

    line = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded uniform positions, Maxwell-Boltzmann velocities, kT=1)",
            "config": {"workload": WORKLOAD, "particles_per_gpu": n, "cells": scn["cells"],
                       "l2": "flushed between steps (256 MiB write outside the per-step CUDA events)",
                       "rng": "reference DPD random term (xi = 1)", "parallelism": f"replicas x{world}"},
            "clocks": clocks, "gpu_launches": 3 * K,
            "e2e": {"value": e2e, "unit": "particle-steps/s", "steps": Kl, "h2d_bytes_per_step": 36 * n,
                    "d2h_bytes_per_step": 36 * n,
                    "statistic": f"median of {NB} blocks of {KB} round trips, each block timed as a whole "
                                 "on the host clock (its mean per round trip)",
                    "block_ms_per_step": [round(x, 4) for x in blocks],
                    "path": "mxg_engine_load (absolute x double[3], v float[3] by id, pinned host -> device; "
                            "placement and (cell, id) ordering on the device), mxg_engine_step, "
                            "mxg_engine_unload (x, v by id, device -> pinned host); host wall clock",
                    "raw_state_copy": {"value": e2e_raw, "steps": Ke, "h2d_bytes_per_step": 32 * n,
                                       "d2h_bytes_per_step": 32 * n + 16,
                                       "path": "mxg_engine_copy_state (slot-order float4 pos, vel), mxg_engine_step, "
                                               "mxg_engine_copy_state back, mxg_engine_energy_async; CUDA events"}},
            "roofline": roofline, "cpu_baseline": cpu, "accuracy": accuracy,
            "forms": forms, "wall_s_timed_region": t_wall}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
