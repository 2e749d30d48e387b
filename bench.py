#!/usr/bin/env python
"""Benchmark: MD throughput (atom-steps/s) of 98,304-atom water NVE on one
B200, BF16/FP32 mixed form beside the plain FP32 form.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One "step" is one velocity-Verlet MD step of the whole box through the
device-resident engine: drift test + gated neighbour rebuild, status checks,
the force/virial evaluation and both half kicks (deepmd_jax/md.py:763-795).
Synthetic input: the water builder (O on a 32^3 lattice with N(0, 0.1 A)
jitter, H at gas-phase geometry, Maxwell-Boltzmann velocities at 300 K) and
the random-init se_a model (25-50-100 / 240^3 / axis 16, rcut 6 A).
Multi-GPU: the MD path does not shard here (replicas only) - each rank runs
its own replica and the job value is the sum over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "deepmd-jax_b200"))
sys.path.insert(0, ROOT)

METRIC = "atom-steps/s, 98k-atom water MD (NVE, dt 0.5 fs), mixed vs plain FP32 on 1 B200"
N_SIDE, BOX = 32, 99.3
DT = 0.5
CHUNK = 10
WORKLOAD = ("98,304-atom water (32,768 H2O, L=99.3 A), NVE velocity Verlet dt 0.5 fs, "
            "random-init se_a model 25-50-100/240^3/axis 16, rcut 6 A, skin 0.3 A")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp32"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ncu-case", action="store_true",
                    help="profiling case: plain MD steps (direct launches, no timing) for ncu")
    ap.add_argument("--n-side", type=int, default=N_SIDE, help="waters per box side (profiling case)")
    ap.add_argument("--serve-seconds", type=float, default=4.0, help="serving study: seconds of arrivals")
    ap.add_argument("--serve-in-bench", type=float, default=2.0,
                    help="seconds of serving arrivals (mixed form) measured after the MD line; 0 skips")
    ap.add_argument("--study", default="none", choices=["none", "drift", "pimd", "serving"],
                    help="drift: NVE total-energy drift of both forms on the 98,304-atom box; "
                         "pimd: 32-bead PILE-L throughput of both forms (1,536-atom water)")
    ap.add_argument("--report-every", type=int, default=100, help="drift study: steps between energy samples")
    return ap.parse_args()


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region: NVML
    polled every 5 ms from a thread (the device found by its UUID, else by
    index), which gives samples inside a region of a few tens of ms; where
    NVML cannot be used, nvidia-smi at 200 ms intervals.  Read-only queries."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))
    PERIOD_S = 0.005

    def __init__(self, index):
        self.index = index
        self.rows = []      # (sm MHz, max sm MHz, [reason names])
        self.proc = None
        self.nvml = None
        self.source = None

    def __enter__(self):
        self._stop = threading.Event()
        if self._open_nvml():
            self._sample_nvml()
            self.t = threading.Thread(target=self._poll_nvml, daemon=True)
            self.t.start()
            self.source = "nvml, %g ms" % (1e3 * self.PERIOD_S)
            return self
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            self.source = "nvidia-smi, 200 ms"
        except Exception:
            self.proc = None
        return self

    def _open_nvml(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = None
            try:
                import torch
                u = str(torch.cuda.get_device_properties(self.index).uuid)
                h = pynvml.nvmlDeviceGetHandleByUUID(u if u.startswith("GPU-") else "GPU-" + u)
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.h = h
            self.mx = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self.reasons_fn = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
            self.nvml = pynvml
            return True
        except Exception:
            self.nvml = None
            return False

    def _sample_nvml(self):
        try:
            sm = float(self.nvml.nvmlDeviceGetClockInfo(self.h, self.nvml.NVML_CLOCK_SM))
            mask = int(self.reasons_fn(self.h))
            self.rows.append((sm, self.mx, [n for n, bit in self.REASONS if mask & bit]))
        except Exception:
            pass

    def _poll_nvml(self):
        while not self._stop.wait(self.PERIOD_S):
            self._sample_nvml()

    def _read(self):
        for line in self.proc.stdout:
            r = [x.strip() for x in line.split(",")]
            try:
                sm, mx = float(r[1]), float(r[2])
            except (ValueError, IndexError):
                continue
            self.rows.append((sm, mx, [n for k, (n, _) in enumerate(self.REASONS)
                                       if len(r) > 5 + k and r[5 + k] == "Active"]))

    def __exit__(self, *a):
        self._stop.set()
        if self.nvml is not None:
            self.t.join(timeout=5)
            self._sample_nvml()   # the end of the region
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "source": self.source}
        return {"sm_mhz": statistics.median(r[0] for r in self.rows), "sm_max_mhz": max(r[1] for r in self.rows),
                "reasons": sorted({n for r in self.rows for n in r[2]}), "samples": len(self.rows),
                "source": self.source}


# ----------------------------------------------------------------------------- work model
EMB_FWD_FLOP_ROW = 2 * (25 + 25 * 50 + 50 * 100) + 2 * 10 * 100          # 14,550
EMB_BWD_FLOP_ROW = 2 * (25 + 2 * 25 * 50 + 2 * 50 * 100) + 2 * 2 * 10 * 100  # 29,050
FIT_FLOP_ATOM = 2 * 2 * (1600 * 240 + 2 * 240 * 240)                       # fwd + adjoint GEMMs
G_FLOP_ATOM = 2 * 16 * 100 * 10 * 3                                        # G and its adjoint


def max_over_ranks(x, dist=None, device="cuda"):
    """The slowest rank's time: every rank contributes its own figure and all
    get the maximum (a no-op on one rank)."""
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, world, seconds):
    """Whole-job throughput of independent replicas: the units every rank
    processed over the slowest rank's time."""
    return units_per_rank * world / seconds


def rows_within_rcut(pos_sorted, nbrs, type_count, sel, box, rcut):
    """Average number of (centre, neighbour) rows with 0 < r < rcut."""
    import torch
    N = pos_sorted.shape[0]
    offs = [0]
    for c in type_count:
        offs.append(offs[-1] + c)
    col = 0
    total = 0
    L = torch.tensor(box, dtype=torch.float32, device=pos_sorted.device)
    for j, s in enumerate(sel):
        idx = nbrs[:, col:col + s].long()
        valid = idx < type_count[j]
        g = offs[j] + idx.clamp(max=type_count[j] - 1)
        d = pos_sorted[g] - pos_sorted[:, None, :]
        d = torch.remainder(d - L / 2, L) - L / 2
        r = d.norm(dim=-1)
        total += int(((r < rcut) & (r > 1e-14) & valid).sum())
        col += s
    return total / N


# ----------------------------------------------------------------------------- reference arm
def reference_arm(args):
    """The reference's own CPU implementation cannot run here (pure JAX, jax is
    not installed); its CPU restatement (oracle, torch FP32 on all host cores)
    is timed instead on MD steps of the 12,288-atom box."""
    import torch
    import numpy as np
    from deepmd_jax_b200.systems import water_box, init_dp_params, nnbrs_rule, MASS_UNIT_CONVERSION
    from oracle import model as om, nlist as onl
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    w0 = water_box(4, 12.42, seed=0)
    params, variables = init_dp_params(nnbrs=nnbrs_rule(w0["position"], w0["box"], w0["type_idx"], 6.0))
    w = water_box(16, 49.66, seed=0)
    m = om.OracleModel(params, variables, torch.float32)
    cnt = np.bincount(w["type_idx"], minlength=2)
    sel = [46, 92]

    # the neighbour list (skin 0.3 A) stays valid over the few timed steps,
    # as in the reference's soft update; it is built once, outside the timing
    c = onl.canonicalize(w["position"], w["box"], w["type_idx"])
    nb, _, _ = onl.typed_nlist(c, w["box"].astype(np.float32), onl.cutoff_sq(6.3), cnt, sel)

    def forces(pos):
        r = om.energy_force(m, pos, w["box"], w["type_idx"], nbrs=nb, sel=sel, virial=False)
        return r["force"]

    mass = (w["mass"] * MASS_UNIT_CONVERSION)[:, None]
    r, p = w["position"].copy(), w["velocity"] * mass
    F = forces(r)

    def vv_step(r, p, F):
        p = p + 0.5 * DT * F
        r = r + DT * p / mass
        F = forces(r)
        return r, p + 0.5 * DT * F, F

    # at most 3 untimed and 3 timed steps (about 2 s each on 16 cores)
    warm = max(0, min(args.warmup, 3))
    for _ in range(warm):
        r, p, F = vv_step(r, p, F)
    steps = max(1, min(args.steps, 3))
    t0 = time.perf_counter()
    for _ in range(steps):
        r, p, F = vv_step(r, p, F)
    dt = time.perf_counter() - t0
    N = len(r)
    val = N * steps / dt
    install = _reference_install_state()
    return {"metric": METRIC, "value": val, "unit": "atom-steps/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": steps, "warmup": warm, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "form": "reference (CPU restatement)", "parallelism": "single",
                       "cpu_sample": "12,288-atom box (4,096 H2O, L=49.66 A), same model and step",
                       "sample_atoms": N, "same_config": False,
                       "extrapolation": "atom-steps/s of the 12,288-atom sample, taken per atom-step for the "
                                        "98,304-atom workload; neighbour list built outside the timed steps"},
            "cpu_baseline": {"value": val, "unit": "atom-steps/s", "cores": threads, "kind": "port",
                             "sample": "%d velocity-Verlet steps of the 12,288-atom water box with the FP32 "
                                       "torch restatement of the reference model (the reference is JAX and "
                                       "cannot be installed here)" % steps},
            "e2e": {"value": val, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "reference_install": install}


def _reference_install_state():
    """Why the reference itself is not the timed arm: import it from
    baseline/_ref (installed there with --no-deps) and report the outcome."""
    path = os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isdir(path):
        return "baseline/_ref absent (pip install fails: dependency jax-md is a git URL, no network)"
    code = "import sys; sys.path.insert(0, %r); import deepmd_jax" % path
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    if r.returncode == 0:
        return "deepmd_jax imports from baseline/_ref (jax present); the port is still timed"
    return "baseline/_ref holds deepmd_jax 0.2.1 (--no-deps); import fails: " + (r.stderr.strip().splitlines() or ["?"])[-1]


def cpu_baseline_sample():
    """Short CPU sample for the GPU arm's cpu_baseline key (same port)."""
    class A:
        steps, warmup, gpus = 1, 0, 1
    r = reference_arm(A)
    return r["cpu_baseline"]


# ----------------------------------------------------------------------------- GPU arm
def gpu_arm(args, rank, world, local_rank):
    import numpy as np
    import torch
    from deepmd_jax_b200 import _lib
    from deepmd_jax_b200.md import Simulation
    from deepmd_jax_b200.systems import water_box, init_dp_params, nnbrs_rule
    torch.cuda.set_device(local_rank)
    lib = _lib.load()
    lib.dpb_profile_enable.argtypes = [ctypes.c_int]
    lib.dpb_profile_read.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint64)]
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    w0 = water_box(4, 12.42, seed=0)
    params, variables = init_dp_params(nnbrs=nnbrs_rule(w0["position"], w0["box"], w0["type_idx"], 6.0))
    w = water_box(N_SIDE, BOX, seed=rank)
    N = len(w["position"])

    def make_sim(precision):
        return Simulation((params, variables), w["box"], w["type_idx"], w["mass_per_type"], "NVE", DT,
                          w["position"], initial_velocity=w["velocity"], report_interval=10 ** 9,
                          precision=precision, verbose=False)

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed_device_steps(sim, K, graph=True):
        sim._use_graph = graph
        n_full, rem = divmod(K, CHUNK)
        barrier()
        torch.cuda.synchronize()
        l0 = lib.dpb_kernel_launch_count()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(n_full):
            sim._run_chunk(CHUNK, None, None)
        if rem:
            sim._run_chunk(rem, None, None)
        e.record()
        torch.cuda.synchronize()
        barrier()
        ms = s.elapsed_time(e)
        launches = lib.dpb_kernel_launch_count() - l0 + sim._graph_launches_replayed
        sim._graph_launches_replayed = 0
        return max_over_ranks(ms, dist), launches

    results = {}
    for prec in (["fp32", "mixed"] if args.precision == "mixed" else ["fp32"]):
        try:
            sim = make_sim(prec)
        except Exception as ex:  # precision not available
            results[prec] = {"error": str(ex)}
            continue
        # warm-up in the timed chunk shape, so every CUDA graph is captured before timing
        timed_device_steps(sim, max(args.warmup, 3))
        timed_device_steps(sim, CHUNK)
        with ClockSampler(local_rank) as clk:
            ms, launches = timed_device_steps(sim, args.steps)
        r = sim._report_struct()
        # per-stage durations, live, with CUDA events on the launching stream (direct launches)
        lib.dpb_profile_enable(1)
        _, _ = timed_device_steps(sim, min(args.steps, 10), graph=False)
        stages = {}
        for sid, name in enumerate(["nlist", "embed_fwd", "fit", "embed_bwd", "integrate",
                                    "mixed_embed_fwd", "mixed_fit", "mixed_embed_bwd", "mixed_dT"]):
            msr, cnt = ctypes.c_double(), ctypes.c_uint64()
            lib.dpb_profile_read(sid, ctypes.byref(msr), ctypes.byref(cnt))
            if cnt.value:
                stages[name] = (msr.value / cnt.value, cnt.value)
        lib.dpb_profile_enable(0)
        results[prec] = dict(ms=ms, launches=launches, clocks=clk.summary(), stages=stages, sim=sim,
                             launch_shapes=sim.launch_shapes,
                             status=int(r.status), rebuilds=int(r.rebuilds), steps=int(r.steps))
    head = "mixed" if "mixed" in results and "error" not in results["mixed"] else "fp32"
    R = results[head]
    K = args.steps
    value = job_rate(N * K, world, R["ms"] / 1e3)
    # rows with s(r) != 0 (the work the kernels do; padded slots are skipped)
    sim = R["sim"]
    ptrs = None
    pos_sorted = torch.tensor(np.ascontiguousarray(w["position"][sim._perm]), dtype=torch.float32, device="cuda")
    from deepmd_jax_b200.engine import NeighborBuilder
    nbb = NeighborBuilder(N, 1, sim._type_count, sim._sel, w["box"], 6.3)
    nb, _ = nbb.build(pos_sorted[None].contiguous())
    rows = rows_within_rcut(pos_sorted, nb[0], list(sim._type_count), list(sim._sel), list(w["box"]), 6.0)
    flop_atom = rows * (EMB_FWD_FLOP_ROW + EMB_BWD_FLOP_ROW) + FIT_FLOP_ATOM + G_FLOP_ATOM
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak_src = "of measured"
    except Exception:
        peak_src = "of fallback"
    pk_tensor = float(peaks.get("bf16_tflops", 1590.0))
    stg = R["stages"]
    pref = "mixed_" if head == "mixed" else ""
    cand = {k: v for k, v in stg.items() if k.startswith(pref) or head == "fp32"}
    dom = max(cand, key=lambda k: cand[k][0]) if cand else None
    flop_stage = {"embed_fwd": rows * EMB_FWD_FLOP_ROW, "embed_bwd": rows * EMB_BWD_FLOP_ROW,
                  "fit": FIT_FLOP_ATOM}
    roof = None
    traffic = {}
    try:
        traffic = json.load(open(os.path.join(ROOT, "profiles", "roofline_traffic.json")))
    except Exception:
        pass
    if dom:
        key = dom.replace("mixed_", "")
        fl = flop_stage.get(key, 0) * N
        t_ms = cand[dom][0]
        ach = fl / (t_ms / 1e3) / 1e12 if fl else 0.0
        tr = traffic.get(dom)
        roof = {"bound": "tensor", "achieved": ach, "peak": pk_tensor, "unit": "TFLOP/s",
                "frac": ach / pk_tensor, "traffic": tr["bytes_per_step"] if tr else None,
                "traffic_source": tr["source"] if tr else None, "kernel": dom, "launch_ms": t_ms,
                "algorithmic_flop_per_launch": fl, "peak_source": peak_src + " (bf16 dense, burst)"}
    line = {
        "metric": METRIC, "value": value, "unit": "atom-steps/s", "n_gpus": world, "steps": K,
        "warmup": max(args.warmup, 3), "ms_per_step": R["ms"] / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "bf16+f32" if head == "mixed" else "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD,
                   "form": head, "parallelism": "replicas" if world > 1 else "single",
                   "l2": "working set > L2 (per-step scratch ~2 GB)", "rows_per_atom_within_rcut": rows,
                   "algorithmic_gflop_per_step": flop_atom * N / 1e9},
        "ns_per_day": 1e-6 * DT * 86400 * K / (R["ms"] / 1e3),
        "gpu_launches": int(R["launches"]),
        "clocks": R["clocks"],
        "roofline": roof,
        "forms": {p: {"atom_steps_per_s": N * K * world / (v["ms"] / 1e3), "ms_per_step": v["ms"] / K,
                      "stage_ms": {k: s[0] for k, s in v["stages"].items()}, "status": v["status"],
                      "rebuilds": v["rebuilds"], "launch_shapes": v["launch_shapes"]} if "error" not in v else v
                  for p, v in results.items()},
    }
    if "mixed" in line["forms"] and "fp32" in line["forms"] and "error" not in results.get("mixed", {"error": 1}):
        line["mixed_over_fp32"] = line["forms"]["mixed"]["atom_steps_per_s"] / line["forms"]["fp32"]["atom_steps_per_s"]
    # e2e through the public API: host state in, trajectory of every step out
    if not args.no_e2e:
        sim2 = R["sim"]
        sim2._use_graph = True
        # untimed warm-up of the same call: captures the graphs that write the
        # per-step trajectory buffers and faults in the host trajectory arrays
        sim2.setPosition(w["position"])
        sim2.setVelocity(w["velocity"])
        sim2.run(K)
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim2.setPosition(w["position"])
        sim2.setVelocity(w["velocity"])
        traj = sim2.run(K)
        torch.cuda.synchronize()
        dt_e2e = time.perf_counter() - t0
        barrier()
        dt_e2e = max_over_ranks(dt_e2e, dist)
        line["e2e"] = {"value": job_rate(N * K, world, dt_e2e), "unit": "atom-steps/s",
                       "h2d_bytes_per_step": int(2 * N * 3 * 8 / K),
                       "d2h_bytes_per_step": int(2 * N * 3 * 8),  # user-order float64 positions + velocities
                       "api": "Simulation.setPosition + setVelocity + run(K) returning the per-step trajectory"}
    if rank == 0 and world == 1 and args.serve_in_bench > 0:
        # the serving workload's latency line (BASELINE's p50 / p99): Poisson
        # arrivals at 200 requests/s of evaluate() and MD-continuation requests
        sv = study_serving(args, forms=("mixed",), seconds=args.serve_in_bench)
        f = sv["forms"]["mixed"]
        line["serving"] = {"form": "mixed", "seconds_of_arrivals": sv["seconds_of_arrivals"],
                           "requests": sv["requests"], "md_requests": sv["md_requests"],
                           "eval_p50_s": f["latency"].get("eval", {}).get("p50_s"),
                           "eval_p99_s": f["latency"].get("eval", {}).get("p99_s"),
                           "eval_queue_p50_s": f["latency"].get("eval", {}).get("queue_p50_s"),
                           "eval_service_p50_s": f["latency"].get("eval", {}).get("service_p50_s"),
                           "md_p50_s": f["latency"].get("md", {}).get("p50_s"),
                           "md_p99_s": f["latency"].get("md", {}).get("p99_s"),
                           "frames_per_s": f["frames_per_s"], "atom_evals_per_s": f["atom_evals_per_s"],
                           "wall_s": f["wall_s"],
                           "note": "atom_evals_per_s of the Poisson stream is bounded by its arrival rate; "
                                   "burst_* is the capacity (200 evaluate() requests of the stream at once)",
                           "burst_atom_evals_per_s": f["burst"]["atom_evals_per_s"],
                           "burst_frames_per_s": f["burst"]["frames_per_s"]}
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline_sample()
    for v in results.values():
        v.pop("sim", None)
    if dist is not None:
        dist.destroy_process_group()
    return line


def ncu_case(args):
    """Small fixed case for Nsight Compute: args.warmup + args.steps MD steps
    of a water box of args.n_side^3 molecules, direct kernel launches."""
    import torch
    from deepmd_jax_b200.md import Simulation
    from deepmd_jax_b200.systems import water_box, init_dp_params, nnbrs_rule
    w0 = water_box(4, 12.42, seed=0)
    params, variables = init_dp_params(nnbrs=nnbrs_rule(w0["position"], w0["box"], w0["type_idx"], 6.0))
    n = args.n_side
    w = water_box(n, BOX * n / N_SIDE, seed=0)
    sim = Simulation((params, variables), w["box"], w["type_idx"], w["mass_per_type"], "NVE", DT, w["position"],
                     initial_velocity=w["velocity"], precision=args.precision, use_cuda_graph=False, verbose=False,
                     autotune=False)
    sim._run_chunk(args.warmup + args.steps, None, None)
    torch.cuda.synchronize()
    r = sim._report_struct()
    print(json.dumps({"case": "md", "atoms": len(w["position"]), "precision": args.precision,
                      "steps": args.warmup + args.steps, "status": int(r.status), "pe": r.potential_energy}))
    return 0


def _models():
    from deepmd_jax_b200.systems import water_box, init_dp_params, nnbrs_rule
    w0 = water_box(4, 12.42, seed=0)
    return init_dp_params(nnbrs=nnbrs_rule(w0["position"], w0["box"], w0["type_idx"], 6.0))


def study_drift(args):
    """Total-energy drift of NVE on the 98,304-atom box, FP32 and mixed forms:
    args.steps steps from the same state, the invariant sampled every
    args.report_every steps; slope of a least-squares line in eV/atom/ps."""
    import numpy as np
    import torch
    from deepmd_jax_b200.md import Simulation
    from deepmd_jax_b200.systems import water_box
    params, variables = _models()
    w = water_box(N_SIDE, BOX, seed=0)
    N = len(w["position"])
    out = {"study": "nve_drift", "atoms": N, "dt_fs": DT, "steps": args.steps, "forms": {}}
    # the 192-atom NVE workload over its full 1,000 steps, energy every 10 steps
    w0 = water_box(4, 12.42, seed=0)
    out["config0_1000_steps"] = {}
    for prec in ("fp32", "mixed"):
        sim = Simulation((params, variables), w0["box"], w0["type_idx"], w0["mass_per_type"], "NVE", DT,
                         w0["position"], initial_velocity=w0["velocity"], report_interval=10, precision=prec,
                         verbose=False)
        sim.run(1000, trajectory=False)
        rows = np.array([[r[0], r[4]] for r in sim.log])
        e = rows[:, 1] / len(w0["position"])
        out["config0_1000_steps"][prec] = {
            "drift_eV_per_atom_per_ps": float(np.polyfit(rows[:, 0] * DT / 1000.0, e, 1)[0]),
            "max_dev_eV_per_atom": float(np.abs(e - e[0]).max()),
            "first_100_steps_max_dev_eV_per_atom": float(np.abs(e[:11] - e[0]).max())}
    for prec in ("fp32", "mixed"):
        sim = Simulation((params, variables), w["box"], w["type_idx"], w["mass_per_type"], "NVE", DT,
                         w["position"], initial_velocity=w["velocity"], report_interval=args.report_every,
                         precision=prec, verbose=False)
        t0 = time.perf_counter()
        sim.run(args.steps, trajectory=False)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        rows = np.array([[r[0], r[4]] for r in sim.log])
        t_ps = rows[:, 0] * DT / 1000.0
        e = rows[:, 1] / N
        slope = float(np.polyfit(t_ps, e, 1)[0]) if len(t_ps) > 1 else None
        out["forms"][prec] = {"drift_eV_per_atom_per_ps": slope, "max_dev_eV_per_atom": float(np.abs(e - e[0]).max()),
                              "E0_eV_per_atom": float(e[0]), "samples": len(e), "wall_s": wall,
                              "status": int(sim._report_struct().status)}
    return out


def study_pimd(args):
    """32-bead PILE-L PIMD (1,536-atom water, L = 24.83 A, 300 K, dt 0.25 fs):
    all beads evaluated in one batched launch per kernel; atom-steps/s counts
    beads x atoms, timed with CUDA events over args.steps steps (graphs).
    NVT in both forms, then NPT PIMD (1 bar, Langevin barostat tau_p 1 ps,
    isotropic) in the mixed form."""
    import numpy as np
    import torch
    from deepmd_jax_b200 import _lib
    from deepmd_jax_b200.md import Simulation
    from deepmd_jax_b200.systems import water_box
    params, variables = _models()
    w = water_box(8, 24.83, seed=0)
    N, P = len(w["position"]), 32
    lib = _lib.load()
    out = {"study": "pimd_pile_l", "atoms": N, "beads": P, "dt_fs": 0.25, "steps": args.steps, "forms": {}}
    for prec, routine in (("fp32", "NVT"), ("mixed", "NVT"), ("mixed", "NPT")):
        kw = dict(pressure=1.0, tau_p=1000.0) if routine == "NPT" else {}
        sim = Simulation((params, variables), w["box"], w["type_idx"], w["mass_per_type"], routine, 0.25,
                         w["position"], temperature=300.0, n_bead=P, tau_t=100.0, seed=1,
                         report_interval=10 ** 9, precision=prec, verbose=False, **kw)
        for _ in range(max(args.warmup, 3)):
            sim._run_chunk(1, None, None)
        sim._run_chunk(CHUNK, None, None)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n_full, rem = divmod(args.steps, CHUNK)
        s.record()
        for _ in range(n_full):
            sim._run_chunk(CHUNK, None, None)
        if rem:
            sim._run_chunk(rem, None, None)
        e.record()
        torch.cuda.synchronize()
        ms = s.elapsed_time(e)
        r = sim._report_struct()
        key = prec if routine == "NVT" else "mixed_npt"
        out["forms"][key] = {"atom_steps_per_s": N * P * args.steps / (ms / 1e3), "ms_per_step": ms / args.steps,
                              "ns_per_day": 1e-6 * 0.25 * 86400 * args.steps / (ms / 1e3),
                              "status": int(r.status), "rebuilds": int(r.rebuilds)}
    return out


def study_serving(args, forms=("fp32", "mixed"), seconds=None):
    """Serving stream of the benchmark model: Poisson arrivals at 200
    requests/s for args.serve_seconds; 98 % are evaluate() requests of 1-16
    water frames with the atom count log-uniform in [96, 24,576] (multiples
    of 3; waters on the first n_w sites of a ceil(n_w^(1/3))^3 lattice, box
    12.42 (n_w / 64)^(1/3) A), 2 % are MD continuations of 100 NVT steps on
    3,000-30,000-atom boxes; 60 GB HBM admission budget.  Both forms.
    Latency = submit to result on the host; throughput over the whole run
    (arrivals + drain)."""
    import numpy as np
    import torch
    from deepmd_jax_b200.serving import Server
    from deepmd_jax_b200.systems import serving_water
    params, variables = _models()
    rng = np.random.default_rng(0)
    cache = {}

    def water(n_w):
        if n_w not in cache:
            cache[n_w] = serving_water(n_w, seed=n_w)
        return cache[n_w]

    sched, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / 200.0)
        if t > (args.serve_seconds if seconds is None else seconds):
            break
        if rng.random() < 0.02:
            n_w = int(np.exp(rng.uniform(np.log(1000), np.log(10000))))
            sched.append((t, "md", n_w, 100))
        else:
            n_w = max(32, int(np.exp(rng.uniform(np.log(96), np.log(24576)))) // 3)
            sched.append((t, "eval", n_w, int(rng.integers(1, 17))))
    for _, _, n_w, _ in sched:
        water(n_w)
    out = {"study": "serving", "arrival_rate_per_s": 200,
           "seconds_of_arrivals": args.serve_seconds if seconds is None else seconds,
           "requests": len(sched), "md_requests": sum(1 for x in sched if x[1] == "md"),
           "hbm_budget_GB": 60, "forms": {}}
    for prec in forms:
        with Server((params, variables), precision=prec, hbm_budget=60e9) as srv:
            w = water(64)
            srv.submit_evaluate(w["position"], w["box"], w["type_idx"]).result()   # warm-up
            srv.completed.clear()
            srv.batch_log.clear()
            futs, atoms_eval, frames = [], 0, 0
            # the clients' frames are drawn before the stream starts, so the
            # submitting thread does no numpy work between arrivals
            frames_of = [(w["position"][None] + 0.01 * rng.standard_normal((k,) + w["position"].shape)
                          ).astype(np.float32) if kind == "eval" else None
                         for _, kind, n_w, k in sched for w in (water(n_w),)]
            t0 = time.perf_counter()
            for (ta, kind, n_w, k), pos in zip(sched, frames_of):
                dt = t0 + ta - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
                w = water(n_w)
                if kind == "eval":
                    futs.append(srv.submit_evaluate(pos, w["box"], w["type_idx"]))
                    atoms_eval += k * len(w["type_idx"])
                    frames += k
                else:
                    futs.append(srv.submit_md(w["position"], w["box"], w["type_idx"], w["mass_per_type"], k,
                                              routine="NVT", seed=n_w))
            for f in futs:
                f.result()
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
            lat = srv.latency_summary()
            del frames_of
            out["forms"][prec] = {"latency": lat, "batch_phases": srv.batch_summary(), "wall_s": wall,
                                  "frames_per_s": frames / wall,
                                  "atom_evals_per_s": atoms_eval / wall, "batches": srv.batches,
                                  "mean_batch_atoms": float(np.mean(srv.batch_sizes)) if srv.batch_sizes else 0,
                                  "peak_reserved_GB": srv.budget.peak / 1e9}
            # capacity: the stream's first 200 evaluate() requests submitted at
            # once (the Poisson stream above is bounded by its arrival rate)
            burst = [x for x in sched if x[1] == "eval"][:200]
            futs, b_atoms, b_frames = [], 0, 0
            nb0 = srv.batches
            t1 = time.perf_counter()
            for _, _, n_w, k in burst:
                w = water(n_w)
                pos = w["position"][None] + 0.01 * rng.standard_normal((k,) + w["position"].shape)
                futs.append(srv.submit_evaluate(pos, w["box"], w["type_idx"]))
                b_atoms += k * len(w["type_idx"])
                b_frames += k
            for f in futs:
                f.result()
            wall_b = time.perf_counter() - t1
            out["forms"][prec]["burst"] = {"requests": len(burst), "atom_evals": b_atoms, "wall_s": wall_b,
                                           "atom_evals_per_s": b_atoms / wall_b, "frames_per_s": b_frames / wall_b,
                                           "batches": srv.batches - nb0}
    return out


def main():
    args = parse()
    if args.ncu_case:
        return ncu_case(args)
    if args.study != "none":
        fn = {"drift": study_drift, "pimd": study_pimd, "serving": study_serving}[args.study]
        print(json.dumps(fn(args)))
        return 0
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus if args.gpus == 1 else 1)))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(reference_arm(args)))
        return 0
    line = gpu_arm(args, rank, world, local_rank)
    if rank == 0:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
