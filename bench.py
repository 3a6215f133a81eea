"""Benchmark: simulated ns/s of the MagTense micromagnetic hot path on B200.

Headline workload ("film-batch", the batching configuration): B = 256
instances of the 80x20x1 std-problem-4 thin film (500x125x3 nm, n = 1600,
Ms 8e5 A/m, A 1.3e-11 J/m, K 0) sharing one demag tensor, each driven by a
seeded in-plane field (angle U[0,360) deg, magnitude U[0,50] mT), integrated
for 1 ns at alpha = gamma*0.02 (gamma = 2.211e5) from an s-state with per-
instance RKSUITE 'M' step control, tol 1e-6, output every 1 ps.  The demag
products run as one exact fixed-point tcgen05 GEMM (int8 limbs, kind::i8) per
right-hand-side evaluation inside one persistent kernel; --precision picks the
split-FP16/BF16 or FP32 SIMT products instead.  Seeded synthetic inputs stand in
for the std-problem-4 dataset workflow.  One step = every instance of the
rank integrated over the window.

Other workloads: "film-plain" (the same film, single-instance FP32 path) and
"ragged" (64 films of seeded sizes nx in 20..120, ny = nx/4, each with its own
tensor, field and adaptive steps, in one persistent launch on per-instance SM
groups, replayed from a CUDA graph), "adjoint" (the differentiation configuration: forward and adjoint backward of
a 2 ns fixed-step RK4 trajectory of the film with 200 piecewise-constant field
segments and per-cell Ms) and
"large-plain" (64x64x8 cubes of 5 nm, n = 32768, 25.8 GB FP32 tensor, the
HBM-bound demag matvec).  large-plain --shards W splits that one instance by
receiver rows: on one GPU into W shards run as CTA groups of one launch (the
multi-GPU code path, its peer stores landing in local memory); under torchrun
with W = --gpus over the ranks, each GPU holding 25.8/W GB of tensor rows and
exchanging stage arguments and error norms with its peers through CUDA IPC
regions ("scaling": "strong").

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload film-batch|film-plain|large-plain|adjoint|ragged] [--shards W]

Multi-GPU: one process per GPU (torchrun); instances are sharded across ranks
with no data-path collective ("scaling": "weak"); the step time is the max over
ranks.  --impl reference times the CPU restatement of the reference (oracle/)
on the same workload, rank 0 only: the instances side by side on the host cores,
one single-threaded process each, as the reference runs one problem per thread.

Besides the headline, the default film-batch line carries the FP64 error of
<m>(t) for a seeded sample of instances ("m_err_vs_fp64"), the film-plain path on
those instances ("plain_fp32_same_workload"), the large-plain HBM record
("large_plain"), the ragged and adjoint configurations ("ragged", "adjoint")
and the split 16-bit product next to int8 on a short window
("split16_short_window").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

MU0 = 4 * np.pi * 1e-7
GAMMA = 2.211e5
FILM_RES = (80, 20, 1)
FILM_L = (500e-9, 125e-9, 3e-9)
# DRAM bytes (read + write) per algorithmic tensor byte of the streaming integrator,
# from an ncu capture of large-plain at 32x32x4 (43.906 GB read + 0.065 GB written
# for 43.89 GB of tensor rows)
TRAFFIC_PER_TENSOR_BYTE = (43.906 + 0.065) / 43.89
# DRAM bytes (read + write) per lock-step tick of the batched integrator with all four
# 64-instance tiles active, from an ncu capture of the first 200 ticks of the headline
# workload (38.142 GB read + 11.452 GB written); ticks per full launch of the kernel
BATCH_TRAFFIC_PER_TICK = (38.142e9 + 11.452e9) / 200
BATCH_TICKS_PER_LAUNCH = 4000
LARGE_RES = (64, 64, 8)
LARGE_L = (320e-9, 320e-9, 40e-9)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="film-batch", choices=["film-batch", "film-plain", "large-plain", "adjoint", "ragged"])
    ap.add_argument("--instances", type=int, default=256, help="instances per rank (film-batch)")
    ap.add_argument("--precision", default="int8", choices=["int8", "fp16s", "bf16x3", "bf16x2", "fp32"])
    ap.add_argument("--plain-sample", type=int, default=4,
                    help="film-batch: instances of the same workload run through the plain FP32 path for the ratio")
    ap.add_argument("--window", type=float, default=None, help="simulated ns per instance per step")
    ap.add_argument("--cpu-window", type=float, default=0.3, help="simulated ns of the bounded CPU sample")
    ap.add_argument("--ref-window", type=float, default=0.05,
                    help="film workloads: simulated ns per instance per step of the reference arm (and CPU baseline)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3, help="end-to-end repetitions (median reported)")
    ap.add_argument("--no-fp64", action="store_true", help="film-batch: skip the FP64 error statement")
    ap.add_argument("--no-large", action="store_true", help="film-batch: skip the large-plain sub-record")
    ap.add_argument("--no-others", action="store_true",
                    help="film-batch: skip the ragged, adjoint and precision-study sub-records")
    ap.add_argument("--no-tune", action="store_true", help="film-batch: keep the default GEMM schedule")
    ap.add_argument("--no-split16", action="store_true",
                    help="film-batch: skip the short-window record of the split 16-bit product")
    ap.add_argument("--shards", type=int, default=1,
                    help="large-plain: row shards of the one instance (over the ranks when --gpus > 1)")
    ap.add_argument("--res", type=int, nargs=3, default=None,
                    help="large-plain: override the grid (cubes of 5 nm), e.g. a small case for profiling")
    return ap.parse_args()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), float(d.get("bf16_tflops_sustained", d["bf16_tflops"])), \
            "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


def instance_fields(seed, count):
    rng = np.random.default_rng(seed)
    ang = rng.uniform(0, 2 * np.pi, count)
    mag = rng.uniform(0, 50e-3, count) / MU0
    return np.stack([mag * np.cos(ang), mag * np.sin(ang), np.zeros(count)], 1)


def start_state(n, seed=0):
    """Seeded start: (1,1,1)/sqrt3 + N(0, 0.01^2) per component, renormalised."""
    rng = np.random.default_rng(seed)
    m = np.ones((3, n)) / np.sqrt(3) + 0.01 * rng.standard_normal((3, n))
    return (m / np.linalg.norm(m, axis=0)).reshape(-1)


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.rows.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), int(os.environ.get("LOCAL_RANK", "0"))


# --------------------------------------------------------------------------------------------
# The reference arm and the CPU baseline: the oracle (the CPU restatement of the reference's
# FP32-demag path) on the host cores.  The film workload runs as the reference runs it: one
# problem per process, each process single-threaded (LandauLifshitzEquationSolver.f90:927 sets
# one OpenMP thread), the instances side by side on all host cores.
def film_config(B_total, window, nt):
    """The film-batch workload, identical in both arms' JSON lines."""
    return {"workload": f"film-batch: {B_total} instances of the 80x20x1 std-problem-4 film (n=1600), each "
                        f"{window} ns at alpha_G=0.02 from the s-state (seeded start relaxed 0.2 ns in zero field "
                        "at alpha_G=1), in-plane field seeded per instance (seed 1000: angle U[0,360) deg, "
                        "magnitude U[0,50] mT), per-instance RKSUITE 'M' (tol 1e-6), output every 1 ps",
            "instances": B_total, "window_ns": window, "outputs": nt, "field_seed": 1000,
            "parallelism": "instances split over ranks (device arm) or host processes (reference arm); no "
                           "data-path exchange",
            "l2": "device arm: flushed (256 MB write) before every timed step"}


_REF = {}


def _ref_init(res, L, m_s, fields, window_ns, barrier):
    """Worker set-up (spawned process): one OpenMP thread, one oracle problem per instance."""
    os.environ["OMP_NUM_THREADS"] = "1"
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as O
    K32, _ = O.assemble(list(res), list(L), fp32=True)
    win = window_ns * 1e-9
    _REF.update(O=O, res=res, L=L, m_s=m_s, fields=fields, window_ns=window_ns, K32=K32, probs={},
                barrier=barrier, t=np.linspace(0, win, max(2, int(round(window_ns / 1e-3)) + 1)))


def _ref_run(k):
    """Integrate instance k of the sample over the window from the s-state; returns (start,
    end) wall-clock times and the RHS evaluations.  Every task waits at a barrier of all the
    pool's processes first, so each process holds exactly one task and all start together."""
    R = _REF
    if k not in R["probs"]:
        h = R["fields"][k]
        win = R["window_ns"] * 1e-9
        R["probs"][k] = R["O"].Problem(R["res"], R["L"], mode=0, gamma=GAMMA, alpha=GAMMA * 0.02,
                                       hext=np.array([[0.0, *h], [win, *h]]), K32=R["K32"])
    R["barrier"].wait()
    t0 = time.time()
    _, _, _, st = R["probs"][k].solve(R["t"], R["m_s"], tol=1e-6)
    return t0, time.time(), int(st["f_evals"])


class RefPool:
    """The film workload's instance sample on the host cores through the oracle."""

    def __init__(self, B_total, window_ns, procs=None):
        import multiprocessing as mp
        from oracle import oracle as O
        self.procs = procs or os.cpu_count() or 1
        n = int(np.prod(FILM_RES))
        # the s-state by the same recipe as the device arm, on the oracle (all host threads)
        relax = 0.2e-9
        P = O.Problem(FILM_RES, FILM_L, mode=0, gamma=GAMMA, alpha=GAMMA * 1.0,
                      hext=np.array([[0, 0, 0, 0], [relax, 0, 0, 0.0]]))
        _, yr, _, _ = P.solve(np.linspace(0, relax, 3), start_state(n), tol=1e-6)
        m_s = yr[-1].copy()
        del P
        allf = instance_fields(1000, B_total)
        self.pick = [int(k * B_total // self.procs) for k in range(self.procs)]
        self.window_ns = window_ns
        ctx = mp.get_context("spawn")
        barrier = ctx.Barrier(self.procs)
        self.pool = ctx.Pool(self.procs, initializer=_ref_init,
                             initargs=(FILM_RES, FILM_L, m_s, {k: allf[k] for k in self.pick}, window_ns, barrier))

    def step(self):
        """One step: every process integrates its instance; the step's time runs from the
        common start to the last process's end (set-up and process start-up excluded)."""
        out = self.pool.map(_ref_run, self.pick, chunksize=1)
        wall = max(b for _, b, _ in out) - min(a for a, _, _ in out)
        return wall, sum(e for _, _, e in out)

    def close(self):
        self.pool.close()
        self.pool.join()

    def describe(self, wall, evals):
        return (f"{len(self.pick)} instances of the set (indices {self.pick[0]}, {self.pick[1] if len(self.pick) > 1 else ''}"
                f"...), each integrated over the first {self.window_ns} ns of its window from the s-state by its own "
                f"single-threaded process ({evals} RHS evals, {wall:.1f} s wall); the early part of the window "
                "needs fewer evaluations per ns than the whole window, so this rate is an upper bound for the CPU")


def cpu_film_sample(B_total, window_ns):
    """cpu_baseline of the film workloads: one bounded step of the reference arm."""
    rp = RefPool(B_total, window_ns)
    try:
        wall, evals = rp.step()
    finally:
        rp.close()
    return {"value": len(rp.pick) * window_ns / wall, "unit": "simulated ns/s", "cores": len(rp.pick),
            "kind": "port", "sample": rp.describe(wall, evals)}


def cpu_large_sample(evals_per_ns, rows=256, reps=3):
    """cpu_baseline of large-plain: the 25.8 GB tensor does not fit a bounded CPU sample,
    so the oracle's FP32 demag product (all host threads) is timed on a subset of receiver
    rows and scaled to all n rows; one right-hand side costs that product, and the device
    run's evaluations per simulated ns convert it to simulated ns/s."""
    from oracle import oracle as O
    res, L = LARGE_RES, LARGE_L
    n = int(np.prod(res))
    pick = np.sort(np.random.default_rng(3).choice(n, rows, replace=False))
    K32, _ = O.assemble(list(res), list(L), rows=pick, fp32=True)
    rng = np.random.default_rng(1)
    m = rng.standard_normal((3, n))
    m = (m / np.linalg.norm(m, axis=0)).reshape(-1)
    best = None
    for _ in range(reps):
        t0 = time.perf_counter()
        O.demag_rows(K32, None, m, 8e5, mode=0)
        dt = time.perf_counter() - t0
        best = dt if best is None else min(best, dt)
    t_eval = best * n / rows
    return {"value": 1.0 / (t_eval * evals_per_ns), "unit": "simulated ns/s", "cores": O.threads(), "kind": "port",
            "sample": f"FP32 demag product of {rows} of the {n} receiver rows ({best * 1e3:.1f} ms, best of {reps}) "
                      f"scaled to one right-hand side ({t_eval:.2f} s) and to the device run's {evals_per_ns:.0f} "
                      "evaluations per simulated ns; tensor assembly excluded"}


def run_reference(args):
    ws, rank, _ = dist_setup()
    if rank != 0:
        return
    B_total = ws * args.instances
    window = 1.0 if args.window is None else args.window
    nt = int(round(window / 1e-3)) + 1
    rp = RefPool(B_total, args.ref_window)
    try:
        for _ in range(args.warmup):
            rp.step()
        walls, evals = [], 0
        for _ in range(args.steps):
            w, e = rp.step()
            walls.append(w)
            evals += e
    finally:
        rp.close()
    ms = statistics.mean(walls) * 1e3
    v = len(rp.pick) * args.ref_window / (ms / 1e3)
    cb = {"value": v, "unit": "simulated ns/s", "cores": len(rp.pick), "kind": "port",
          "sample": rp.describe(sum(walls), evals)}
    line = {"metric": "simulated ns/s", "value": v, "unit": "simulated ns/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": film_config(B_total, window, nt),
            "sample_per_step": {"instances": rp.pick, "window_ns": args.ref_window, "processes": len(rp.pick),
                                "threads_per_process": 1},
            "note": "CPU restatement of the reference (oracle/, FP32 demag product as the reference; the Fortran "
                    "reference cannot be built here: no Fortran compiler, no MKL); one single-threaded process "
                    "per host core, each integrating its own instance, as the reference solves one problem per "
                    "single-threaded call",
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "simulated ns/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------------------------
def relaxed_state(torch, res, L, relax_ns=0.2):
    """s-state: seeded start relaxed in zero field at alpha_G = 1 (untimed input preparation)."""
    from magtense_b200 import Solver
    n = int(np.prod(res))
    s = Solver(res, L)
    s.assemble()
    s.set_dynamics(solver=2, gamma=GAMMA, alpha=GAMMA * 1.0,
                   hext=np.array([[0, 0, 0, 0], [relax_ns * 1e-9, 0, 0, 0.0]]))
    _, yr, _, _ = s.integrate(np.linspace(0, relax_ns * 1e-9, 3), torch.as_tensor(start_state(n), device="cuda"),
                              tol=1e-6)
    return s, yr[-1].clone()


def timed_steps(torch, step_fn, steps, warmup, dist, local):
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB > L2
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        step_fn()
    times, stats = [], []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        for _ in range(steps):
            flush.fill_(1.0)
            if dist:
                dist.barrier()
            torch.cuda.synchronize()
            ev0.record(stream)
            st = step_fn()
            ev1.record(stream)
            torch.cuda.synchronize()
            times.append(ev0.elapsed_time(ev1))
            stats.append(st)
    return times, stats, clk.summary(), flush


def run_ours(args):
    import torch
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    hbm, bf16, bf16_sus, src = peaks()
    line = None
    if args.workload == "film-batch":
        line = bench_film_batch(torch, args, ws, rank, local, dist, hbm, bf16_sus, src)
    elif args.workload == "adjoint":
        line = bench_adjoint(torch, args, ws, rank, local, dist, hbm, src)
    elif args.workload == "ragged":
        line = bench_ragged(torch, args, ws, rank, local, dist, hbm, src)
    else:
        line = bench_plain(torch, args, ws, rank, local, dist, hbm, src)
    if rank == 0 and line is not None:
        if not args.no_cpu:
            if args.workload == "adjoint":
                line["cpu_baseline"] = cpu_adjoint_sample(args.cpu_window)
            elif args.workload == "ragged":
                line["cpu_baseline"] = cpu_ragged_sample(args.cpu_window)
            elif args.workload == "large-plain":
                line["cpu_baseline"] = cpu_large_sample(line["evals_per_ns"])
            else:
                line["cpu_baseline"] = cpu_film_sample(ws * args.instances, args.ref_window)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def max_over_ranks(torch, dist, vals):
    from magtense_b200.shard import max_over_ranks as mx
    return mx(vals)


def fp64_error(res, L, m_s, fields, window, t, runs):
    """<m>(t) error of device runs against the FP64 oracle (FP64 tensor and FP64 product)
    of the same instances: max over instances, components and the samples that both took
    at the requested time (a flag-3 return every 5000 evaluations moves a sample to the
    internal time, RKSuitef90.f90:1374-1387).  Test infrastructure: runs after timing."""
    from oracle import oracle as O
    n = int(np.prod(res))
    win = window * 1e-9
    _, K64 = O.assemble(list(res), list(L), fp32=False, fp64=True)
    err = {name: 0.0 for name in runs}
    matched = {name: 0 for name in runs}
    evals = []
    for k, h in enumerate(fields):
        P = O.Problem(res, L, mode=1, gamma=GAMMA, alpha=GAMMA * 0.02, hext=np.array([[0.0, *h], [win, *h]]),
                      K64=K64)
        t_ref, y_ref, _, st = P.solve(t, m_s, tol=1e-6)
        evals.append(int(st["f_evals"]))
        m_ref = y_ref.reshape(len(t), 3, n).mean(axis=2)
        for name, per in runs.items():
            t_got, m_got = per[k]
            same = t_got == t_ref
            matched[name] += int(same.sum())
            err[name] = max(err[name], float(np.abs(m_got[same] - m_ref[same]).max()))
    return err, matched, evals


def large_plain_record(torch, hbm, src, local, reps=3):
    """The large single-instance configuration (64x64x8 cubes, n = 32768, 25.8 GB FP32
    tensor streamed from HBM once per right-hand side): device time of the persistent
    integrator over a short window, as tensor GB/s against the measured HBM copy peak."""
    from magtense_b200 import Solver
    res, L = LARGE_RES, LARGE_L
    n = int(np.prod(res))
    rng = np.random.default_rng(1)
    axis = rng.standard_normal(3)
    axis /= np.linalg.norm(axis)
    m = rng.standard_normal((3, n))
    m0 = torch.as_tensor((m / np.linalg.norm(m, axis=0)).reshape(-1), device="cuda")
    h = np.array([10e-3 / MU0, 0.0, 0.0])
    win = 0.002e-9
    s = Solver(res, L, K0=5e3, u_ea=np.tile(axis, (n, 1)))
    try:
        s.assemble()
        s.set_dynamics(solver=2, gamma=GAMMA, alpha=GAMMA * 0.1, hext=np.array([[0.0, *h], [win, *h]]))
        t = np.linspace(0, win, 3)
        s.integrate(t, m0, tol=1e-6)   # warm-up
        runs = []
        with Clocks(local) as clk:
            for _ in range(reps):
                torch.cuda.synchronize()
                _, y, _, st = s.integrate(t, m0, tol=1e-6)
                torch.cuda.synchronize()
                runs.append((st["f_evals"], st["kernel_ms"], st["launches"]))
                del y
        clocks = clk.summary()
    finally:
        s.close()
    evals = sum(r[0] for r in runs)
    kms = sum(r[1] for r in runs)
    gbs = 24.0 * n * n * evals / (kms / 1e3) / 1e9
    return {"workload": "large-plain: 64x64x8 cubes of 5 nm (n=32768, 25.77 GB FP32 tensor), K=5e3 J/m^3 along a "
                        "seeded axis, 10 mT field, alpha_G=0.1, tol 1e-6, 0.002 ns windows",
            "rhs_evals": evals, "kernel_ms": kms, "ms_per_eval": kms / evals,
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                         "traffic": TRAFFIC_PER_TENSOR_BYTE * 24.0 * n * n * evals / sum(r[2] for r in runs),
                         "note": f"integrate_kernel: 24*n^2 tensor bytes per RHS evaluation x {evals} evaluations "
                                 f"over {kms:.1f} ms of device time ({reps} runs); peak {src} HBM copy; traffic in "
                                 "DRAM bytes per launch, scaled from the 32x32x4 ncu capture"},
            "clocks": clocks}


def ragged_record(torch, hbm, src, local, window_ns=0.05, reps=2):
    """The ragged configuration (64 films of the seeded sizes, each its own tensor and
    field, one graph-replayed persistent launch on per-instance SM groups): device time
    of whole integrations of the set after a warm-up, as tensor GB/s."""
    from magtense_b200 import Solver, integrate_ragged
    sizes = ragged_sizes(2, 64)
    fields = instance_fields(1000, 64)
    win = window_ns * 1e-9
    t = np.linspace(0, win, int(round(window_ns / 1e-3)) + 1)
    solvers, m0s = [], []
    try:
        for (res, L), h in zip(sizes, fields):
            s = Solver(res, L)
            solvers.append(s)
            s.assemble()
            s.set_dynamics(solver=2, gamma=GAMMA, alpha=GAMMA * 0.02, hext=np.array([[0.0, *h], [win, *h]]))
            m0s.append(torch.as_tensor(start_state(int(np.prod(res))), device="cuda"))
        integrate_ragged(solvers, t, m0s, tol=1e-6, graph=True)   # warm-up (graph capture)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        runs = []
        with Clocks(local) as clk:
            for _ in range(reps):
                torch.cuda.synchronize()
                ev0.record()
                _, ys, _, st = integrate_ragged(solvers, t, m0s, tol=1e-6, graph=True)
                ev1.record()
                torch.cuda.synchronize()
                runs.append((ev0.elapsed_time(ev1), st))
                del ys
        clocks = clk.summary()
        ns = [s.n for s in solvers]
    finally:
        for s in solvers:
            s.close()
    step_ms = statistics.median(r[0] for r in runs)
    st = runs[-1][1]
    evals = [x["f_evals"] for x in st]
    kms = st[0]["kernel_ms"]
    gbs = sum(24.0 * x * x * e for x, e in zip(ns, evals)) / (kms / 1e3) / 1e9
    return {"workload": f"ragged: 64 films, nx ~ U{{20..120}}, ny = nx/4, 6.25x6.25x3 nm cells (n {min(ns)}..{max(ns)},"
                        f" {sum(24 * x * x for x in ns) / 1e9:.2f} GB of FP32 tensors), seeded in-plane fields, "
                        f"{window_ns} ns each, tol 1e-6, output every 1 ps; one persistent launch sequence on "
                        "per-instance SM groups, replayed from a CUDA graph",
            "value": 64 * window_ns / (step_ms / 1e3), "unit": "simulated ns/s", "ms_per_step": step_ms,
            "rhs_evals_per_instance": {"min": int(min(evals)), "median": float(np.median(evals)), "max": int(max(evals))},
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                         "traffic": None,
                         "note": f"integrate_ragged_kernel: sum over instances of 24*n_k^2 tensor bytes x evaluations "
                                 f"over {kms:.1f} ms of device time; peak {src} HBM copy"},
            "gpu_launches": int(st[0]["launches"]), "clocks": clocks}


def adjoint_record(torch, hbm, src, local, reps=2):
    """The differentiation configuration: forward and adjoint backward of the 2 ns
    fixed-step RK4 trajectory (200 field segments, per-cell Ms), CUDA-event time of whole
    steps after a warm-up."""
    from magtense_b200 import TrajectoryProblem, mean_m_trajectory
    n = int(np.prod(FILM_RES))
    hseg, Ms, m0, tg = adjoint_config(4)
    prob = TrajectoryProblem(FILM_RES, FILM_L, gamma=GAMMA, alpha=GAMMA * 0.02, m0=m0, t_seg=10e-12,
                             steps_per_segment=10, sample_every=10, checkpoint_every=50)
    steps = hseg.shape[0] * prob.steps_per_segment
    tt = prob.dt * prob.sample_every * np.arange(1, steps // prob.sample_every + 1)
    tgt = torch.as_tensor(adjoint_target(tt, tg), device="cuda")

    def step():
        hs = torch.as_tensor(hseg, device="cuda").requires_grad_(True)
        ms = torch.as_tensor(Ms, device="cuda").requires_grad_(True)
        loss = ((mean_m_trajectory(hs, ms, prob)[:, 0] - tgt) ** 2).sum()
        loss.backward()
        return hs.grad, ms.grad

    step()   # warm-up (graph capture of the replayed steps)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times = []
    with Clocks(local) as clk:
        for _ in range(reps):
            torch.cuda.synchronize()
            ev0.record()
            step()
            ev1.record()
            torch.cuda.synchronize()
            times.append(ev0.elapsed_time(ev1))
    clocks = clk.summary()
    step_ms = statistics.median(times)
    rhs_like = steps * (4 + 4 + 2 * 4)
    gbs = 24.0 * n * n * rhs_like / (step_ms / 1e3) / 1e9
    return {"workload": "adjoint: 80x20x1 film, per-cell Ms ~ U[7.5e5, 8.5e5], 200 piecewise-constant in-plane field "
                        "segments over 2 ns, fixed-step RK4 dt = 1 ps; one step = forward + adjoint backward "
                        "(gradients for the 600 field values and 1600 Ms values)",
            "value": 2.0 / (step_ms / 1e3), "unit": "simulated ns/s", "ms_per_step": step_ms,
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                         "traffic": None,
                         "note": f"field_kernel streaming demag: 24*n^2 bytes x {rhs_like} products per step over the "
                                 f"whole step time (the 61 MB tensor sits in L2); peak {src} HBM copy"},
            "clocks": clocks}


def sweep_state(seed, B=512, n=4096):
    """The precision configuration's inputs: mu0 H along x swept from -100 to +100 mT over
    the B instances, each tilted in plane by a seeded +-1 degree, and a shared seeded state
    (1, 0.2, 0) + N(0, 0.1^2) per component, renormalised."""
    rng = np.random.default_rng(seed)
    mag = np.linspace(-100e-3, 100e-3, B) / MU0
    tilt = np.deg2rad(1.0) * rng.choice([-1.0, 1.0], B)
    fields = np.stack([mag * np.cos(tilt), mag * np.sin(tilt), np.zeros(B)], 1)
    m = np.array([1.0, 0.2, 0.0])[:, None] + 0.1 * rng.standard_normal((3, n))
    return fields, (m / np.linalg.norm(m, axis=0)).reshape(-1)


def precision_record(torch, local, window_ns=0.005, precisions=("int8", "fp16s", "bf16x3", "fp32")):
    """The precision configuration (128x32x1 film of 4x4x3 nm cells, n = 4096, 512
    quasi-static field steps relaxing at alpha_G = 1 from a shared state): the batched
    integration with each demag precision over a short window, simulated ns/s from device
    time, and the H_d error of each precision's product against FP64 on seeded rows."""
    from magtense_b200 import BatchSolver
    from oracle import oracle as O
    res, L = (128, 32, 1), (512e-9, 128e-9, 3e-9)
    n, B = 4096, 512
    fields, m_sh = sweep_state(3, B, n)
    win = window_ns * 1e-9
    t = np.linspace(0, win, int(round(window_ns / 1e-3)) + 1)
    hext = np.zeros((B, 2, 4))
    hext[:, 1, 0] = win
    hext[:, :, 1:] = fields[:, None, :]
    m0 = torch.as_tensor(np.tile(m_sh, (B, 1)), device="cuda")
    # H_d check: per instance the shared state rotated in plane by a seeded angle; 256 seeded
    # receiver rows of the FP64 tensor, 8 of the instances
    rng = np.random.default_rng(4)
    ang = rng.uniform(-np.pi, np.pi, B)
    base = m_sh.reshape(3, n)
    c, s = np.cos(ang)[:, None], np.sin(ang)[:, None]
    mh = np.stack([c * base[0] - s * base[1], s * base[0] + c * base[1], np.broadcast_to(base[2], (B, n))], 1)
    rows = np.sort(rng.choice(n, 256, replace=False))
    check = np.linspace(0, B - 1, 8).astype(int)
    _, K64 = O.assemble(list(res), list(L), rows=rows, fp32=False, fp64=True)
    Href = np.stack([O.demag_rows(None, K64, mh[b], 8e5, mode=1) for b in check])
    mh_dev = torch.as_tensor(mh.reshape(B, -1), device="cuda")
    out = {}
    with Clocks(local) as clk:
        for prec in precisions:
            bs = BatchSolver(res, L, B, precision=prec)
            try:
                bs.assemble()
                H = bs.demag_field(mh_dev).cpu().numpy().reshape(B, 3, n)
                herr = float(np.abs(H[check][:, :, rows] - Href).max() / np.abs(Href).max())
                bs.set_dynamics(hext=hext, alpha=GAMMA * 1.0, gamma=GAMMA)
                bs.integrate(t, m0, tol=1e-6)   # warm-up
                torch.cuda.synchronize()
                _, y, _, st = bs.integrate(t, m0, tol=1e-6)
                torch.cuda.synchronize()
                del y
            finally:
                bs.close()
            ev = [x["f_evals"] for x in st]
            kms = st[0]["kernel_ms"]
            out[prec] = {"value": B * window_ns / (kms / 1e3), "unit": "simulated ns/s", "kernel_ms": kms,
                         "rhs_evals_per_instance": {"min": int(min(ev)), "median": float(np.median(ev)),
                                                    "max": int(max(ev))},
                         "h_d_err_vs_fp64": herr}
    out["workload"] = (f"precision: 128x32x1 film of 4x4x3 nm cells (n = 4096), {B} instances, mu0 H along x swept "
                       f"-100..+100 mT, each tilted by a seeded 1 degree, relaxing at alpha_G = 1 from a shared seeded "
                       f"state, tol 1e-6, {window_ns} ns, output every 1 ps")
    out["note"] = ("device time of one integration per precision after a warm-up; h_d_err_vs_fp64 = max over 8 "
                   "instances, 3 components and 256 seeded receiver rows of |H - H_FP64| / max |H_FP64| for a "
                   "seeded in-plane rotation of the state per instance (FP64 rows from the oracle, outside the "
                   "timed region); the <m>(t) error of these precisions on this geometry is checked in the tests")
    out["clocks"] = clk.summary()
    return out


def split16_record(torch, res, L, m_s, fields, window_ns=0.02, precisions=("fp16s", "int8")):
    """The split 16-bit form of the batched product next to int8 on the same instances
    over a short window: simulated ns/s from device time, RHS evaluations per instance.
    FP32-level rounding in the 16-bit sums sets the step size of the weakest-field
    instances, so the lock-step batch runs at their pace."""
    from magtense_b200 import BatchSolver
    B = len(fields)
    win = window_ns * 1e-9
    t = np.linspace(0, win, int(round(window_ns / 1e-3)) + 1)
    hext = np.zeros((B, 2, 4))
    hext[:, 1, 0] = win
    hext[:, :, 1:] = fields[:, None, :]
    m0 = m_s.unsqueeze(0).expand(B, -1).contiguous()
    out = {}
    for prec in precisions:
        bs = BatchSolver(res, L, B, precision=prec)
        try:
            bs.assemble()
            bs.set_dynamics(hext=hext, alpha=GAMMA * 0.02, gamma=GAMMA)
            bs.integrate(t, m0, tol=1e-6)   # warm-up
            torch.cuda.synchronize()
            _, y, _, st = bs.integrate(t, m0, tol=1e-6)
            torch.cuda.synchronize()
            del y
        finally:
            bs.close()
        ev = [x["f_evals"] for x in st]
        kms = st[0]["kernel_ms"]
        out[prec] = {"value": B * window_ns / (kms / 1e3), "unit": "simulated ns/s", "kernel_ms": kms,
                     "rhs_evals_per_instance": {"min": int(min(ev)), "median": float(np.median(ev)),
                                                "max": int(max(ev))}}
    out["window_ns"] = window_ns
    out["note"] = (f"{B} instances of the headline set over {window_ns} ns from the same s-state, device time of "
                   "one integration after a warm-up; the 16-bit split product accumulates in FP32, whose rounding "
                   "noise sets the step size of the weakest-field instances")
    return out


def bench_film_batch(torch, args, ws, rank, local, dist, hbm, peak_tf, src):
    from magtense_b200 import BatchSolver
    res, L = FILM_RES, FILM_L
    n = int(np.prod(res))
    B = args.instances
    window = 1.0 if args.window is None else args.window
    win = window * 1e-9
    nt = int(round(window / 1e-3)) + 1
    t = np.linspace(0, win, nt)
    plain, m_s = relaxed_state(torch, res, L)
    # the global instance list (ws * B seeded fields), this rank's contiguous slice
    from magtense_b200.shard import shard_range
    a0, a1 = shard_range(ws * B, ws, rank)
    fields = instance_fields(1000, ws * B)[a0:a1]
    hext = np.zeros((B, 2, 4))
    hext[:, 1, 0] = win
    hext[:, :, 1:] = fields[:, None, :]
    bs = BatchSolver(res, L, B, precision=args.precision)
    bs.assemble()
    t0 = time.perf_counter()
    sched = bs.tune() if not args.no_tune else bs.schedule()
    tune_s = time.perf_counter() - t0
    bs.set_dynamics(hext=hext, alpha=GAMMA * 0.02, gamma=GAMMA)
    m0 = m_s.unsqueeze(0).expand(B, -1).contiguous()
    m0_host = m0.cpu().numpy()

    def step():
        _, y, _, st = bs.integrate(t, m0, tol=1e-6)
        return st

    # the plain FP32 single-instance path on the same workload, for the ratio: seeded instances
    # of this rank's set, each integrated over the same window, one after another (before the
    # batched timing, on an idle device)
    pick = sorted(int(k) for k in np.random.default_rng(7).choice(B, size=min(args.plain_sample, B), replace=False))
    plain_s, plain_evals, plain_kms, plain_m = 0.0, 0, 0.0, []
    for k in pick:
        plain.set_dynamics(solver=2, gamma=GAMMA, alpha=GAMMA * 0.02,
                           hext=np.array([[0.0, *fields[k]], [win, *fields[k]]]))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tp, yp, _, pst = plain.integrate(t, m_s, tol=1e-6)
        torch.cuda.synchronize()
        plain_s += time.perf_counter() - t0
        plain_evals += pst["f_evals"]
        plain_kms += pst["kernel_ms"]
        plain_m.append((tp, yp.view(nt, 3, n).mean(dim=2).cpu().numpy()))
        del yp
    plain_rate = len(pick) * window / plain_s
    times, stats, clocks, flush = timed_steps(torch, step, args.steps, args.warmup, dist, local)
    # end to end through the public API: host m0 in (pinned), host trajectories out
    e2e_ms, batch_m = None, None
    if not args.no_e2e:
        pin_in = torch.from_numpy(m0_host).pin_memory()
        pin_out = torch.empty((B, nt, 3 * n), dtype=torch.float64).pin_memory()
        e2e = []
        for _ in range(max(1, min(args.steps, args.e2e_steps))):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            dev_in = pin_in.to("cuda", non_blocking=True)
            # the trajectories stream to the pinned host buffer while the integration runs
            t_b, _, _, _ = bs.integrate(t, dev_in, tol=1e-6, host_out=pin_out)
            torch.cuda.synchronize()
            e2e.append((time.perf_counter() - t0) * 1e3)
        e2e_ms = statistics.median(e2e)
        batch_m = [(t_b[k], pin_out[k].view(nt, 3, n).mean(dim=2).numpy()) for k in pick]
        del pin_out
    step_ms = sum(times) / len(times)   # the K timed steps as one bracket, L2 flushes excluded
    step_ms, e2e_red = max_over_ranks(torch, dist, [step_ms, e2e_ms or 0.0])
    if rank != 0:
        return None
    flat = [x for st in stats for x in st]
    evals = sum(x["f_evals"] for x in flat)
    kms = sum(st[0]["kernel_ms"] for st in stats)
    launches = sum(st[0]["launches"] for st in stats)
    flops = 18.0 * n * n * evals
    achieved = flops / (kms / 1e3) / 1e12
    sim_ns = ws * B * window
    value = sim_ns / (step_ms / 1e3)
    line = {
        "metric": "simulated ns/s", "value": value, "unit": "simulated ns/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
        "config": film_config(ws * B, window, nt),
        "precision": f"{args.precision} tcgen05 demag GEMM inside one persistent kernel",
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak_tf, "unit": "TFLOP/s",
                     "frac": achieved / peak_tf,
                     "traffic": BATCH_TRAFFIC_PER_TICK * BATCH_TICKS_PER_LAUNCH if args.precision == "int8" else None,
                     "traffic_note": "DRAM bytes per full 4000-tick launch, from the per-tick bytes of an ncu capture "
                                     "of 200 ticks with all four instance tiles active (the heaviest ticks: an upper "
                                     "bound for the tail)",
                     "note": f"batch_kernel (the whole persistent integrator, GEMM and RKSUITE coroutines): 18*n^2 "
                             f"useful flops per instance RHS evaluation x {evals} evaluations over {kms:.1f} ms of "
                             f"device time; peak = sustained cuBLAS bf16 ({src})"
                             + ("; the int8 product executes 16 int8 limb products per useful product" if
                                args.precision == "int8" else "")},
        "rhs_evals_per_instance": {"min": int(min(x["f_evals"] for x in stats[-1])),
                                   "median": float(np.median([x["f_evals"] for x in stats[-1]])),
                                   "max": int(max(x["f_evals"] for x in stats[-1]))},
        "plain_fp32_same_workload": {"value": plain_rate, "unit": "simulated ns/s",
                                     "rhs_evals": plain_evals, "instances": pick, "kernel_ms": plain_kms,
                                     "us_per_eval": plain_kms * 1e3 / plain_evals,
                                     "roofline": {"bound": "hbm", "unit": "GB/s", "peak": hbm,
                                                  "achieved": 24.0 * n * n * plain_evals / (plain_kms / 1e3) / 1e9,
                                                  "frac": 24.0 * n * n * plain_evals / (plain_kms / 1e3) / 1e9 / hbm,
                                                  "traffic": None,
                                                  "note": f"integrate_kernel (film-plain): 24*n^2 tensor bytes per "
                                                          f"RHS evaluation over {plain_kms:.1f} ms of device time; the "
                                                          f"61.4 MB tensor is served mostly from L2 (part of its lines "
                                                          f"kept with evict_last); peak {src} HBM copy"},
                                     "note": f"film-plain: the single-instance FP32 path (the reference's arithmetic) "
                                             f"on {len(pick)} seeded instances of the same set, {window} ns each, one "
                                             f"after another"},
        "batched_over_plain": value / ws / plain_rate,
        "gemm_schedule": {"tuned": not args.no_tune, "tuning_s": round(tune_s, 3),
                          "per_active_tiles": [{"tiles": k, "streamk_ctas": g, "order": o} for k, g, o in sched],
                          "note": "autotuned Stream-K schedule of the int8 product (mt_batch_tune), set up before "
                                  "timing"} if args.precision == "int8" else None,
        "gpu_launches": int(launches),
        "rhs_evals_per_s": evals / (sum(times) / 1e3) * ws,
        "clocks": clocks,
    }
    if e2e_ms is not None:
        line["e2e"] = {"value": sim_ns / (e2e_red / 1e3), "unit": "simulated ns/s",
                       "h2d_bytes_per_step": B * 3 * n * 8, "d2h_bytes_per_step": B * nt * 3 * n * 8}
    if not args.no_fp64 and batch_m is not None:
        err, matched, ev = fp64_error(res, L, m_s.cpu().numpy(), [fields[k] for k in pick], window, t,
                                      {args.precision: batch_m, "plain_fp32": plain_m})
        line["m_err_vs_fp64"] = {
            "max_abs_mean_m": err, "samples_compared": matched, "instances": pick, "fp64_rhs_evals": ev,
            "bound": 1e-4, "within_bound": all(v <= 1e-4 for v in err.values()),
            "note": f"max over the {len(pick)} instances, 3 components and all {nt} output samples taken at the "
                    "requested time of |<m>_device - <m>_FP64|, <m> the mean over cells; FP64 = the oracle with "
                    "the FP64 tensor and FP64 demag product, same s-state, field and tolerances, run after timing"}
    if not args.no_large:
        line["large_plain"] = large_plain_record(torch, hbm, src, local)
    if not args.no_others:
        line["ragged"] = ragged_record(torch, hbm, src, local)
        line["adjoint"] = adjoint_record(torch, hbm, src, local)
        line["precision_study"] = precision_record(torch, local)
    if not args.no_split16 and args.precision == "int8":
        bs.close()
        line["split16_short_window"] = split16_record(torch, res, L, m_s, fields)
    return line


def adjoint_config(seed):
    """The differentiation configuration: per-cell Ms ~ U[7.5e5, 8.5e5] A/m, 200 field
    segments over 2 ns with in-plane components ~ U[-20, 20] mT, a seeded three-sinusoid
    target of amplitude 0.5 for <m_x>(t), config-0 start state."""
    rng = np.random.default_rng(seed)
    n = int(np.prod(FILM_RES))
    S = 200
    hseg = np.zeros((S, 3))
    hseg[:, :2] = rng.uniform(-20e-3, 20e-3, (S, 2)) / MU0
    Ms = rng.uniform(7.5e5, 8.5e5, n)
    tg = (rng.uniform(0.0, 0.5 / 3, 3), rng.uniform(2 * np.pi * 1e9, 2 * np.pi * 10e9, 3), rng.uniform(0, 2 * np.pi, 3))
    return hseg, Ms, start_state(n), tg


def adjoint_target(t, tg):
    a, w, ph = tg
    return (a[None, :] * np.sin(w[None, :] * t[:, None] + ph[None, :])).sum(1)


def cpu_adjoint_sample(window_ns):
    """Torch FP64 autograd of a plain right-hand side (FP64 tensor from the oracle) on the
    host cores, same RK4 scheme, on the first window_ns of the trajectory."""
    import torch
    from oracle import oracle as O
    hseg, Ms, m0, tg = adjoint_config(4)
    res, L = FILM_RES, FILM_L
    n = int(np.prod(res))
    _, K64 = O.assemble(list(res), list(L), fp32=False, fp64=True)
    blk = [[0, 1, 2], [1, 3, 4], [2, 4, 5]]
    K = torch.as_tensor(np.block([[K64[blk[a][b]] for b in range(3)] for a in range(3)]))
    nx, ny, _ = res
    d = [L[0] / nx, L[1] / ny]
    mu0 = (4.0 * np.pi) * 1e-7

    def lap(m):
        g = m.reshape(3, ny, nx)
        out = torch.zeros_like(g)
        for ax, nn, dd in ((2, nx, d[0]), (1, ny, d[1])):
            lo = torch.cat([g.narrow(ax, 0, 1), g.narrow(ax, 0, nn - 1)], dim=ax)
            hi = torch.cat([g.narrow(ax, 1, nn - 1), g.narrow(ax, nn - 1, 1)], dim=ax)
            out = out + (lo - 2 * g + hi) / (dd * dd)
        return out.reshape(3, -1)

    dt, spseg, every = 1e-12, 10, 10
    steps = int(round(window_ns * 1e-9 / dt))
    hs = torch.tensor(hseg, requires_grad=True)
    ms = torch.tensor(Ms, requires_grad=True)

    def rhs(m, h):
        he = -h[:, None] - 2 * (1.3e-11 / (mu0 * ms)) * lap(m) - ms * (K @ m.reshape(-1)).reshape(3, -1)
        c = torch.cross(he, m, dim=0)
        return -GAMMA * c - GAMMA * 0.02 * torch.cross(m, c, dim=0)

    t0 = time.perf_counter()
    m = torch.as_tensor(m0.reshape(3, -1))
    samples = []
    for k in range(steps):
        h = hs[k // spseg]
        k1 = rhs(m, h)
        k2 = rhs(m + 0.5 * dt * k1, h)
        k3 = rhs(m + 0.5 * dt * k2, h)
        k4 = rhs(m + dt * k3, h)
        m = m + (dt / 6.0) * (k1 + 2 * k2 + 2 * k3 + k4)
        if (k + 1) % every == 0:
            samples.append(m.mean(dim=1))
    tt = dt * every * np.arange(1, len(samples) + 1)
    loss = ((torch.stack(samples)[:, 0] - torch.as_tensor(adjoint_target(tt, tg))) ** 2).sum()
    loss.backward()
    dtw = time.perf_counter() - t0
    return {"value": window_ns / dtw, "unit": "simulated ns/s", "cores": torch.get_num_threads(), "kind": "port",
            "sample": f"{window_ns} ns of the 80x20x1 trajectory, forward and backward by torch FP64 autograd on the "
                      f"host ({steps} RK4 steps, {dtw:.1f} s); the reference itself computes no gradients"}


def bench_adjoint(torch, args, ws, rank, local, dist, hbm, src):
    from magtense_b200 import TrajectoryProblem, mean_m_trajectory
    n = int(np.prod(FILM_RES))
    hseg, Ms, m0, tg = adjoint_config(4 + rank)
    prob = TrajectoryProblem(FILM_RES, FILM_L, gamma=GAMMA, alpha=GAMMA * 0.02, m0=m0, t_seg=10e-12,
                             steps_per_segment=10, sample_every=10, checkpoint_every=50)
    window = 2.0
    steps = hseg.shape[0] * prob.steps_per_segment
    tt = prob.dt * prob.sample_every * np.arange(1, steps // prob.sample_every + 1)
    tgt = torch.as_tensor(adjoint_target(tt, tg), device="cuda")
    hs_host, ms_host = torch.as_tensor(hseg), torch.as_tensor(Ms)
    out = {}

    def step():
        hs = hs_host.to("cuda").requires_grad_(True)
        ms = ms_host.to("cuda").requires_grad_(True)
        loss = ((mean_m_trajectory(hs, ms, prob)[:, 0] - tgt) ** 2).sum()
        loss.backward()
        out["g"] = (hs.grad, ms.grad)
        return [{"f_evals": 0, "kernel_ms": 0.0, "launches": 0}]

    times, _, clocks, flush = timed_steps(torch, step, args.steps, args.warmup, dist, local)
    e2e = []
    for _ in range(max(1, args.steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        step()
        gh, gm = out["g"][0].cpu(), out["g"][1].cpu()
        torch.cuda.synchronize()
        e2e.append((time.perf_counter() - t0) * 1e3)
    step_ms, e2e_ms = max_over_ranks(torch, dist, [sum(times) / len(times), statistics.median(e2e)])
    if rank != 0:
        return None
    # right-hand sides per step: forward 4 RK4 stages; backward 4 recomputed stages plus 4
    # vector-Jacobian products (each two streaming demag passes)
    rhs_like = steps * (4 + 4 + 2 * 4)
    achieved = 24.0 * n * n * rhs_like / (step_ms / 1e3) / 1e9
    sim_ns = ws * window
    return {
        "metric": "simulated ns/s", "value": sim_ns / (step_ms / 1e3), "unit": "simulated ns/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 (FP32 demag)", "data": "synthetic",
        "config": {"workload": "adjoint: 80x20x1 film, per-cell Ms ~ U[7.5e5, 8.5e5], 200 piecewise-constant "
                               "in-plane field segments over 2 ns ~ U[-20, 20] mT, loss sum_t (<m_x> - target)^2, "
                               "fixed-step RK4 dt = 1 ps, checkpoints every 50 steps; one step = forward + adjoint "
                               "backward (gradients for the 600 field values and 1600 Ms values)",
                   "window_ns": window, "rk4_steps": steps, "parallelism": f"one trajectory per rank, {ws} rank(s)",
                   "l2": "flushed (256 MB write) before every timed step"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None,
                     "note": f"field_kernel streaming demag: 24*n^2 bytes x {rhs_like} products per step over the "
                             f"whole step time (launch- and latency-bound at n = 1600: the 61 MB tensor sits in L2); "
                             f"peak {src} HBM copy"},
        "e2e": {"value": sim_ns / (e2e_ms / 1e3), "unit": "simulated ns/s",
                "h2d_bytes_per_step": (hseg.size + Ms.size) * 8, "d2h_bytes_per_step": (hseg.size + Ms.size) * 8},
        "gpu_launches": int(steps * (4 * 2 + 4 * 2 + 4 * 2)),
        "clocks": clocks,
    }


def ragged_sizes(seed, count=64):
    """Seeded film sizes of the ragged batch: nx ~ U{20..120}, ny = nx // 4, nz = 1, cells of
    6.25 x 6.25 x 3 nm (100 to 3600 cells)."""
    rng = np.random.default_rng(seed)
    nxs = rng.integers(20, 121, count)
    return [((int(nx), int(nx) // 4, 1), (nx * 6.25e-9, (nx // 4) * 6.25e-9, 3e-9)) for nx in nxs]


def cpu_ragged_sample(window_ns):
    """The oracle (FP32 restatement, all host cores) on one mid-sized film of the ragged set."""
    from oracle import oracle as O
    res, L = ragged_sizes(2)[0]
    n = int(np.prod(res))
    h = instance_fields(1000, 1)[0]
    win = window_ns * 1e-9
    P = O.Problem(res, L, mode=0, gamma=GAMMA, alpha=GAMMA * 0.02, hext=np.array([[0.0, *h], [win, *h]]))
    t0 = time.perf_counter()
    _, _, _, st = P.solve(np.linspace(0, win, max(2, int(round(window_ns / 1e-3)) + 1)), start_state(n), tol=1e-6)
    dt = time.perf_counter() - t0
    return {"value": window_ns / dt, "unit": "simulated ns/s", "cores": O.threads(), "kind": "port",
            "sample": f"{window_ns} ns of one {res[0]}x{res[1]}x1 film of the ragged set ({st['f_evals']} RHS evals, "
                      f"{dt:.1f} s); per-instance rate on the host"}


def bench_ragged(torch, args, ws, rank, local, dist, hbm, src):
    from magtense_b200 import Solver, integrate_ragged
    from magtense_b200.shard import shard_range
    sizes = ragged_sizes(2, 64 * ws)
    a0, a1 = shard_range(len(sizes), ws, rank)
    sizes = sizes[a0:a1]
    fields = instance_fields(1000, 64 * ws)[a0:a1]
    window = 0.05 if args.window is None else args.window
    win = window * 1e-9
    nt = int(round(window / 1e-3)) + 1
    t = np.linspace(0, win, nt)
    solvers, m0s = [], []
    for (res, L), h in zip(sizes, fields):
        s = Solver(res, L)
        s.assemble()
        s.set_dynamics(solver=2, gamma=GAMMA, alpha=GAMMA * 0.02, hext=np.array([[0.0, *h], [win, *h]]))
        solvers.append(s)
        m0s.append(torch.as_tensor(start_state(int(np.prod(res))), device="cuda"))
    out = {}

    def step():
        _, _, _, st = integrate_ragged(solvers, t, m0s, tol=1e-6, graph=True)
        out["st"] = st
        return st

    times, stats, clocks, flush = timed_steps(torch, step, args.steps, args.warmup, dist, local)
    # end to end: host states in, host trajectories out
    m0_host = [m.cpu() for m in m0s]
    e2e = []
    for _ in range(max(1, args.steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dev = [m.to("cuda") for m in m0_host]
        _, ys, _, _ = integrate_ragged(solvers, t, dev, tol=1e-6, graph=True)
        host = [y.cpu() for y in ys]
        torch.cuda.synchronize()
        e2e.append((time.perf_counter() - t0) * 1e3)
        del ys, host
    # the same instances one after another through the single-instance path
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s, m in zip(solvers, m0s):
        s.integrate(t, m, tol=1e-6)
    torch.cuda.synchronize()
    seq_s = time.perf_counter() - t0
    step_ms, e2e_ms = max_over_ranks(torch, dist, [sum(times) / len(times), statistics.median(e2e)])
    if rank != 0:
        return None
    K = len(solvers)
    st = stats[-1]
    evals = [x["f_evals"] for x in st]
    bytes_ = sum(24.0 * s.n * s.n * e for s, e in zip(solvers, evals))
    kms = st[0]["kernel_ms"]
    achieved = bytes_ / (kms / 1e3) / 1e9
    sim_ns = ws * K * window
    ns = [s.n for s in solvers]
    return {
        "metric": "simulated ns/s", "value": sim_ns / (step_ms / 1e3), "unit": "simulated ns/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"ragged: {K} films/rank, nx ~ U{{20..120}}, ny = nx/4, 6.25x6.25x3 nm cells "
                               f"(n {min(ns)}..{max(ns)}, {sum(24 * x * x for x in ns) / 1e9:.2f} GB of FP32 "
                               f"tensors), seeded in-plane fields, {window} ns each at alpha_G = 0.02, tol 1e-6, "
                               "output every 1 ps; one cooperative launch on per-instance SM groups, replayed from "
                               "a CUDA graph",
                   "instances_per_rank": K, "window_ns": window, "parallelism": f"instances sharded over {ws} rank(s)",
                   "l2": "flushed (256 MB write) before every timed step"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None,
                     "note": f"integrate_ragged_kernel: sum over instances of 24*n_k^2 tensor bytes x evaluations "
                             f"({sum(evals)} evaluations) over {kms:.1f} ms of device time; peak {src} HBM copy"},
        "sequential_single_instance": {"value": ws * K * window / seq_s, "unit": "simulated ns/s",
                                       "note": "the same instances one after another through mt_integrate"},
        "e2e": {"value": sim_ns / (e2e_ms / 1e3), "unit": "simulated ns/s",
                "h2d_bytes_per_step": sum(3 * x * 8 for x in ns), "d2h_bytes_per_step": sum(nt * 3 * x * 8 for x in ns)},
        "rhs_evals_per_instance": {"min": int(min(evals)), "median": float(np.median(evals)), "max": int(max(evals))},
        "gpu_launches": int(st[0]["launches"]),
        "clocks": clocks,
    }


def bench_plain(torch, args, ws, rank, local, dist, hbm, src):
    from magtense_b200 import Solver, integrate_shards_local, link_shards_local
    from magtense_b200.shard import gather_rows, link_row_shard
    large = args.workload == "large-plain"
    W = args.shards
    mode = None if W <= 1 else ("ranks" if ws > 1 else "local")
    if mode and not large:
        raise SystemExit("--shards applies to large-plain")
    if mode == "ranks" and W != ws:
        raise SystemExit("--shards must equal --gpus for row shards over ranks")
    res, L = (LARGE_RES, LARGE_L) if large else (FILM_RES, FILM_L)
    if large and args.res:
        res = tuple(args.res)
        L = tuple(5e-9 * v for v in res)
    n = int(np.prod(res))
    window = (0.002 if large else 0.05) if args.window is None else args.window
    win = window * 1e-9
    nt = max(2, int(round(window / 1e-3)) + 1)
    t = np.linspace(0, win, nt)
    if large:
        rng = np.random.default_rng(1)
        axis = rng.standard_normal(3)
        axis /= np.linalg.norm(axis)
        m = rng.standard_normal((3, n))
        m_s = torch.as_tensor((m / np.linalg.norm(m, axis=0)).reshape(-1), device="cuda")
        h = np.array([10e-3 / MU0, 0.0, 0.0])

        def make(shard=None):
            sv = Solver(res, L, K0=5e3, u_ea=np.tile(axis, (n, 1)), shard=shard)
            sv.assemble()
            sv.set_dynamics(solver=2, gamma=GAMMA, alpha=GAMMA * 0.1, hext=np.array([[0.0, *h], [win, *h]]))
            return sv

        if mode == "local":
            shards = [make((r, W)) for r in range(W)]
            link_shards_local(shards)
        else:
            s = make((rank, ws) if mode == "ranks" else None)
            if mode == "ranks":
                link_row_shard(s)
    else:
        s, m_s = relaxed_state(torch, res, L)
        h = instance_fields(1000, ws)[rank]
        s.set_dynamics(solver=2, gamma=GAMMA, alpha=GAMMA * 0.02, hext=np.array([[0.0, *h], [win, *h]]))

    def run(m0):
        if mode == "local":
            return integrate_shards_local(shards, t, m0, tol=1e-6)
        return s.integrate(t, m0, tol=1e-6)

    def step():
        return [run(m_s)[3]]

    times, stats, clocks, flush = timed_steps(torch, step, args.steps, args.warmup, dist, local)
    m_host = m_s.cpu().numpy()
    e2e = []
    for _ in range(max(1, args.steps)):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        m0 = torch.from_numpy(m_host).pin_memory().to("cuda", non_blocking=True)
        _, y, _, _ = run(m0)
        if mode == "ranks":
            y = gather_rows(y, n)
        y.cpu()
        torch.cuda.synchronize()
        e2e.append((time.perf_counter() - t0) * 1e3)
    step_ms, e2e_ms = max_over_ranks(torch, dist, [sum(times) / len(times), statistics.median(e2e)])
    if rank != 0:
        return None
    flat = [x for st in stats for x in st]
    evals = sum(x["f_evals"] for x in flat)
    kms = sum(x["kernel_ms"] for x in flat)
    launches = sum(x["launches"] for x in flat)
    # tensor bytes one GPU streams per evaluation: its rows only when the ranks share the instance
    rows = -(-n // ws) if mode == "ranks" else n
    achieved = 24.0 * n * rows * evals / (kms / 1e3) / 1e9
    sim_ns = window if mode == "ranks" else ws * window
    if mode == "local":
        par = f"one instance as {W} row shards on one GPU (CTA groups of one launch, peer stores into local memory)"
    elif mode == "ranks":
        par = f"one instance as {ws} row shards, one per GPU (CUDA IPC exchange regions)"
    else:
        par = f"one instance per rank, {ws} rank(s)"
    kern = "integrate_ragged_kernel (shard groups)" if mode == "local" else "integrate_kernel"
    return {
        "metric": "simulated ns/s", "value": sim_ns / (step_ms / 1e3), "unit": "simulated ns/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True,
        "scaling": "strong" if mode == "ranks" else "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": (f"large-plain: {res[0]}x{res[1]}x{res[2]} cubes of 5 nm (n={n}, "
                                f"{24 * n * n / 1e9:.2f} GB FP32 tensor), K=5e3 J/m^3 "
                                "along a seeded axis, 10 mT field, alpha_G=0.1" if large else
                                "film-plain: 80x20x1 std-problem-4 film (n=1600), single instance") +
                               ", plain FP32 demag, persistent single-instance integrator, tol 1e-6",
                   "window_ns": window, "outputs": nt, "parallelism": par,
                   "l2": "flushed (256 MB write) before every timed step"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     # DRAM bytes per launch: an ncu capture of a 32x32x4 case read 1.0004 x the tensor bytes of
                     # its evaluations (writes 0.15 %); scaled here by this run's evaluations per launch
                     "traffic": (TRAFFIC_PER_TENSOR_BYTE * 24.0 * n * rows * evals / max(1, launches)) if large else None,
                     "note": f"{kern}: 24*n*{rows} tensor bytes per RHS evaluation per GPU x {evals} evaluations "
                             f"over {kms:.2f} ms of device time; peak {src} HBM copy"
                             + ("; traffic in bytes per launch, scaled from the 32x32x4 ncu capture" if large else "")},
        "e2e": {"value": sim_ns / (e2e_ms / 1e3), "unit": "simulated ns/s", "h2d_bytes_per_step": 3 * n * 8,
                "d2h_bytes_per_step": nt * 3 * n * 8},
        "gpu_launches": int(launches),
        "rhs_evals_per_s": evals / (sum(times) / 1e3) * ws,
        "evals_per_ns": evals / (len(stats) * window),
        "step_ms_each": [round(x, 3) for x in times],
        "kernel_ms_each": [round(sum(x["kernel_ms"] for x in st), 3) for st in stats],
        "clocks": clocks,
    }


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
