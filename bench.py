"""Benchmark of the HIF hot path on B200: factor + FP64-residual PCG solve.

One step = assemble the face-coefficient operator from HBM-resident coefficient
arrays, hif_factor (every level: assembly, eliminations, IDs) and one PCG solve
to relative residual 1e-10 with the factor's inverse apply as preconditioner,
at n = 128 (N = 127, 2,048,383 DOFs), a = exp(GRF) at faces (correlation length
1/16 of the unit cube, sigma 1, seed 2), eps = 1e-6, FP64 and mixed precision. The metric's unit is whole-job
(factor + solve) steps per second; factor seconds, solves per second and PCG
iterations are reported alongside.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--n 128]

Multi-GPU: replicas (each rank factors and solves its own operator; the path has
no exchange step), timing is the max over ranks.

--impl reference times the reference's own CPU build (oracle/_ref, built from
arbenson/HIFDE3D's sources) on this host's cores over a bounded sample.
"""
from __future__ import annotations

import argparse
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

METRIC = ("factor s + solves/sec at N=128^3, resid<=1e-10: mixed vs FP64 GPU; "
          "serving p50/p99 ms")
REF_PROBE = os.path.join(ROOT, "oracle", "_ref", "hif_ref_probe")


def dofs(n: int) -> int:
    return (n - 1) ** 3


# Correlation length of the coefficient field on the unit cube, and the value the
# generator takes for it: synth maps the cube onto its periodic box of length 2.
GRF_CORRELATION = 1.0 / 16
GRF_ELL_PARAM = 2 * GRF_CORRELATION


# ---------------------------------------------------------------------------
# replicas (N > 1): every rank factors and solves its own operator
# ---------------------------------------------------------------------------
def replica_seeds(rank: int):
    """(coefficient-field seed, right-hand-side seed) of a rank's operator: the
    replicas factor different operators of the same size."""
    return 2 + rank, rank


def replica_times(ms_step: float, e2e_s: float, world: int, device=None):
    """Max over ranks of the device time per step and of the end-to-end step
    time: the job's step ends when its slowest replica's does. Every rank calls
    this once, with the same collective on every path."""
    if world <= 1:
        return ms_step, e2e_s
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms_step, e2e_s], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t[0]), float(t[1])


def workload_config(n: int, eps: float, world: int) -> dict:
    """The `config` object of both arms' JSON lines: the workload they measure."""
    return {"workload": f"hif factor + pcg(1e-10), n={n} (N={n - 1}, {dofs(n)} DOFs), "
                        f"face a=exp(GRF sigma=1, correlation length 1/16 of the unit cube), "
                        f"eps={eps}, P=4",
            "parallelism": f"replicas x{world}"}


def job_value(world: int, ms_step: float) -> float:
    """Whole-job steps per second: `world` replicas each finish one step per
    (max over ranks) `ms_step` milliseconds."""
    return world * 1e3 / ms_step


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.samples = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# reference CPU build on this host
# ---------------------------------------------------------------------------
def reference_sample(n_sample: int, threads: int, workdir: str, eps: float = 1e-6):
    """The reference's own Factor() + one Apply(u, true) at n_sample on the bench's
    operator: the face-coefficient form with a = exp(GRF) (the same field as the
    GPU arm at that size), entered into the reference's sparse matrix by the probe
    (oracle/ref_probe.cpp, mode timef). Returns (factor + apply seconds, wall
    seconds, the probe's record with per-level times)."""
    from hifde3d_b200 import synth
    N = n_sample - 1
    ax, ay, az = synth.face_coefficients_grf(N, 2, GRF_ELL_PARAM, 1.0)
    V = np.zeros((n_sample + 1,) * 3)
    names = []
    for nm, a in (("ax", ax), ("ay", ay), ("az", az), ("V", V)):
        path = os.path.join(workdir, nm + ".bin")
        a.ravel(order="F").astype("<f8").tofile(path)
        names.append(path)
    env = dict(os.environ, OPENBLAS_NUM_THREADS=str(threads), OMP_NUM_THREADS=str(threads))
    t0 = time.perf_counter()
    out = subprocess.run([REF_PROBE, "timef", str(N), "4", repr(eps), "-1", *names], env=env,
                         capture_output=True, text=True, check=True).stdout
    wall = time.perf_counter() - t0
    rec = json.loads(out.strip().splitlines()[-1])
    return rec["factor_s"] + max(rec["apply_inv_s"], 0.0), wall, rec


# The reference's factorization cost grows far faster than its DOF count (its
# sparse update is quadratic: 13 s at n = 32, about 11 min at n = 64 on one core),
# so it is timed at n = 32, a size it finishes in seconds; longer runs recorded
# beside it are read from this file (written by the measurements it names).
REF_RECORD = os.path.join(ROOT, "profiles", "reference_cpu_times.json")
REF_N = 32
REF_ARM_BUDGET_S = 150.0


def reference_record() -> dict | None:
    if not os.path.exists(REF_RECORD):
        return None
    with open(REF_RECORD) as fh:
        return json.load(fh)


def run_reference_arm(args, rank: int, world: int):
    """The reference's CPU build on this host's cores, at n = 32 on the bench's
    operator: its config names n = 32 and the steps it actually ran (as many of
    the requested ones as fit in about REF_ARM_BUDGET_S seconds)."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if not os.path.exists(REF_PROBE):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/hif_ref_probe not built (make -C oracle)"}))
        return
    n_ref = args.ref_n
    times, per_level = [], None
    with tempfile.TemporaryDirectory() as td:
        # one untimed run (page cache, library load), then timed runs
        s0, _, _ = reference_sample(n_ref, threads, td, args.eps)
        steps_run = max(1, min(args.steps, int(REF_ARM_BUDGET_S / max(s0, 1e-3))))
        for _ in range(steps_run):
            s, _, rec = reference_sample(n_ref, threads, td, args.eps)
            times.append(s)
            per_level = rec["per_level"]
    t = float(np.mean(times))
    value = 1.0 / t
    unit = f"factor+solve steps/s at n={n_ref}"
    sample = (f"reference Factor() + Apply(u, true) at n={n_ref} ({dofs(n_ref)} DOFs) on the "
              f"face operator a=exp(GRF) (the GPU arm's field at that size), eps={args.eps}, "
              f"OpenBLAS {threads} threads; {steps_run} timed runs after one untimed run; "
              "measured, not scaled")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": unit,
        "n_gpus": world, "steps": steps_run, "warmup": 1, "requested_steps": args.steps,
        "requested_warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {**workload_config(n_ref, args.eps, world),
                   "arithmetic": "FP64 (the reference's CPU build from its own sources)",
                   "note": (f"the GPU arm's headline is n={args.n}; the reference runs n={n_ref} "
                            "here (hours at n=128); the GPU arm's line carries its own rate at "
                            f"n={n_ref} under same_size for a like-for-like ratio")},
        "per_level_s": per_level,
        "cpu_baseline": {"value": value, "unit": unit, "cores": threads, "kind": "reference",
                         "sample": sample, "measured_sample_s": t},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def fp64_gemm_peak(torch, dev):
    """cuBLAS DGEMM 8192^3 burst rate in TFLOP/s (the FP64 roofline denominator)."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2 * 8192 ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    return best


# ---------------------------------------------------------------------------
# serving: operators of n in {32, 48, 64, 96} resident on the GPU, Poisson arrivals
# ---------------------------------------------------------------------------
SERVE_SIZES = (32, 48, 64, 96)


def serving_schedule(nreq: int, rate: float, seed: int = 5):
    """Seeded arrivals: (time s, kind, size index or op slot, nrhs, rhs seed).
    70 % solves of 1-32 right-hand sides against resident operators, 30 % new
    factorizations of a random pool size."""
    from hifde3d_b200 import synth
    u = synth.uniform(seed, 5 * nreq).reshape(nreq, 5)
    t = np.cumsum(-np.log(1.0 - u[:, 0]) / rate)
    out = []
    for q in range(nreq):
        kind = "factor" if u[q, 1] < 0.3 else "solve"
        out.append((float(t[q]), kind, int(u[q, 2] * 1e6), 1 + int(u[q, 3] * 32), 1000 + q))
    return out


def run_serving(hb, synth, prec: int, nreq: int, rate: float, budget_gb: float = 120.0,
                max_resident: int = 12, burst: int = 96):
    """One pass of the serving workload at one precision; latencies from the
    server's own submit / admission / completion clock. Solves submitted while
    their operator was still being factored are reported as their own class
    (their queue time includes that factorization). Then `burst` solve requests
    submitted at once against the warm pool measure capacity at saturation."""
    srv = hb.Server(budget_bytes=int(budget_gb * (1 << 30)), max_active_solves=64,
                    factor_workers=2)
    sched = serving_schedule(nreq, rate)
    next_op = [0]
    resident = []  # (op id, n) usable as solve targets, oldest first
    releases = []
    fids, sids = [], []

    def new_op(n):
        op = next_op[0]
        next_op[0] += 1
        N = n - 1
        ax, ay, az = synth.face_coefficients_lognormal(N, 100 + op, 1.0)
        V = np.zeros((n + 1,) * 3)
        # the clipped partition: NC = 48 and 96 are not P * 2^l, where the
        # reference partition leaves the top level without cells
        return op, srv.submit_factor(op, N, ax, ay, az, V, eps=1e-6, precision=prec,
                                     partition=hb.PARTITION_CLIPPED)

    # warm pool: one operator of each size, ready before the clock starts
    warm = []
    for n in SERVE_SIZES:
        op, rid = new_op(n)
        r = srv.wait(rid)
        if r["status"] != hb.HIF_OK:
            raise RuntimeError(f"serving warm pool: {r}")
        resident.append((op, n))
        warm.append((op, n))
    rhs_cache = {}

    def rhs(n, nrhs, seed):
        key = (n, nrhs, seed % 8)
        if key not in rhs_cache:
            rhs_cache[key] = synth.dof_vector(n - 1, seed % 8, nrhs)
        return rhs_cache[key]

    t0 = time.perf_counter()
    for (ta, kind, pick, nrhs, seed) in sched:
        dt = ta - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        if kind == "factor":
            n = SERVE_SIZES[pick % len(SERVE_SIZES)]
            if len(resident) >= max_resident:
                old, _ = resident.pop(0)
                th = threading.Thread(target=srv.release, args=(old,))
                th.start()
                releases.append(th)
            op, rid = new_op(n)
            fids.append((rid, n, op, time.perf_counter()))
            resident.append((op, n))
        else:
            op, n = resident[pick % len(resident)]
            sids.append((srv.submit_solve(op, rhs(n, nrhs, seed), tol=1e-10, maxit=100), n,
                         nrhs, op, time.perf_counter()))
    fac_done = {}
    lat_f, q_f, s_f, fails, errors = [], [], [], 0, []
    for rid, n, op, ts in fids:
        r = srv.wait(rid)
        if r["status"] != hb.HIF_OK:
            fails += 1
            errors.append(f"factor n={n}: {r.get('error', r['status'])}")
            continue
        fac_done[op] = ts + 1e-3 * r["latency_ms"]
        lat_f.append(r["latency_ms"])
        q_f.append(r["queue_ms"])
        s_f.append(r["service_ms"])
    ready = {"lat": [], "queue": [], "service": []}
    waited = {"lat": [], "queue": [], "service": []}
    iters, worst, rhs_total = [], 0.0, 0
    for rid, n, nrhs, op, ts in sids:
        r = srv.wait(rid)
        if r["status"] != hb.HIF_OK:
            fails += 1
            errors.append(f"solve n={n}: {r.get('error', r['status'])}")
            continue
        cls = waited if fac_done.get(op, 0.0) > ts else ready
        cls["lat"].append(r["latency_ms"])
        cls["queue"].append(r["queue_ms"])
        cls["service"].append(r["service_ms"])
        iters.append(r["iters"])
        worst = max(worst, r["relres"])
        rhs_total += nrhs
    makespan = time.perf_counter() - t0
    for th in releases:
        th.join()
    st = srv.stats()
    # capacity: a burst of solves against the operators resident at the end
    cap = None
    live = [x for x in resident if x in warm or x[0] in fac_done]
    if burst > 0 and live:
        u = synth.uniform(7, 3 * burst).reshape(burst, 3)
        ids = []
        tb = time.perf_counter()
        nr_b = 0
        for q in range(burst):
            op, n = live[int(u[q, 0] * 1e6) % len(live)]
            nrhs = 1 + int(u[q, 1] * 32)
            nr_b += nrhs
            ids.append(srv.submit_solve(op, rhs(n, nrhs, q), tol=1e-10, maxit=100))
        ok = sum(1 for i in ids if srv.wait(i)["status"] == hb.HIF_OK)
        tspan = time.perf_counter() - tb
        cap = {"requests": burst, "completed": ok, "makespan_s": tspan,
               "solves_per_s": ok / tspan, "rhs_per_s": nr_b / tspan,
               "workload": f"{burst} solve requests of 1-32 right-hand sides (seed 7) "
                           "submitted at once against the resident operators"}
    srv.close()
    pct = lambda v, q: float(np.percentile(v, q)) if v else None  # noqa: E731

    def summ(c):
        return {"count": len(c["lat"]), "latency_p50_ms": pct(c["lat"], 50),
                "latency_p99_ms": pct(c["lat"], 99), "queue_p50_ms": pct(c["queue"], 50),
                "queue_p99_ms": pct(c["queue"], 99), "service_p50_ms": pct(c["service"], 50),
                "service_p99_ms": pct(c["service"], 99)}

    nsol = len(ready["lat"]) + len(waited["lat"])
    return {"requests": nreq, "solves": nsol, "factorizations": len(lat_f),
            "failed": fails, "makespan_s": makespan,
            "solves_per_s": nsol / makespan, "rhs_per_s": rhs_total / makespan,
            "solve_p50_ms": pct(ready["lat"], 50), "solve_p99_ms": pct(ready["lat"], 99),
            "solves_ready_operator": summ(ready),
            "solves_waiting_for_factorization": summ(waited),
            "factor_p50_ms": pct(lat_f, 50), "factor_p99_ms": pct(lat_f, 99),
            "factor_queue_p99_ms": pct(q_f, 99), "factor_service_p50_ms": pct(s_f, 50),
            "factor_service_p99_ms": pct(s_f, 99),
            "pcg_iters_max": max(iters) if iters else None, "relres_max": worst,
            "server_iterations": st["iterations"], "batched_launches": st["batched_launches"],
            "peak_resident_ops": max_resident, "capacity": cap, "errors": errors[:4]}


def run_multi_rhs(hb, synth, torch, dev, prec: int, n: int = 96, nrhs: int = 64):
    """High-contrast operator with many right-hand sides in one batched solve:
    a piecewise constant on 8^3 sub-cubes with values 10^U(-3, 3) (seed 1),
    V = 1e-2, eps = 1e-8, 64 right-hand sides N(0, 1) (seeds 0..63), PCG to
    1e-10 with every right-hand side in the same preconditioner applies."""
    N = n - 1
    ax, ay, az = synth.face_coefficients_blocks(N, 1)
    V = np.full((n + 1,) * 3, 1e-2)
    f = hb.HIFFactor(N, 4, 1e-8, hb.PARTITION_CLIPPED)
    f.set_option(hb.OPT_PRECISION, prec)
    stream = torch.cuda.Stream(device=dev)
    hb.set_stream(f, stream.cuda_stream)
    hb.SetupStencilFaces(f, N, 1.0 / n, ax, ay, az, V)
    b = np.asfortranarray(np.stack([synth.dof_vector(N, s) for s in range(nrhs)], axis=1))
    db = torch.from_numpy(np.ascontiguousarray(b.T)).to(dev)  # column c contiguous
    dx = torch.zeros_like(db)
    for _ in range(2):  # warm: the handle's device arenas reach their size
        f.Factor()
        f.solve_pcg_device(db.data_ptr(), dx.data_ptr(), nrhs, n ** 3, 1e-10, 200)
    torch.cuda.synchronize()
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record(stream)
    f.Factor()
    e1.record(stream)
    it, rr = f.solve_pcg_device(db.data_ptr(), dx.data_ptr(), nrhs, n ** 3, 1e-10, 200)
    e2.record(stream)
    e2.synchronize()
    f.close()
    return {"factor_s": e0.elapsed_time(e1) / 1e3, "solve_s": e1.elapsed_time(e2) / 1e3,
            "rhs": nrhs, "pcg_iters_max": int(np.max(it)), "relres_max": float(np.max(rr))}


def time_steps(hb, synth, torch, dev, n: int, eps: float, prec: int, steps: int = 3,
               warmup: int = 2) -> dict:
    """Factor + PCG(1e-10) steps of the bench operator at size n (CUDA events on
    the handle's stream), for the same-size comparison with the reference."""
    N = n - 1
    ax, ay, az = synth.face_coefficients_grf(N, 2, GRF_ELL_PARAM, 1.0)
    V = np.zeros((n + 1,) * 3)
    dco = [torch.from_numpy(np.ascontiguousarray(x.ravel(order="F"))).to(dev)
           for x in (ax, ay, az, V)]
    db = torch.from_numpy(synth.dof_vector(N, 0)).to(dev)
    dx = torch.zeros_like(db)
    g = hb.HIFFactor(N, 4, eps)
    g.set_option(hb.OPT_PRECISION, prec)
    st = torch.cuda.Stream(device=dev)
    hb.set_stream(g, st.cuda_stream)

    def one():
        hb.SetupStencilFacesDevice(g, N, 1.0 / n, *[t.data_ptr() for t in dco])
        g.Factor()
        return g.solve_pcg_device(db.data_ptr(), dx.data_ptr(), 1, n ** 3, 1e-10, 100)

    for _ in range(warmup):
        one()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        it, rr = one()
    e1.record(st)
    e1.synchronize()
    g.close()
    ms = e0.elapsed_time(e1) / steps
    return {"steps_per_s": 1e3 / ms, "ms_per_step": ms, "pcg_iters": int(it[0]),
            "pcg_relres": float(rr[0])}


def per_level_error(hb, f, N: int, h: float, coef, b: np.ndarray) -> dict:
    """Mixed against FP64 on the same operator, per level: with x = F^{-1} b from
    each factor, the relative difference of x over the DOFs each level eliminates
    (as the FP64 factor assigns them), and over all DOFs."""
    out = {}
    xs = {}
    for name, prec in (("fp64", hb.PRECISION_FP64), ("mixed", hb.PRECISION_MIXED)):
        f.set_option(hb.OPT_PRECISION, prec)
        hb.SetupStencilFacesDevice(f, N, h, *[t.data_ptr() for t in coef])
        f.Factor()
        y = b.copy()
        f.Apply(y, True)
        xs[name] = y
        if name == "fp64":
            phase = f.dof_levels()
    e = xs["mixed"] - xs["fp64"]
    ref = xs["fp64"]
    levels = {}
    for lev in range(int(phase.max()) // 2 + 1):
        m = (phase == 2 * lev) | (phase == 2 * lev + 1)
        if m.any():
            levels[str(lev)] = float(np.linalg.norm(e[m]) / max(np.linalg.norm(ref[m]), 1e-300))
    out["per_level"] = levels
    out["all_dofs"] = float(np.linalg.norm(e) / np.linalg.norm(ref))
    out["definition"] = ("relative difference ||x_mixed - x_fp64|| / ||x_fp64|| of x = F^-1 b "
                         "over the DOFs eliminated at each level (FP64 factor's assignment); "
                         "the FP64 GPU factor is pinned to the reference at n=64 "
                         "(tests/test_gpu_parity_bench.py)")
    return out


def run_ours(args, rank: int, world: int):
    import torch
    import torch.distributed as dist

    import hifde3d_b200 as hb
    from hifde3d_b200 import synth

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n
    N, NC = n - 1, n
    eps = args.eps

    # synthetic operator (per-rank seed for replicas) and right-hand side
    seed_op, seed_rhs = replica_seeds(rank)
    ax, ay, az = synth.face_coefficients_grf(N, seed_op, GRF_ELL_PARAM, 1.0)
    V = np.zeros((NC + 1,) * 3)
    b = synth.dof_vector(N, seed_rhs)
    host = [np.ascontiguousarray(x.ravel(order="F")) for x in (ax, ay, az, V)]
    dcoef = [torch.from_numpy(x).to(dev) for x in host]
    db = torch.from_numpy(b).to(dev)
    dx = torch.zeros_like(db)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MB > L2

    peak_fp64 = fp64_gemm_peak(torch, dev) if rank == 0 else None

    f = hb.HIFFactor(N, 4, eps)
    # tile shapes of the batched FP64 products are tuned during the warm-up
    # factorizations (two suffice for every batch signature to decide)
    f.set_option(hb.OPT_AUTOTUNE, 0 if args.no_autotune else 1)
    stream = torch.cuda.Stream(device=dev)
    hb.set_stream(f, stream.cuda_stream)
    h = 1.0 / NC

    def step():
        hb.SetupStencilFacesDevice(f, N, h, *[t.data_ptr() for t in dcoef])
        f.Factor()
        it, rr = f.solve_pcg_device(db.data_ptr(), dx.data_ptr(), 1, NC ** 3, 1e-10, 100)
        return int(it[0]), float(rr[0])

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def measure(prec):
        """W warm-up steps, one profiled step (kernel statistics, untimed), then
        K timed steps (CUDA events on the engine stream), then solve-only
        timings with the resident factor."""
        f.set_option(hb.OPT_PRECISION, prec)
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        # kernel statistics from one profiled, untimed step (per-launch events
        # stay out of the timed steps)
        f.set_option(hb.OPT_PROFILE, 1)
        with torch.cuda.stream(stream):
            flush.zero_()
        step()
        kst = f.kernel_stats()
        f.set_option(hb.OPT_PROFILE, 0)
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        barrier()
        clocks.start()
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        iters, rel, fac = [], [], []
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            it, rr = step()
            iters.append(it)
            rel.append(rr)
            fac.append(f.factor_stats()["total_s"])
        t_end.record(stream)
        t_end.synchronize()
        barrier()
        clk = clocks.stop()
        ms_total = t_start.elapsed_time(t_end)
        solve_ms = []
        for _ in range(max(3, args.steps)):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            f.solve_pcg_device(db.data_ptr(), dx.data_ptr(), 1, NC ** 3, 1e-10, 100)
            e1.record(stream)
            e1.synchronize()
            solve_ms.append(e0.elapsed_time(e1))
        return {"ms_step": ms_total / args.steps, "factor_s": float(np.mean(fac)),
                "solve_ms": float(np.median(solve_ms)), "pcg_iters": iters[-1],
                "pcg_relres": rel[-1], "clocks": clk, "kst": kst}

    runs = {}
    fp64_chol = None
    precs = {"fp64": [hb.PRECISION_FP64], "mixed": [hb.PRECISION_MIXED],
             "both": [hb.PRECISION_FP64, hb.PRECISION_MIXED]}[args.precision]
    for prec in precs:
        runs[prec] = measure(prec)
        if prec == hb.PRECISION_FP64 and not args.no_fp64_cholesky:
            # FP64 with the Cholesky elimination of the symmetric interiors (the
            # FP64 default keeps the reference's Gauss-Jordan inverse)
            f.set_option(hb.OPT_ELIMINATION, hb.ELIM_CHOLESKY)
            fp64_chol = measure(prec)
            f.set_option(hb.OPT_ELIMINATION, hb.ELIM_AUTO)
    head_prec = precs[-1]
    head = runs[head_prec]
    ms_total = head["ms_step"] * args.steps
    kst = head["kst"]
    clk = head["clocks"]
    iters, rel, fac = [head["pcg_iters"]], [head["pcg_relres"]], [head["factor_s"]]
    solve_ms = [head["solve_ms"]]

    # end to end through the public API with host buffers
    e2e_s, it_e2e, rr_e2e = float("nan"), None, None
    if not args.no_e2e:
        # host buffers in the reference's layout (NumTns: i fastest), which the
        # API takes without a host-side transpose
        hx = [np.asfortranarray(x) for x in (ax, ay, az, V)]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            hb.SetupStencilFaces(f, N, h, *hx)
            f.Factor()
            _xh, it_e2e, rr_e2e = f.solve_pcg(b, 1e-10, 100)
        torch.cuda.synchronize()
        e2e_s = (time.perf_counter() - t0) / args.steps
    h2d = 4 * (NC + 1) ** 3 * 8 + NC ** 3 * 8
    d2h = NC ** 3 * 8

    # max over ranks
    ms_step = ms_total / args.steps
    ms_step, e2e_s = replica_times(ms_step, e2e_s, world, dev)
    if rank != 0:
        f.close()
        return

    # roofline of the dominant kernel class
    dom = max(kst, key=lambda k: kst[k]["ms"])
    k = kst[dom]
    per_launch_ms = k["ms"] / max(k["launches"], 1)
    traffic = None
    tf_path = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(tf_path):
        with open(tf_path) as fh:
            traffic = json.load(fh).get(dom)
    peaks = {}
    pk_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk_path):
        with open(pk_path) as fh:
            peaks = json.load(fh)
    if k["flops"] > 0 and dom == "gemm_mixed":
        achieved = k["flops"] / max(k["launches"], 1) / (per_launch_ms * 1e-3) / 1e12
        tf32 = peaks.get("bf16_tflops", 1590.0) / 2
        roof = {"bound": "tensor", "kernel_class": dom, "achieved": achieved, "peak": tf32,
                "unit": "TFLOP/s", "frac": achieved / tf32, "traffic": traffic,
                "launches": k["launches"], "avg_launch_ms": per_launch_ms,
                "peak_source": "TF32 dense rate taken as half of MEASURED_PEAKS.json bf16_tflops; "
                               "achieved counts each FP64-equivalent product once (split-TF32 "
                               "issues three tensor products per product)"}
    elif k["flops"] > 0 and dom == "gemm_int8":
        achieved = k["flops"] / max(k["launches"], 1) / (per_launch_ms * 1e-3) / 1e12
        i8 = 2 * peaks.get("bf16_tflops", 1590.0)
        roof = {"bound": "tensor", "kernel_class": dom, "achieved": achieved, "peak": i8,
                "unit": "TOP/s (int8)", "frac": achieved / i8, "traffic": traffic,
                "launches": k["launches"], "avg_launch_ms": per_launch_ms,
                "peak_source": "int8 dense rate taken as twice MEASURED_PEAKS.json bf16_tflops; "
                               "achieved counts the int8 operations of the slice products over "
                               "the class's time, operand slicing launches included"}
    elif k["flops"] > 0:
        achieved = k["flops"] / max(k["launches"], 1) / (per_launch_ms * 1e-3) / 1e12
        roof = {"bound": "fp64", "kernel_class": dom, "achieved": achieved, "peak": peak_fp64,
                "unit": "TFLOP/s", "frac": achieved / peak_fp64 if peak_fp64 else None,
                "traffic": traffic, "launches": k["launches"],
                "avg_launch_ms": per_launch_ms,
                "peak_source": "cuBLAS DGEMM 8192^3 burst measured in this run (FP64 has no "
                               "entry in MEASURED_PEAKS.json)"}
    else:
        hbm = peaks.get("hbm_gbs", 6650.0)
        achieved = k["bytes"] / max(k["launches"], 1) / (per_launch_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel_class": dom, "achieved": achieved, "peak": hbm,
                "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                "launches": k["launches"], "avg_launch_ms": per_launch_ms,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback"}
    share = {kk: round(v["ms"] / max(sum(x["ms"] for x in kst.values()), 1e-9), 4)
             for kk, v in kst.items() if v["launches"]}

    # Same-size comparison with the reference: the GPU's own step rate at the
    # sizes the reference was timed at (n = 32 live below; n = 64 and the capped
    # n = 128 run from the recorded measurements).
    same = {}
    if not args.no_same_size:
        for ns in (32, 64):
            same[f"n{ns}"] = {nm: time_steps(hb, synth, torch, dev, ns, eps, pr)
                              for nm, pr in (("fp64", hb.PRECISION_FP64),
                                             ("mixed", hb.PRECISION_MIXED))}
    cpu = None
    if world == 1 and not args.no_cpu_baseline and os.path.exists(REF_PROBE):
        with tempfile.TemporaryDirectory() as td:
            s, _, rec = reference_sample(REF_N, 1, td, eps)
        unit32 = f"factor+solve steps/s at n={REF_N}"
        cpu = {"value": 1.0 / s, "unit": unit32, "cores": 1, "kind": "reference",
               "sample": (f"reference Factor() + Apply(u, true) at n={REF_N} ({dofs(REF_N)} "
                          f"DOFs) on the face operator a=exp(GRF), 1 core: {s:.2f} s measured "
                          "(not scaled); compare with same_size.n32"),
               "per_level_s": rec["per_level"]}
        if "n32" in same:
            same["n32"]["reference_1core"] = {"steps_per_s": 1.0 / s, "ms_per_step": 1e3 * s}
            for nm in ("fp64", "mixed"):
                same["n32"][f"{nm}_vs_reference"] = same["n32"][nm]["steps_per_s"] * s
    rec_ref = reference_record()
    if rec_ref and "n64" in same:
        r64 = rec_ref.get("n64")
        if r64 and r64.get("factor_s"):
            t64 = r64["factor_s"] + max(r64.get("apply_inv_s", 0.0), 0.0)
            same["n64"]["reference_1core_recorded"] = {
                "steps_per_s": 1.0 / t64, "ms_per_step": 1e3 * t64,
                "host": rec_ref.get("host"), "source": os.path.relpath(REF_RECORD, ROOT)}
            for nm in ("fp64", "mixed"):
                same["n64"][f"{nm}_vs_reference"] = same["n64"][nm]["steps_per_s"] * t64
    # n = 128 (this workload): the reference's capped run, levels reached so far;
    # their elapsed time is a lower bound on its factor time
    r128 = rec_ref.get("n128") if rec_ref else None
    if r128 and r128.get("per_level") and n == 128:
        t128 = float(r128["per_level"][-1]["elapsed_s"])
        same["n128"] = {
            "reference_1core_lower_bound_s": t128,
            "levels_completed": len(r128["per_level"]),
            "status": r128.get("status"),
            "source": os.path.relpath(REF_RECORD, ROOT)}
        for nm, prec in (("fp64", hb.PRECISION_FP64), ("mixed", hb.PRECISION_MIXED)):
            if prec in runs:
                same["n128"][f"{nm}_vs_reference_at_least"] = t128 / (runs[prec]["ms_step"] * 1e-3)

    value = job_value(world, ms_step)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": f"factor+solve steps/s at n={n}",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if head_prec == hb.PRECISION_FP64 else "f64+int8-slices",
        "data": "synthetic",
        "config": {**workload_config(n, eps, world),
                   "arithmetic": ("FP64" if head_prec == hb.PRECISION_FP64 else
                                  "mixed: the long-K products of every elimination (S, and "
                                  "Y = L^-1 A21 or X = A22^-1 A21) from int8 slices per value "
                                  "(5 for S, 6 for Y, 7 for X) on the tcgen05 tensor cores "
                                  "(exact int32 sums); FP64 diagonal-block factorization "
                                  "(Cholesky or Gauss-Jordan, chosen per phase by the tuner), "
                                  "ID pivots and rank, factor storage and PCG residual"),
                   "l2_flush": "256 MB write per step",
                   "inputs": "coefficients and rhs resident in HBM"},
        "factor_s": float(np.mean(fac)),
        "solve_ms": float(np.median(solve_ms)),
        "solves_per_s": 1e3 / float(np.median(solve_ms)),
        "pcg_iters": iters[-1],
        "pcg_relres": rel[-1],
        "clocks": clk,
        "e2e": {"value": world / e2e_s if e2e_s == e2e_s else None,
                "unit": f"factor+solve steps/s at n={n}",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "pcg_iters": it_e2e, "pcg_relres": rr_e2e},
        "roofline": roof,
        "kernel_share": share,
        # our kernels launched in the timed region: per-step count (from the
        # profiled step) times the timed steps
        "gpu_launches": int(sum(v["launches"] for v in kst.values())) * args.steps,
        "cpu_baseline": cpu,
        "same_size": same or None,
        "reference_recorded": rec_ref,
        "autotune": None if args.no_autotune else f.autotune_stats(),
    }
    for name, prec in (("fp64", hb.PRECISION_FP64), ("mixed", hb.PRECISION_MIXED)):
        if prec in runs:
            r = runs[prec]
            line[name] = {"steps_per_s": 1e3 / r["ms_step"], "ms_per_step": r["ms_step"],
                          "factor_s": r["factor_s"], "solve_ms": r["solve_ms"],
                          "solves_per_s": 1e3 / r["solve_ms"], "pcg_iters": r["pcg_iters"],
                          "pcg_relres": r["pcg_relres"]}
    if fp64_chol is not None:
        r = fp64_chol
        line["fp64_cholesky"] = {
            "steps_per_s": 1e3 / r["ms_step"], "ms_per_step": r["ms_step"],
            "factor_s": r["factor_s"], "solve_ms": r["solve_ms"], "pcg_iters": r["pcg_iters"],
            "pcg_relres": r["pcg_relres"],
            "arithmetic": ("FP64 throughout, Cholesky elimination of the symmetric interiors "
                           "(HIF_OPT_ELIMINATION = HIF_ELIM_CHOLESKY); pinned to the reference's "
                           "F^-1 u at n = 64 by tests/test_gpu_cholesky.py")}
    if len(runs) == 2 and not args.no_level_error:
        # mixed against FP64 per level on the headline operator (the FP64 factor is
        # pinned to the reference's at n = 64 by the parity tests)
        line["mixed"]["error_vs_fp64"] = per_level_error(hb, f, N, h, dcoef, b)
    if not (args.no_multi_rhs and args.no_serving):
        # the n = 128 operator and its pool memory leave the device first
        f.close()
        torch.cuda.synchronize()
        hb.trim_device_pool()
    if not args.no_multi_rhs:
        mr = {}
        for name, prec in (("fp64", hb.PRECISION_FP64), ("mixed", hb.PRECISION_MIXED)):
            if prec in runs:
                mr[name] = run_multi_rhs(hb, synth, torch, dev, prec)
        line["multi_rhs"] = {
            "workload": "n=96 (clipped partition), a piecewise constant on 8^3 sub-cubes, "
                        "10^U(-3,3) seed 1, V=1e-2, eps=1e-8, 64 RHS N(0,1) seeds 0..63 in one "
                        "batched PCG to 1e-10",
            **mr}
    if not args.no_serving:
        serve = {}
        for name, prec in (("fp64", hb.PRECISION_FP64), ("mixed", hb.PRECISION_MIXED)):
            if prec in runs:
                serve[name] = run_serving(hb, synth, prec, args.serve_requests, args.serve_rate)
        line["serving"] = {
            "workload": (f"{args.serve_requests} requests, Poisson arrivals at "
                         f"{args.serve_rate}/s (seed 5): 30% factorizations of n in "
                         f"{list(SERVE_SIZES)} (a = exp(N(0,1)) per face, per-operator seed), "
                         "70% PCG solves to 1e-10 of 1-32 right-hand sides against resident "
                         "operators; HBM budget 120 GB; at most 12 resident operators (oldest "
                         "released); 64 solve slots batched per iteration; clipped partition "
                         "(cells of P * 2^l DOFs per side, the last one per direction cut at "
                         "the boundary)"),
            **serve}
    if len(runs) == 2:
        line["mixed_vs_fp64"] = {
            "step_speedup": runs[hb.PRECISION_FP64]["ms_step"] / runs[hb.PRECISION_MIXED]["ms_step"],
            "factor_speedup": runs[hb.PRECISION_FP64]["factor_s"] / runs[hb.PRECISION_MIXED]["factor_s"]}
    print(json.dumps(line))
    f.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--eps", type=float, default=1e-6)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer pass (profiling)")
    ap.add_argument("--precision", default="both", choices=["fp64", "mixed", "both"])
    ap.add_argument("--no-serving", action="store_true", help="skip the serving workload")
    ap.add_argument("--no-multi-rhs", action="store_true", help="skip the 64-RHS workload")
    ap.add_argument("--no-autotune", action="store_true", help="fixed tile rules")
    ap.add_argument("--no-same-size", action="store_true",
                    help="skip the GPU rates at n = 32 and 64 (same-size reference comparison)")
    ap.add_argument("--no-fp64-cholesky", action="store_true",
                    help="skip the FP64 run with the Cholesky elimination")
    ap.add_argument("--no-level-error", action="store_true",
                    help="skip the per-level mixed-vs-FP64 error")
    ap.add_argument("--ref-n", type=int, default=REF_N,
                    help="size the reference arm runs at (it needs hours at n = 128)")
    ap.add_argument("--serve-requests", type=int, default=80)
    ap.add_argument("--serve-rate", type=float, default=8.0, help="arrivals per second")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
