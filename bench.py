"""Benchmark: batched mixed-precision refactor + solve on one B200 (or N).

Workload (one step): the 63x64 power-grid MNA matrix plus 18 Vdd pad rows
(n = 4050), 50 Newton refactorizations on the same pattern with element
values perturbed log-normally (sigma = 0.1), each followed by a full solve:
fp32 factors (frozen pivots) + fp64 GMRES-IR (restart 30, inner stop 1e-4,
rtol 1e-10), all 50 systems in one CUDA graph of the engine's persistent
kernels.  `value` counts only systems whose solution is within rel-L2 1e-6
of the fp64 oracle (the compiled reference's solve, checked after timing).

Also reported on the same line: the plain fp64 GPU path on the same inputs
and the same timing protocol (batched; per request), p50/p99 single-request
latency, the end-to-end figure through the public API with host buffers
(e2e), the roofline of the sparse refactor kernel (the dominant kernel) and
of the solve kernel, the reference's CPU path on one pinned core
(cpu_baseline), and the other workloads as keys: config0 (n = 989 analog
circuit: CPU factor+solve time, GPU per request and batched), config2 (512
uneven analog matrices x 8 refactors in one launch) and config3 (n = 40,000
circuit: SpMV variants and the full solve).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
For N > 1 launch with torch.distributed.run (one rank per GPU); ranks run
independent replicas of the workload (no exchange), value = all ranks'
systems / max time.  --impl reference times the reference's CPU path over
all host cores on the same value sets (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "refactor+solves/s at rel err ≤1e-6 (mixed vs fp64 GPU); p50/p99 solve latency"
UNIT = "refactor+solves/s"
NSYS = 50
# Device-side spin (SM cycles, ~0.1 ms) enqueued before a timed interval so
# the host has queued the timed work before the GPU reaches it.
HOST_AHEAD_CYCLES = 200_000
WORKLOAD = ("power-grid MNA n=4050 (63x64 mesh + 18 Vdd pads), 50 Newton refactors on one "
            "pattern (log-normal sigma=0.1 element perturbation), each followed by a full solve")
METHOD = ("fp32 factor (frozen pivots, fp64 work vector) + fp64 GMRES-IR (restart 30, inner stop 1e-4, "
          "rtol 1e-10, forward-error stop 1e-8); one CUDA graph of the engine's kernels per step")


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}


def algorithmic_bytes(info, stats, vs=4):
    """Compulsory bytes (refactor part, solve part) summed over the systems,
    from the pattern sizes and the iteration counts the kernel reported:
      refactor  nnz(A)(8+4) + (n+1)4 + nnz(L+U)(vs+4) + 4n
      trisolve  nnz(L+U)(vs+4) + 2(n+1)4 + 3*8n
      SpMV      nnz(A)(s_v+4) + (n+1)4 + 8n + 8n
      inner j   SpMV(vs) + trisolve + 2 passes (j+1) 2*8n + 8n (z_j kept)
      outer     SpMV(fp64) + 3*8n; the correction sum_j y_j z_j reads the
                kept z_j (8n each) and writes 8n."""
    n, nnz = info["n"], info["nnz_a"]
    lu = info["cap"]
    refactor = nnz * 12 + (n + 1) * 4 + lu * (vs + 4) + 4 * n
    tri = lu * (vs + 4) + 2 * (n + 1) * 4 + 3 * 8 * n
    spmv_in = nnz * (vs + 4) + (n + 1) * 4 + 16 * n
    spmv64 = nnz * 12 + (n + 1) * 4 + 16 * n
    total_ref, total = 0, 0
    for st in stats:
        total_ref += refactor
        b = 0
        outer = max(st["outer_iters"], 0)
        inner = max(st["inner_iters"], 0)
        b += max(st["nres"], 1) * (spmv64 + 3 * 8 * n)
        if outer:
            per = inner / outer
            js = []
            left = inner
            for _ in range(outer):
                c = int(round(per)) if left > per else left
                js.extend(range(c))
                left -= c
            for j in js:
                b += spmv_in + tri + 2 * (j + 1) * 2 * 8 * n + 8 * n
            b += inner * 8 * n + outer * 8 * n
        total += b
    return total_ref, total


def host_cpu():
    """Host CPU description for the CPU legs: model, logical cores, cores
    this process may run on."""
    model = "unknown"
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"model": model, "nproc": os.cpu_count(), "allowed": len(os.sched_getaffinity(0))}


def cpu_pinned_pass_times(units, repeats=5, budget_s=None):
    """The reference CPU path (one lu_factor + one lu_solve_perm per unit,
    src/cpu_ref_lu.c:15-58, compiled from the reference's sources) run on ONE
    pinned core: one untimed unit, then `repeats` timed passes over the
    units.  Returns (seconds per pass for each pass, the core, kind)."""
    from oracle import oracle
    kind = "reference" if oracle.ref_available() else "port"
    allowed = sorted(os.sched_getaffinity(0))
    core = allowed[-1]
    old = set(allowed)
    os.sched_setaffinity(0, {core})
    try:
        oracle.ref_cpu_solve(*units[0])
        ts = []
        t_all = time.perf_counter()
        for _ in range(repeats):
            t = time.perf_counter()
            for u in units:
                oracle.ref_cpu_solve(*u)
            ts.append(time.perf_counter() - t)
            if budget_s is not None and len(ts) >= 5 and time.perf_counter() - t_all > budget_s:
                break
    finally:
        os.sched_setaffinity(0, old)
    return ts, core, kind


def cpu_baseline_1core(m, vals, q, repeats=5):
    """cpu_baseline of the default line: the step's value sets, one core."""
    units = [(m.n, m.Ap, m.Ai, v, q, m.b) for v in vals]
    ts, core, kind = cpu_pinned_pass_times(units, repeats)
    med, mn = statistics.median(ts), min(ts)
    return {"value": len(units) / med, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"{len(units)} refactor+solves (the step's value sets, one lu_factor + one "
                      f"lu_solve_perm each) per pass, {len(ts)} passes on core {core} (pinned); value from "
                      f"the median pass {1000 * med:.1f} ms, best pass {1000 * mn:.1f} ms",
            "best_value": len(units) / mn, "cpu": host_cpu()}


_REF_WORK = None


def _ref_pool_init(counter, cores, work):
    """Pool worker set-up: pin to the next free core, keep the workload."""
    global _REF_WORK
    with counter.get_lock():
        i = counter.value
        counter.value += 1
    os.sched_setaffinity(0, {cores[i % len(cores)]})
    _REF_WORK = work


def _ref_pool_unit(i):
    from oracle import oracle
    n, Ap, Ai, vals, q, b = _REF_WORK
    return oracle.ref_cpu_solve(n, Ap, Ai, vals[i % len(vals)], q, b) is not None


def workload_config(m, world):
    """The `config` of both arms (the driver compares them)."""
    return {"workload": WORKLOAD, "systems_per_step": NSYS, "n": m.n, "nnz": m.nnz,
            "parallelism": f"replicas x{world}"}


def setup_dist(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def max_over_ranks(v, world):
    from luspice_b200.shard import max_over_ranks as mor
    return mor(v, world)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_reference(args):
    """The reference's CPU path (lu_factor + lu_solve_perm compiled from its
    sources) over all host cores, one pinned worker process per core, on the
    same value sets and column order as the GPU arm.  A step = the step's 50
    refactor+solves.  This process loads only the checker libraries: the
    column order comes from oracle/power_grid_colamd_q.npy (the reference has
    no COLAMD), the matrix from the pure-Python generator."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp
    from luspice_b200 import mna
    from oracle import oracle
    m = mna.power_grid()
    vals = m.perturbed(NSYS, seed=4242)
    q = np.load(ROOT / "oracle" / "power_grid_colamd_q.npy")
    cores = sorted(os.sched_getaffinity(0))
    kind = "reference" if oracle.ref_available() else "port"
    ctx = mp.get_context("spawn")
    counter = ctx.Value("i", 0)
    work = (m.n, m.Ap, m.Ai, vals, q, m.b)
    with ctx.Pool(len(cores), initializer=_ref_pool_init, initargs=(counter, cores, work)) as pool:
        for _ in range(max(args.warmup, 1)):
            assert all(pool.map(_ref_pool_unit, range(NSYS), chunksize=1))
        ts = []
        for _ in range(args.steps):
            t = time.perf_counter()
            pool.map(_ref_pool_unit, range(NSYS), chunksize=1)
            ts.append(time.perf_counter() - t)
    total = sum(ts)
    rate = NSYS * len(ts) / total
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / len(ts),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": workload_config(m, world),
            "path": "reference CPU lu_factor + lu_solve_perm (src/cpu_ref_lu.c, splu.h compiled from the "
                    "reference's sources), one factorization per unit; column order: the GPU arm's COLAMD "
                    "order read from oracle/power_grid_colamd_q.npy",
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": len(cores), "kind": kind,
                             "sample": f"{args.steps} steps x {NSYS} refactor+solves, {len(cores)} worker "
                                       f"processes pinned one per core, after {max(args.warmup, 1)} warm-up "
                                       f"steps; median step {1000 * statistics.median(ts):.1f} ms",
                             "cpu": host_cpu()},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# --suite: the other workloads of the path, one JSON line each (not part of
# the default run): uneven batches, SpMV variants + a large solve, serving.
# ---------------------------------------------------------------------------
def _ev_ms(torch, fn, stream, reps, flush=None):
    """Device time of fn(), L2 flushed before each rep.  A
    short device-side spin before the start event keeps the host's launch
    overhead out of the timed interval; one untimed call first (module
    loading, first-touch allocations).  Median of the reps."""
    fn()
    torch.cuda.synchronize()
    ts = []
    for i in range(reps):
        with torch.cuda.stream(stream):
            torch.cuda._sleep(HOST_AHEAD_CYCLES)
            if flush is not None:
                flush.fill_(float(i))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def suite_uneven(torch, api, mna, oracle, stream, flush, reps=3, nsample=128):
    """512 analog matrices, n ~ U[100, 5000], distinct patterns, 8 Newton
    refactors each: 4096 systems in one launch (one CUDA graph of the
    engine's kernels), mixed and plain fp64 on the same inputs, L2 flushed
    before each timed launch.  Acceptance: a seeded sample of the systems
    against the compiled reference's fp64 solve."""
    rng = np.random.default_rng(42)
    sizes = rng.integers(100, 5001, 512)
    t0 = time.perf_counter()
    mats = [mna.analog(int(n), 42 + i) for i, n in enumerate(sizes)]
    pats = [api.Pattern.from_matrix(m) for m in mats]
    t_an = time.perf_counter() - t0
    vals, rhs, plist, owner = [], [], [], []
    for i, m in enumerate(mats):
        for v in m.perturbed(8, seed=1000 + i):
            vals.append(v)
            rhs.append(m.b)
            plist.append(pats[i])
            owner.append(i)
    out = {"workload": "512 analog MNA matrices, n ~ U[100,5000], distinct patterns, 8 refactors each "
                       "(4096 systems per launch)", "host_analysis_s_for_512_patterns": t_an}
    sample = np.random.default_rng(7).choice(len(vals), nsample, replace=False)
    for prec, name in ((api.MIXED, "mixed"), (api.FP64, "fp64")):
        B = api.Batch(plist, prec=prec)
        B.upload(vals, rhs, stream=stream)
        for _ in range(2):
            B.run(api.RUN_BOTH, stream=stream, graph=True)
        ms = _ev_ms(torch, lambda: B.run(api.RUN_BOTH, stream=stream, graph=True), stream, reps, flush)
        xs = B.split(B.download(stream=stream))
        torch.cuda.synchronize()
        acc = 0
        for s in sample:
            m = mats[owner[s]]
            _, q = plist[s].perm()
            ref = oracle.ref_cpu_solve(m.n, m.Ap, m.Ai, vals[s], q, m.b)
            acc += int(np.linalg.norm(xs[s] - ref) / np.linalg.norm(ref) <= 1e-6)
        out[name] = {"ms_per_launch": ms, "systems_per_s": len(vals) / (ms / 1000.0),
                     "accepted_in_sample": f"{acc}/{len(sample)}", "launches": B.launch_count()}
        B.close()
    out["mixed_over_fp64"] = out["mixed"]["systems_per_s"] / out["fp64"]["systems_per_s"]
    for p in pats:
        p.close()
    return out


def suite_large(torch, api, mna, oracle, stream, flush, lib, spmv_reps=20, solve_reps=3):
    """n = 40,000 circuit with supply nets: SpMV variants (HBM GB/s vs the
    measured peak, L2 flushed before each call) and a full refactor + solve
    in both precisions, accepted against the compiled reference's solve."""
    import ctypes as C
    hbm, kind = peaks()
    m = mna.large_circuit()
    A = m.csr()
    n, nnz = m.n, A.nnz
    x = np.random.default_rng(4).standard_normal(n)
    dev = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dt)
    rp, ci = dev(A.indptr, torch.int32), dev(A.indices, torch.int32)
    v64, v32 = dev(A.data, torch.float64), dev(A.data.astype(np.float32), torch.float32)
    dx, dy = dev(x, torch.float64), torch.zeros(n, dtype=torch.float64, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())
    st = C.c_void_p(stream.cuda_stream)
    out = {"workload": f"large circuit n={n}, nnz={nnz}, "
                       f"{100 * m.meta.get('frac_below_fp16_normal', 0):.0f}% of values below the fp16 normal minimum",
           "peak_gbs": hbm, "peak_kind": kind}
    spmv = {}

    def rec(name, fn, sv):
        ms = _ev_ms(torch, fn, stream, spmv_reps, flush)
        b = nnz * (sv + 4) + (n + 1) * 4 + 16 * n
        spmv[name] = {"us": ms * 1000.0, "GB_s": b / (ms / 1000.0) / 1e9, "frac": b / (ms / 1000.0) / 1e9 / hbm}

    rec("csr_fp64", lambda: lib.spmv_launch(n, p(rp), p(ci), p(v64), p(dx), p(dy), st), 8)
    rec("csr_fp32", lambda: lib.lusp_csr_spmv32(n, p(rp), p(ci), p(v32), p(dx), p(dy), st), 4)
    for kind_, sv in (("fp64", 8), ("fp32", 4), ("fp16", 2)):
        try:
            S = api.Sell(n, A.indptr, A.indices, A.data, 32, 256, kind_)
        except api.LuspError as e:
            spmv[f"sell32_256_{kind_}"] = {"refused": str(e)}
            continue
        rec(f"sell32_256_{kind_}", lambda: S.spmv(dx.data_ptr(), dy.data_ptr(), stream=stream), sv)
        spmv[f"sell32_256_{kind_}"]["padding"] = S.stored / max(S.nnz, 1)
        S.close()
    out["spmv"] = spmv
    t0 = time.perf_counter()
    P = api.Pattern.from_matrix(m)
    out["host_analysis_s"] = time.perf_counter() - t0
    _, q = P.perm()
    ref = oracle.ref_cpu_solve(n, m.Ap, m.Ai, m.Ax, q, m.b)
    for prec, inner, name in ((api.MIXED, 1, "mixed_inner_fp64"), (api.FP64, 0, "fp64")):
        B = api.Batch([P], prec=prec, inner_prec=inner, max_outer=10)
        B.upload([m.Ax], [m.b], stream=stream)
        B.run(api.RUN_BOTH, stream=stream)
        ms = _ev_ms(torch, lambda: B.run(api.RUN_BOTH, stream=stream), stream, solve_reps, flush)
        xg = B.download(stream=stream)
        torch.cuda.synchronize()
        stt = B.stats(stream=stream)[0]
        err = float(np.linalg.norm(xg - ref) / np.linalg.norm(ref))
        out[name] = {"refactor_solve_ms": ms, "rel_err": err, "accepted": int(err <= 1e-6),
                     "status": stt["status"], "outer": stt["outer_iters"], "inner": stt["inner_iters"],
                     "dense_tail": P.info["dense_tail"]}
        B.close()
    return out


def _pct(v, q):
    return float(np.percentile(v, q)) if len(v) else None


def suite_serving(torch, api, mna, oracle, stream, nreq=2000,
                  rates=(250.0, 250.0, 250.0, 500.0, 1000.0, 2000.0, 2000.0, 2000.0), diag=None):
    """Config 4: a Poisson refactor+solve request stream through the serving
    loop over 64 pattern classes (n log-uniform in [113, 40000]; analog,
    power-grid and supply-net generators in turn): 90% fresh values on a
    cached pattern, 10% a new pattern (host analysis), 5% of the cached ones
    ill-conditioned (a subcircuit's conductances scaled to 1e-14, a node held
    only by gmin); HBM admission budget 150 GB.  Each rate runs its own
    request set; throughput and p50/p99 latency overall and separately for
    cached and new-pattern requests, beside plain per-request fp64 GPU
    solves.  diag: optional path for per-request timings (JSON)."""
    rng = np.random.default_rng(42)
    specs = mna.serving_classes(64)
    t0 = time.perf_counter()
    classes = [mna.serving_class(k, n, 700 + i) for i, (k, n) in enumerate(specs)]
    gen_s = time.perf_counter() - t0
    new_id = [0]

    def make_requests(salt):
        reqs = []
        for r in range(nreq):
            u = rng.random()
            if u < 0.10:
                kind, n = specs[int(rng.integers(len(specs)))]
                m = mna.serving_class(kind, n, 5000 + new_id[0])
                new_id[0] += 1
                reqs.append((m, m.Ax, True, False))
            else:
                m = classes[int(rng.integers(len(classes)))]
                ill = rng.random() < 0.05
                v = mna.ill_conditioned(m, seed=salt + r) if ill else m.perturbed(1, seed=salt + r)[0]
                reqs.append((m, v, False, ill))
        return reqs

    threads = max(4, (os.cpu_count() or 8) - 4)
    out = {"workload": f"{nreq} requests per run over 64 pattern classes (n log-uniform [113, 40000]: analog, "
                       "power-grid and supply-net generators); 10% new patterns, 5% of the cached ones "
                       "ill-conditioned; Poisson arrivals; HBM budget 150 GB",
           "class_generation_s": gen_s, "analysis_threads": threads}
    S = api.Server(max_batch=64, streams=3, arena_gb=4.0, staging_mb=512, hbm_budget_gb=150.0,
                   analysis_threads=threads)
    t0 = time.perf_counter()
    for i in [S.submit(m.n, m.Ap, m.Ai, m.Ax, m.b) for m in classes]:   # the classes are known ahead
        S.poll(i, 600000)
    out["class_analysis_s"] = time.perf_counter() - t0
    # Untimed warm-up with the same mix (its own values and new patterns).
    warm = make_requests(1)[:400]
    for i in [S.submit(m.n, m.Ap, m.Ai, v, m.b) for m, v, _, _ in warm]:
        S.poll(i, 600000)
    runs, records = [], []
    for ri, rate in enumerate(rates):
        reqs = make_requests(1000 * (ri + 2))
        gaps = rng.exponential(1.0 / rate, nreq)
        ids, tsub = [], []
        t0 = time.perf_counter()
        tnext = t0
        for (m, v, _, _), g in zip(reqs, gaps):
            tnext += g
            while time.perf_counter() < tnext:
                pass
            tsub.append(time.perf_counter() - t0)
            ids.append(S.submit(m.n, m.Ap, m.Ai, v, m.b))
        res = [S.poll(i, 600000) for i in ids]
        done = np.array([ts + r[1]["latency_ms"] / 1000.0 for ts, r in zip(tsub, res)])
        lat = np.array([r[1]["latency_ms"] for r in res])
        new = np.array([q[2] for q in reqs])
        nn = np.array([q[0].n for q in reqs])
        hit = ~new
        ok = sum(int(r[1]["rc"] == 0) for r in res)
        acc, chk = 0, 0
        for (m, v, _, _), r in list(zip(reqs, res))[:: max(1, nreq // 40)]:
            ref = oracle.ref_cpu_solve(m.n, m.Ap, m.Ai, v, api.colamd(m.n, m.Ap, m.Ai), m.b)
            if ref is None:
                continue
            chk += 1
            acc += int(np.linalg.norm(r[0] - ref) / np.linalg.norm(ref) <= 1e-6)
        run = {"offered_per_s": rate, "arrival_window_s": float(tsub[-1]),
               "throughput_per_s": nreq / float(done.max()),
               "cached": {"count": int(hit.sum()), "throughput_per_s": int(hit.sum()) / float(done[hit].max()),
                          "p50_ms": _pct(lat[hit], 50), "p99_ms": _pct(lat[hit], 99)},
               "by_size": {name: {"count": int(sel.sum()), "p50_ms": _pct(lat[sel], 50), "p99_ms": _pct(lat[sel], 99),
                                  "throughput_per_s": int(sel.sum()) / float(done[sel].max()) if sel.any() else None}
                           for name, sel in (("n<2048", hit & (nn < 2048)),
                                             ("2048<=n<12288", hit & (nn >= 2048) & (nn < 12288)),
                                             ("n>=12288", hit & (nn >= 12288)))},
               "new_pattern": {"count": int(new.sum()), "p50_ms": _pct(lat[new], 50), "p99_ms": _pct(lat[new], 99),
                               "last_done_s": float(done[new].max()) if new.any() else None},
               "p50_ms": _pct(lat, 50), "p99_ms": _pct(lat, 99), "completed_ok": ok,
               "escalated": sum(int(r[1]["escalated"]) for r in res),
               "accepted_in_sample": f"{acc}/{chk}",
               "mean_batch": float(np.mean([r[1]["batch_size"] for r in res]))}
        runs.append(run)
        records.append([{"t_submit": ts, "latency_ms": r[1]["latency_ms"], "queue_ms": r[1]["queue_ms"],
                         "device_ms": r[1]["device_ms"], "batch": r[1]["batch_size"], "new": bool(q[2]),
                         "ill": bool(q[3]), "n": int(q[0].n), "escalated": r[1]["escalated"]}
                        for ts, r, q in zip(tsub, res, reqs)])
    out["runs"] = runs
    # Agreement of back-to-back runs at the same offered rate.
    out["throughput_spread"] = {}
    for rate in sorted(set(rates)):
        same = [r["throughput_per_s"] for r, rt in zip(runs, rates) if rt == rate]
        if len(same) > 1:
            out["throughput_spread"][str(int(rate))] = (max(same) - min(same)) / float(np.mean(same))
    out["server_stats"] = S.stats()
    S.close()
    # Plain per-request fp64 GPU solves of cached-pattern requests (patterns
    # analysed beforehand, one launch each, copies included).
    times = []
    sample = [q for q in make_requests(99)[:300] if not q[2]][:200]
    pat_cache = {}
    for m, v, _, _ in sample:
        if id(m) not in pat_cache:
            pat_cache[id(m)] = api.Pattern.from_matrix(m)
        B = api.Batch([pat_cache[id(m)]], prec=api.FP64)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        B.upload([v], [m.b], stream=stream)
        B.run(api.RUN_BOTH, stream=stream)
        B.download(stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
        B.close()
    out["fp64_per_request"] = {"mean_ms": statistics.mean(times), "per_s": 1000.0 / statistics.mean(times),
                               "p50_ms": _pct(times, 50), "p99_ms": _pct(times, 99)}
    if diag:
        Path(diag).write_text(json.dumps(records))
    return out


def run_suite(args):
    import torch
    torch.cuda.set_device(0)
    from luspice_b200 import _lib as L, api, mna
    from oracle import oracle
    stream = torch.cuda.Stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    parts = {"uneven": lambda: suite_uneven(torch, api, mna, oracle, stream, flush),
             "large": lambda: suite_large(torch, api, mna, oracle, stream, flush, L.load()),
             "serving": lambda: suite_serving(torch, api, mna, oracle, stream, diag=args.diag or None)}
    for name in args.suite.split(","):
        print(json.dumps({"suite": name, **parts[name]()}), flush=True)


def config0(torch, api, mna, oracle, stream, flush):
    """The analog MNA circuit n = 989 (900 nodes + 89 branch rows): the
    reference's CPU factor+solve on one pinned core (median and best of >= 5
    passes over 50 perturbed value sets), and the GPU paths on the same value
    sets: one request at a time (p50 device time) and the 50 as one batch."""
    m = mna.analog(989, 42)
    vals = m.perturbed(NSYS, seed=989)
    P = api.Pattern.from_matrix(m)
    _, q = P.perm()
    units = [(m.n, m.Ap, m.Ai, v, q, m.b) for v in vals]
    ts, core, kind = cpu_pinned_pass_times(units, repeats=7)
    refs = [oracle.ref_cpu_solve(*u) for u in units]
    out = {"workload": f"analog MNA n={m.n}, nnz={m.nnz} (900 nodes + 89 branch rows), {NSYS} value sets",
           "cpu_reference_1core": {"kind": kind, "core": core, "passes": len(ts),
                                   "factor_solve_ms_median": 1000 * statistics.median(ts) / len(units),
                                   "factor_solve_ms_best": 1000 * min(ts) / len(units)}}
    for prec, name in ((api.MIXED, "mixed"), (api.FP64, "fp64")):
        b1 = api.Batch([P], prec=prec)
        times, acc = [], 0
        for s_ in range(NSYS):
            b1.upload([vals[s_]], [m.b], stream=stream)
            a, bq = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            b1.run(api.RUN_BOTH, stream=stream)
            bq.record(stream)
            x = b1.download(stream=stream)
            torch.cuda.synchronize()
            times.append(a.elapsed_time(bq))
            acc += int(np.linalg.norm(x - refs[s_]) / np.linalg.norm(refs[s_]) <= 1e-6)
        b1.close()
        B = api.Batch([P] * NSYS, prec=prec)
        B.upload(list(vals), np.tile(m.b, NSYS), stream=stream)
        for _ in range(3):
            B.run(api.RUN_BOTH, stream=stream, graph=True)
        ms = _ev_ms(torch, lambda: B.run(api.RUN_BOTH, stream=stream, graph=True), stream, 5, flush)
        xs = B.split(B.download(stream=stream))
        torch.cuda.synchronize()
        accb = sum(int(np.linalg.norm(xs[i] - refs[i]) / np.linalg.norm(refs[i]) <= 1e-6) for i in range(NSYS))
        B.close()
        out[name] = {"single_request_p50_ms": float(np.percentile(times, 50)),
                     "single_request_accepted": f"{acc}/{NSYS}",
                     "batched_ms_per_launch": ms, "batched_systems_per_s": NSYS / (ms / 1000.0),
                     "batched_accepted": f"{accb}/{NSYS}"}
    P.close()
    return out


def timed_steps(torch, fn, stream, steps, flush):
    """Per-step device times (ms) of fn() on stream: before each step a short
    device-side spin (the host queues the step before the GPU reaches it) and
    an L2 flush (256 MiB write), then CUDA events around the step."""
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for i in range(steps):
        with torch.cuda.stream(stream):
            torch.cuda._sleep(HOST_AHEAD_CYCLES)
            flush.fill_(float(i))
            ev[i][0].record(stream)
        fn()
        with torch.cuda.stream(stream):
            ev[i][1].record(stream)
    torch.cuda.synchronize()
    return [a.elapsed_time(b) for a, b in ev]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other workloads' keys (configs 0, 2, 3) of the default line")
    ap.add_argument("--suite", default="", help="comma list of uneven,large,serving: the other "
                    "workloads, one JSON line each, instead of the default run")
    ap.add_argument("--diag", default="", help="--suite serving: write per-request timings to this file")
    args = ap.parse_args()
    if args.suite:
        run_suite(args)
        return
    if args.impl == "reference":
        run_reference(args)
        return
    rank, world, local = setup_dist(args.gpus)
    import torch
    torch.cuda.set_device(local)
    from luspice_b200 import api, mna

    m = mna.power_grid()
    vals = m.perturbed(NSYS, seed=4242)
    P = api.Pattern.from_matrix(m)
    info = P.info
    _, q = P.perm()
    stream = torch.cuda.Stream()
    rhs = np.tile(m.b, NSYS)
    B = api.Batch([P] * NSYS, prec=api.MIXED, krylov=30)
    B.upload(list(vals), rhs, stream=stream)
    B64 = api.Batch([P] * NSYS, prec=api.FP64)
    B64.upload(list(vals), rhs, stream=stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step(batch, what=api.RUN_BOTH):
        batch.run(what, stream=stream, graph=True)

    # Warm-up (captures the graphs), then timed steps, L2 flushed between.
    for _ in range(max(args.warmup, 3)):
        step(B)
        step(B64)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        kern_ms = timed_steps(torch, lambda: step(B), stream, args.steps, flush)
        wall = time.perf_counter() - t0
    barrier(world)
    step_ms = max_over_ranks(statistics.mean(kern_ms), world)
    # The plain fp64 GPU path on the same inputs, same protocol (spin, flush,
    # per-step events, mean over the same number of steps).
    k64 = timed_steps(torch, lambda: step(B64), stream, args.steps, flush)
    fp64_ms = max_over_ranks(statistics.mean(k64), world)

    # Accuracy gate against the fp64 oracle (same value sets, same column
    # order): the compiled reference's lu_factor + lu_solve_perm.
    from oracle import oracle
    refs = [oracle.ref_cpu_solve(m.n, m.Ap, m.Ai, vals[s], q, m.b) for s in range(NSYS)]

    def accept(xs):
        errs = [float(np.linalg.norm(xs[s] - refs[s]) / np.linalg.norm(refs[s])) for s in range(NSYS)]
        return sum(int(e <= 1e-6) for e in errs), errs

    xs = B.split(B.download(stream=stream))
    torch.cuda.synchronize()
    stats = B.stats(stream=stream)
    accepted, errs = accept(xs)
    x64 = B64.split(B64.download(stream=stream))
    torch.cuda.synchronize()
    acc64, errs64 = accept(x64)
    value = accepted * world / (step_ms / 1000.0)
    value64 = acc64 * world / (fp64_ms / 1000.0)

    # Roofline of the dominant kernel: the sparse refactor kernel (the largest
    # share of GPU time in the ncu launch list of this program), with the
    # solve kernel beside it.  Each kernel's device time comes from CUDA
    # events the library records around it on the launching stream
    # (lusp_batch_time_kernels), L2 flushed before each timed launch.
    hbm, peak_kind = peaks()
    alg_ref, alg = algorithmic_bytes(info, stats, vs=4)

    def kernel_times(batch):
        batch.time_kernels(True)
        kms = []
        for i in range(max(3, args.steps // 2)):
            with torch.cuda.stream(stream):
                torch.cuda._sleep(HOST_AHEAD_CYCLES)
                flush.fill_(float(i))
            batch.run(api.RUN_BOTH, stream=stream)
            kms.append(batch.kernel_ms())
        torch.cuda.synchronize()
        batch.time_kernels(False)
        return {k: statistics.mean(d[k] for d in kms) for k in ("refactor", "dense", "solve")}

    def refactor_kernel_name(batch):
        sh = batch.launch_shape()
        if sh["refactor_spread"] > 0:
            return (f"refactor_spread_kernel<float> ({sh['refactor_spread']} CTAs of {sh['refactor_block']} "
                    f"threads per system, {sh['refactor_grid']} CTAs)")
        return (f"refactor_kernel<float> ({sh['refactor_cluster']}-CTA cluster of {sh['refactor_block']} threads "
                f"per system, {sh['refactor_grid']} CTAs)")

    kt = kernel_times(B)
    kt64 = kernel_times(B64)
    ref_kernel = refactor_kernel_name(B)
    refactor_ms, dense_ms, solve_ms = kt["refactor"], kt["dense"], kt["solve"]
    achieved_ref = alg_ref / (refactor_ms / 1000.0) / 1e9
    achieved = alg / (solve_ms / 1000.0) / 1e9

    def traffic_of(name):
        prof = ROOT / "profiles" / name
        return json.loads(prof.read_text()).get("dram_bytes_per_launch") if prof.exists() else None

    # Single requests (one system per launch, no graph): latency p50 / p99.
    single, lat = {}, {}
    for prec in (api.FP64, api.MIXED):
        b1 = api.Batch([P], prec=prec)
        times = []
        for s in range(NSYS):
            b1.upload([vals[s]], [m.b], stream=stream)
            a, bq = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            b1.run(api.RUN_BOTH, stream=stream)
            bq.record(stream)
            torch.cuda.synchronize()
            times.append(a.elapsed_time(bq))
        single[prec] = statistics.mean(times)
        lat[prec] = (float(np.percentile(times, 50)), float(np.percentile(times, 99)))
        b1.close()

    # End to end through the public API with pinned host buffers: every step
    # copies its values and right-hand sides host->device, runs the graph and
    # reads its solutions device->host.  The headline runs the steps one
    # after another on one stream, copies included (a Newton step's values
    # depend on the previous step's solution, so its copy cannot start
    # earlier).  Also reported: two batches on two streams alternating
    # (double buffering), where step k's copies overlap step k-1's kernels
    # while the kernels of consecutive steps still run one after another.
    hv = torch.from_numpy(np.ascontiguousarray(np.concatenate(list(vals)))).pin_memory()
    hb = torch.from_numpy(np.ascontiguousarray(rhs)).pin_memory()
    hxs = [torch.empty(NSYS * m.n, dtype=torch.float64).pin_memory() for _ in range(2)]
    vals_np, rhs_np = hv.numpy(), hb.numpy()
    x_nps = [h.numpy() for h in hxs]
    B2 = api.Batch([P] * NSYS, prec=api.MIXED, krylov=30)
    bats, strs = [B, B2], [stream, torch.cuda.Stream()]
    done = [torch.cuda.Event() for _ in range(2)]

    def e2e_step(i):
        b, st_, prev = bats[i % 2], strs[i % 2], done[(i + 1) % 2]
        b.upload(vals_np, rhs_np, stream=st_)
        if i > 0:
            st_.wait_event(prev)
        b.run(api.RUN_BOTH, stream=st_, graph=True)
        done[i % 2].record(st_)
        b.download(out=x_nps[i % 2], stream=st_)

    # Serial: one batch, one stream.
    x_serial = torch.empty(NSYS * m.n, dtype=torch.float64).pin_memory().numpy()

    def serial_step():
        B.upload(vals_np, rhs_np, stream=stream)
        B.run(api.RUN_BOTH, stream=stream, graph=True)
        B.download(out=x_serial, stream=stream)

    for _ in range(3):
        serial_step()
    torch.cuda.synchronize()
    s_beg, s_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s_beg.record(stream)
    for _ in range(args.steps):
        serial_step()
    s_end.record(stream)
    torch.cuda.synchronize()
    serial_ms = max_over_ranks(s_beg.elapsed_time(s_end) / args.steps, world)
    serial_same = bool(np.array_equal(x_serial, np.concatenate(xs)))

    for i in range(4):
        e2e_step(i)
    torch.cuda.synchronize()
    e_beg, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_beg.record(strs[0])
    strs[1].wait_event(e_beg)
    for i in range(args.steps):
        e2e_step(i)
    tail_ev = torch.cuda.Event()
    tail_ev.record(strs[(args.steps - 1) % 2])
    strs[0].wait_event(tail_ev)
    other = torch.cuda.Event()
    other.record(strs[args.steps % 2])
    strs[0].wait_event(other)
    e_end.record(strs[0])
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e_beg.elapsed_time(e_end) / args.steps, world)
    h2d = int(vals_np.nbytes + rhs_np.nbytes)
    d2h = int(x_nps[0].nbytes)
    # The end-to-end results are the device-timed step's results.
    e2e_same = all(bool(np.array_equal(x, np.concatenate(xs))) for x in x_nps)
    launches = args.steps * B.launch_count()
    B.close()
    B2.close()
    B64.close()

    line = None
    if rank == 0:
        cpu = None if args.no_cpu else cpu_baseline_1core(m, vals, q)
        extra = {}
        if world == 1 and not args.no_configs:
            from luspice_b200 import _lib
            extra["config0_analog_989"] = config0(torch, api, mna, oracle, stream, flush)
            extra["config2_uneven_512x8"] = suite_uneven(torch, api, mna, oracle, stream, flush, reps=3,
                                                         nsample=64)
            extra["config3_large_40k"] = suite_large(torch, api, mna, oracle, stream, flush, _lib.load(),
                                                     spmv_reps=10, solve_reps=2)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": workload_config(m, world),
            "setup": {"method": METHOD, "lu_slots": info["cap"], "col_levels": info["ncol_levels"], "dense_tail": info["dense_tail"],
                      "l2": "flushed between timed steps (256 MiB write)", "graph": True},
            "accepted": accepted, "max_rel_err": max(errs),
            "mean_inner_iters": float(np.mean([s["inner_iters"] for s in stats])),
            "latency_ms": {"mixed_p50": lat[api.MIXED][0], "mixed_p99": lat[api.MIXED][1],
                           "fp64_p50": lat[api.FP64][0], "fp64_p99": lat[api.FP64][1]},
            "fp64_gpu": {"batched_rate": value64, "batched_ms_per_step": fp64_ms,
                         "batched_accepted": acc64, "batched_max_rel_err": max(errs64),
                         "per_request_rate": 1000.0 / single[api.FP64],
                         "protocol": "same as value: spin + L2 flush before each step, CUDA events per step, "
                                     "mean of the same number of steps",
                         "kernel_ms": kt64,
                         "mixed_over_fp64_batched": value / value64 if value64 > 0 else None},
            "e2e": {"value": accepted * world / (serial_ms / 1000.0), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": serial_ms,
                    "pipelining": "none: each step's copies, graph and read-back in order on one stream",
                    "results_equal_device_timed": serial_same,
                    "double_buffered": {"value": accepted * world / (e2e_ms / 1000.0), "ms_per_step": e2e_ms,
                                        "pipelining": "copies of step k overlap kernels of step k-1 (two "
                                        "batches, two streams); kernels of consecutive steps serialized",
                                        "results_equal_device_timed": e2e_same}},
            "roofline": {"bound": "hbm", "achieved": achieved_ref, "peak": hbm, "unit": "GB/s",
                         "frac": achieved_ref / hbm,
                         "traffic": traffic_of("refactor_spread_kernel_power_grid4050x50.json"),
                         "peak_kind": peak_kind, "kernel": ref_kernel,
                         "alg_bytes_per_launch": alg_ref, "kernel_ms": refactor_ms,
                         "dense_kernel_ms": dense_ms,
                         "solve_kernel": {"achieved": achieved, "frac": achieved / hbm,
                                          "traffic": traffic_of("solve_kernel_power_grid4050x50.json"),
                                          "alg_bytes_per_launch": alg, "kernel_ms": solve_ms}},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "wall_s_timed": wall,
            **extra,
        }
        print(json.dumps(line), flush=True)
    P.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
