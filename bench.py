#!/usr/bin/env python
"""Benchmark of the B200 Laplace FMM on the precision workload (one JSON line on rank 0).

Workload (one "step" = one full FMM solve: bounds, tree, upward pass, traversal, M2L, P2P,
downward pass): N = 1,048,576 bodies from a Plummer sphere (a = 1, radii clipped at 10a,
equal charges 1/N), spherical basis P = 10, theta = 0.35, ncrit = 64, nspawn = 1000,
use_rmax = use_ropt = 1, FP32 expansions with compensated potential/gradient sums.

* value: particles/s = N x ranks / (device time of the timed solves, max over ranks),
  bodies already resident in HBM; L2 is flushed (256 MB write) before every timed solve,
  outside its events.
* e2e: the same solve through the host C ABI (fmm_b200_solve_host: pinned double x, q in,
  p, f out, host<->device copies inside the timed region).
* roofline: the M2L kernel (the largest phase), FP32-pipe bound: algorithmic flops per cell
  pair of the contraction in the source's azimuthal frame, 4 * sum_{j<P} (j+1)(P-j)^2 (two
  real multiply-adds per term) + 6 (P(P+1)/2 - P) (rotating the source) + 8 (P(P+1)/2 - P)
  + 2 P (rotating the outputs back) = 5,490 at P = 10, over its event-timed duration,
  against the FP32 FMA peak measured on the same GPU by fmm_b200_fp32_peak.
* cpu_baseline: the reference exafmm-dev CPU FMM (oracle/_ref/perf, compiled from the
  reference's sources) on a bounded sample of the same workload with all host threads.
* --impl reference: that reference CPU FMM as the timed arm (rank 0 only).
* multi-GPU (torchrun): replicas only; every rank solves its own instance, no collective
  on the data path (a barrier and a max-reduction of the timings only).
* batched (rank 0): 256 independent solves of uneven N in one batched call (a forest of
  trees in one set of launches), against the same solves one call each.
* serving (rank 0): the continuous-batching server under Poisson arrivals at three loads,
  with p50/p99 latency, throughput and accuracy per expansion order.
"""
import argparse
import importlib
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particles/sec at N=1M P=10 (L2 err≤1e-4) vs plain GPU FMM; p50/p99 latency"
WORKLOAD = dict(dist="plummer", n=1 << 20, basis="spherical", P=10, theta=0.35, ncrit=64,
                nspawn=1000, use_rmax=1, use_ropt=1)
WORKLOAD_NAME = "plummer_N1048576_spherical_P10_theta0.35_ncrit64_fp32"
REF_CONFIG = "sph_p10_f32k_mass"   # reference build: float + KAHAN + MASS (q = 1/N)
REF_SAMPLE_N = 1 << 18            # bodies per reference step (bounded CPU sample)


def m2l_flops_per_pair(P, basis="spherical"):
    if basis == "spherical":
        rot = P * (P + 1) // 2 - P
        return 4 * sum((j + 1) * (P - j) ** 2 for j in range(P)) + 6 * rot + 8 * rot + 2 * P
    # Cartesian: 2 flops per multiply-add of the truncated tensor contraction
    nt = lambda p: p * (p + 1) * (p + 2) // 6
    return 2 * sum(((o + 1) * (o + 2) // 2) * nt(P - o) for o in range(P))


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 50 ms during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.rows, self.proc = gpu, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = set()
        for r in self.rows:
            if len(r) < 9:
                continue
            for k, name in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "samples": len(sm),
                "reasons": sorted(reasons)}


def reference_lib():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # noqa: E402  (the reference CPU build is the baseline being timed)
    if not oracle.have_reference(REF_CONFIG, "perf"):
        return None, None
    return oracle, oracle.Reference(REF_CONFIG, "perf")


def run_reference_sample(ref, datasets, n, threads, seed=43):
    x, q = datasets.make(WORKLOAD["dist"], n, seed=seed, precision="f32")
    t0 = time.perf_counter()
    run = ref.run(x, q, ncrit=WORKLOAD["ncrit"], nspawn=WORKLOAD["nspawn"],
                  theta=WORKLOAD["theta"], use_rmax=1, use_ropt=1, record=False,
                  threads=threads)
    wall = time.perf_counter() - t0
    return wall, run.times()


# use_ropt = 0 for the mixed workloads: the cube solves carry zero net charge, for which the
# error-optimised radius (a / |M0_root|^(1/3)) grows without bound and every pair fails the
# acceptance test, turning those solves into direct sums (the reference does the same)
BATCH = dict(solves=256, n_min=1000, n_max=200000, P=8, theta=0.4, ncrit=64, nspawn=1000,
             use_ropt=0)
SERVE = dict(requests=48, n_min=1000, n_max=1000000, orders=(6, 8, 10), theta=0.4, ncrit=64,
             use_ropt=0, workers=3, max_batch=64, hbm_budget_gb=60.0, load=(0.3, 0.6, 0.9))


def log_uniform_sizes(rng, count, lo, hi):
    return np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), count))).astype(int)


def rel_err(got, ref):
    pot = float(np.sqrt(((got[:, 0] - ref[:, 0]) ** 2).sum() / (ref[:, 0] ** 2).sum()))
    acc = float(np.sqrt(((got[:, 1:] - ref[:, 1:]) ** 2).sum() / (ref[:, 1:] ** 2).sum()))
    return pot, acc


def bench_batched(fmm, datasets, torch, dev, stream, flush, device, steps):
    """256 independent solves (N log-uniform in [1e3, 2e5], cube / Plummer / sphere surface
    by i mod 3, spherical P = 8, theta = 0.4, FP32 + compensation) in one batched call
    (a forest of independent trees) against the same solves one call each."""
    rng = np.random.default_rng(44)
    sizes = log_uniform_sizes(rng, BATCH["solves"], BATCH["n_min"], BATCH["n_max"])
    dists = ("cube", "plummer", "sphere")
    xs, qs = [], []
    for i, n in enumerate(sizes):
        x, q = datasets.make(dists[i % 3], int(n), seed=1000 + i, precision="f32")
        xs.append(x)
        qs.append(q)
    counts = sizes.astype(np.int32)
    total = int(counts.sum())
    offs = np.concatenate([[0], np.cumsum(counts)])
    host = np.concatenate([np.concatenate([x, q[:, None]], axis=1) for x, q in zip(xs, qs)])
    bodies = torch.tensor(host, dtype=torch.float32, device=dev)
    out = torch.empty_like(bodies)
    kw = dict(basis="spherical", P=BATCH["P"], theta=BATCH["theta"], ncrit=BATCH["ncrit"],
              nspawn=BATCH["nspawn"], use_rmax=1, use_ropt=BATCH["use_ropt"])
    s = fmm.Solver(precision="f32", device=device, **kw)
    s.set_stream(stream.cuda_stream)

    def timed(fn):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    batch = lambda: s.solve_batch_device(counts, bodies.data_ptr(), out.data_ptr())
    for _ in range(3):
        timed(batch)
    ms = [timed(batch) for _ in range(max(3, steps // 2))]
    phases = s.timings()
    nm2l, np2p, body_pairs = s.list_counts()
    res = out.cpu().numpy().astype(np.float64)

    def one_by_one():
        for i in range(len(counts)):
            s.solve_device(int(counts[i]), bodies.data_ptr() + 16 * int(offs[i]),
                           out.data_ptr() + 16 * int(offs[i]))

    timed(one_by_one)
    seq_ms = [timed(one_by_one) for _ in range(2)]
    errs = []
    for i in range(6):  # two solves of each distribution
        idx = datasets.sample_targets(int(counts[i]), 256)
        d = fmm.direct(xs[i][idx], xs[i], qs[i], device=device)
        errs.append(rel_err(res[offs[i]:offs[i + 1]][idx], d))
    del bodies, out, s
    return {
        "workload": "batched: %d solves, N log-uniform [%d, %d] (seed 44), cube/plummer/sphere "
                    "by i mod 3, spherical P=%d theta=%.2f ncrit=%d use_rmax=1 use_ropt=%d, fp32 + "
                    "compensation" % (BATCH["solves"], BATCH["n_min"], BATCH["n_max"], BATCH["P"],
                                      BATCH["theta"], BATCH["ncrit"], BATCH["use_ropt"]),
        "bodies": total, "value": total / (float(np.median(ms)) * 1e-3), "unit": "particles/s",
        "ms_per_batch": {"p50": float(np.median(ms)), "p99": float(np.percentile(ms, 99))},
        "one_call_per_solve": {"ms": float(np.median(seq_ms)),
                               "value": total / (float(np.median(seq_ms)) * 1e-3)},
        "speedup_vs_one_call_per_solve": float(np.median(seq_ms)) / float(np.median(ms)),
        "phases_ms": phases,
        "work": {"m2l_pairs": nm2l, "p2p_cell_pairs": np2p, "p2p_body_pairs": body_pairs},
        "accuracy": {"max_rel_l2_pot": max(e[0] for e in errs),
                     "max_rel_l2_acc": max(e[1] for e in errs),
                     "sample": "256 targets of each of solves 0-5, FP64 direct sum on the GPU"},
        "l2": "256 MB flush before each timed batch"}


def bench_serving(fmm, datasets, device):
    """Continuous batching: Poisson arrivals of solves with N log-uniform in [1e3, 1e6],
    P uniform over {6, 8, 10}, cube or Plummer bodies (FP32 + compensation), submitted
    through the host C ABI at three loads (fractions of the capacity measured by a burst)."""
    import threading as th
    rng = np.random.default_rng(45)
    R = SERVE["requests"]
    sizes = log_uniform_sizes(rng, R, SERVE["n_min"], SERVE["n_max"])
    orders = rng.choice(SERVE["orders"], R)
    reqs = []
    for i in range(R):
        x, q = datasets.make(("cube", "plummer")[i % 2], int(sizes[i]), seed=2000 + i,
                             precision="f32")
        reqs.append((x, q, int(orders[i])))
    total = int(sizes.sum())
    srv = fmm.Server(theta=SERVE["theta"], ncrit=SERVE["ncrit"], use_ropt=SERVE["use_ropt"],
                     workers=SERVE["workers"],
                     max_batch=SERVE["max_batch"], hbm_budget_gb=SERVE["hbm_budget_gb"],
                     device=device)

    def run(gaps):
        ids, t0 = [None] * R, time.perf_counter()

        def submitter():
            t = t0
            for i, (x, q, P) in enumerate(reqs):
                t += gaps[i]
                d = t - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                ids[i] = srv.submit(x, q, P)

        st = th.Thread(target=submitter)
        st.start()
        st.join()
        outs, lat, que = [None] * R, [], []
        for i in range(R):
            o, l, qd = srv.wait(ids[i])
            outs[i] = o
            lat.append(l)
            que.append(qd)
        wall = time.perf_counter() - t0
        return outs, np.array(lat), np.array(que), wall

    b0 = srv.stats()["batches"]
    run(np.zeros(R))  # warm-up: handles per order, pinned staging, device buffers grown
    run(np.zeros(R))  # (the batches of a pass differ from run to run; a second pass
    #                   grows the buffers that the first batches did not reach)
    outs, lat, que, wall = run(np.zeros(R))  # burst: every request at t = 0
    capacity = R / wall
    sweep = [{"load": "burst", "lambda_rps": None, "p50_ms": 1e3 * float(np.median(lat)),
              "p99_ms": 1e3 * float(np.percentile(lat, 99)),
              "queue_p50_ms": 1e3 * float(np.median(que)), "particles_per_s": total / wall}]
    for f in SERVE["load"]:
        lam = f * capacity
        gaps = rng.exponential(1.0 / lam, R)
        gaps[0] = 0.0
        _, lat, que, wall = run(gaps)
        sweep.append({"load": f, "lambda_rps": lam, "p50_ms": 1e3 * float(np.median(lat)),
                      "p99_ms": 1e3 * float(np.percentile(lat, 99)),
                      "queue_p50_ms": 1e3 * float(np.median(que)),
                      "particles_per_s": total / wall})
    st = srv.stats()
    prof = srv.profile()
    srv.close()
    errs = {}
    for i in range(R):
        P = reqs[i][2]
        if P in errs or sizes[i] < 20000:
            continue
        x, q = reqs[i][0], reqs[i][1]
        idx = datasets.sample_targets(len(q), 256)
        errs[P] = rel_err(outs[i][idx], fmm.direct(x[idx], x, q, device=device))
    return {
        "workload": "serving: %d requests, N log-uniform [%d, %d] (seed 45), P in %s, "
                    "cube/plummer, theta=%.2f ncrit=%d use_rmax=1 use_ropt=%d, fp32 + compensation; "
                    "%d workers, max batch %d, HBM budget %.0f GB; host double buffers through "
                    "the C ABI" % (R, SERVE["n_min"], SERVE["n_max"], list(SERVE["orders"]),
                                   SERVE["theta"], SERVE["ncrit"], SERVE["use_ropt"],
                                   SERVE["workers"], SERVE["max_batch"], SERVE["hbm_budget_gb"]),
        "bodies_per_pass": total, "capacity_rps": capacity, "sweep": sweep,
        "batches": st["batches"] - b0,
        "worker_seconds_all_passes": prof,
        "accuracy": {str(P): {"rel_l2_pot": e[0], "rel_l2_acc": e[1]} for P, e in errs.items()},
        "latency": "submit to result ready, host clock; Poisson gaps at load x capacity"}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def bench_reference(args, datasets):
    """--impl reference: the reference CPU FMM, bounded sample per step, rank 0 only."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    oracle, ref = reference_lib()
    if ref is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference CPU build oracle/_ref/perf absent (built from the reference "
                          "sources by make -C oracle where they are present)"}))
        return
    threads = os.cpu_count() or 1
    n = args.ref_n
    for _ in range(args.warmup):
        run_reference_sample(ref, datasets, n, threads)
    walls = []
    for _ in range(args.steps):
        w, _t = run_reference_sample(ref, datasets, n, threads)
        walls.append(w)
    total = sum(walls)
    value = n * args.steps / total
    sample = "Plummer N=%d (same distribution and parameters, %s build, %d threads, %s)" % (
        n, REF_CONFIG, threads, cpu_model())
    print(json.dumps({
        "metric": METRIC, "impl": "reference", "value": value, "unit": "particles/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Plummer, q = 1/N)",
        "config": {"workload": WORKLOAD_NAME, "sample_n_bodies": n},
        "latency_ms": {"p50": 1e3 * float(np.median(walls)),
                       "p99": 1e3 * float(np.percentile(walls, 99))},
        "cpu_baseline": {"value": value, "unit": "particles/s", "cores": threads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "particles/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=WORKLOAD["n"])
    ap.add_argument("--ref-n", type=int, default=REF_SAMPLE_N)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-solves line")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop line")
    ap.add_argument("--profile", action="store_true",
                    help="warm-ups, then one solve between cudaProfilerStart/Stop (for ncu "
                         "--profile-from-start off), then exit")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    datasets = importlib.import_module("exafmm-dev_b200.datasets")
    if args.impl == "reference":
        return bench_reference(args, datasets)

    import torch
    fmm = importlib.import_module("exafmm-dev_b200")
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        pg = dist
    dev = torch.device("cuda", local)
    n = args.n
    x, q = datasets.make(WORKLOAD["dist"], n, seed=43 + rank, precision="f32")
    kw = {k: WORKLOAD[k] for k in ("basis", "P", "theta", "ncrit", "nspawn", "use_rmax", "use_ropt")}
    solver = fmm.Solver(precision="f32", device=local, **kw)
    stream = torch.cuda.Stream(device=dev)
    solver.set_stream(stream.cuda_stream)
    bodies = torch.tensor(np.concatenate([x, q[:, None]], axis=1), dtype=torch.float32, device=dev)
    out = torch.empty_like(bodies)
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2

    def step(ev0, ev1):
        with torch.cuda.stream(stream):
            flush.zero_()
            ev0.record(stream)
            solver.solve_device(n, bodies.data_ptr(), out.data_ptr())
            ev1.record(stream)

    for _ in range(args.warmup):
        step(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    torch.cuda.synchronize()
    if args.profile:
        torch.cuda.profiler.start()
        step(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        if rank == 0:
            print(json.dumps({"profile": WORKLOAD_NAME, "n_bodies": n,
                              "phases_ms": solver.timings(), "lists": solver.list_counts()}))
        return
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    launches0 = fmm.kernel_launches()
    clocks = ClockSampler(local)
    clocks.start()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    phase_sum = None
    for e0, e1 in evs:
        step(e0, e1)
        t = solver.timings()
        phase_sum = t if phase_sum is None else {k: phase_sum[k] + t[k] for k in t}
    torch.cuda.synchronize()
    # keep the GPU under the same load until the sampler has a few readings
    t_extra = time.perf_counter()
    while len(clocks.rows) < 5 and time.perf_counter() - t_extra < 3.0:
        step(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        torch.cuda.synchronize()
    clk = clocks.stop()
    launches = (fmm.kernel_launches() - launches0) // args.steps
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = float(sum(step_ms))
    if pg:
        t = torch.tensor([total_ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
        pg.barrier()
    value = n * world * args.steps / (total_ms * 1e-3)
    phases = {k: v / args.steps for k, v in phase_sum.items()}
    nm2l, np2p, body_pairs = solver.list_counts()

    # accuracy against an FP64 direct sum (GPU) on 1024 stride-sampled targets
    idx = datasets.sample_targets(n, 1024)
    trg = out.cpu().numpy().astype(np.float64)
    dref = fmm.direct(x[idx], x, q, device=local)
    err_pot = float(np.sqrt(((trg[idx, 0] - dref[:, 0]) ** 2).sum() / (dref[:, 0] ** 2).sum()))
    err_acc = float(np.sqrt(((trg[idx, 1:] - dref[:, 1:]) ** 2).sum() / (dref[:, 1:] ** 2).sum()))

    # end to end through the host C ABI: pinned double inputs and outputs
    hx = torch.from_numpy(np.ascontiguousarray(x.reshape(-1))).pin_memory()
    hq = torch.from_numpy(np.ascontiguousarray(q)).pin_memory()
    hp = torch.empty(n, dtype=torch.float64).pin_memory()
    hf = torch.empty(3 * n, dtype=torch.float64).pin_memory()
    for _ in range(2):
        solver.solve_host_ptrs(n, hx.data_ptr(), hq.data_ptr(), hp.data_ptr(), hf.data_ptr())
    e2e_ms = []
    for _ in range(max(3, args.steps // 2)):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solver.solve_host_ptrs(n, hx.data_ptr(), hq.data_ptr(), hp.data_ptr(), hf.data_ptr())
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    e2e_total = float(sum(e2e_ms))
    if pg:
        t = torch.tensor([e2e_total], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = n * world * len(e2e_ms) / (e2e_total * 1e-3)

    # plain FP64 GPU FMM (same pipeline in double, one solve per launch sequence)
    fp64 = None
    if not args.no_fp64:
        s64 = fmm.Solver(precision="f64", device=local, **kw)
        s64.set_stream(stream.cuda_stream)
        b64 = torch.tensor(np.concatenate([x, q[:, None]], axis=1), dtype=torch.float64, device=dev)
        o64 = torch.empty_like(b64)
        s64.solve_device(n, b64.data_ptr(), o64.data_ptr())
        ms64 = []
        for _ in range(3):
            with torch.cuda.stream(stream):
                flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s64.solve_device(n, b64.data_ptr(), o64.data_ptr())
            e1.record(stream)
            torch.cuda.synchronize()
            ms64.append(e0.elapsed_time(e1))
        t64 = o64.cpu().numpy()
        fp64 = {"value": n / (float(np.mean(ms64)) * 1e-3), "unit": "particles/s",
                "ms_per_step": float(np.mean(ms64)),
                "err_pot": float(np.sqrt(((t64[idx, 0] - dref[:, 0]) ** 2).sum() / (dref[:, 0] ** 2).sum())),
                "err_acc": float(np.sqrt(((t64[idx, 1:] - dref[:, 1:]) ** 2).sum() / (dref[:, 1:] ** 2).sum())),
                "fp32_speedup": (n / (total_ms / args.steps * 1e-3)) / (n / (float(np.mean(ms64)) * 1e-3))}
        del s64, b64, o64

    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return

    # what the ncrit autotuner would pick for this workload (the headline keeps ncrit = 64)
    tuner = fmm.Solver(precision="f32", device=local, **kw)
    tuner.set_stream(stream.cuda_stream)
    best, tms = tuner.autotune_ncrit(x, q, candidates=(32, 48, 64, 96, 128), repeats=3)
    autotune = {"best_ncrit": best, "median_ms": {str(k): v for k, v in tms.items()}}
    del tuner

    batched = None if args.no_batch else bench_batched(fmm, datasets, torch, dev, stream, flush,
                                                       local, args.steps)
    serving = None if args.no_serve else bench_serving(fmm, datasets, local)

    peak = fmm.fp32_peak_tflops(local)
    m2l_flops = nm2l * m2l_flops_per_pair(WORKLOAD["P"])
    m2l_tflops = m2l_flops / (phases["m2l"] * 1e-3) / 1e12
    p2p_tflops = 20.0 * body_pairs / (phases["p2p"] * 1e-3) / 1e12
    traffic = None
    prof = os.path.join(ROOT, "profiles", "m2l_traffic.json")
    if os.path.exists(prof):
        try:
            traffic = json.load(open(prof)).get("dram_bytes_per_launch")
        except (OSError, ValueError):
            traffic = None

    cpu = None
    if not args.no_cpu_baseline:
        oracle, ref = reference_lib()
        threads = os.cpu_count() or 1
        if ref is not None:
            walls = [run_reference_sample(ref, datasets, args.ref_n, threads)[0] for _ in range(2)]
            cpu = {"value": args.ref_n / min(walls), "unit": "particles/s", "cores": threads,
                   "kind": "reference",
                   "sample": "Plummer N=%d, same parameters, reference %s build, best of 2, %s" % (
                       args.ref_n, REF_CONFIG, cpu_model())}

    line = {
        "metric": METRIC, "value": value, "unit": "particles/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded Plummer sphere (a=1, r<10a, recentred), q = 1/N",
        "config": {"workload": WORKLOAD_NAME, "n_bodies": n, "basis": "spherical", "P": 10,
                   "theta": 0.35, "ncrit": 64, "nspawn": 1000, "use_rmax": 1, "use_ropt": 1,
                   "precision": "fp32 expansions + compensated potential/gradient",
                   "l2": "256 MB flush before each timed solve", "replicas": world},
        "latency_ms": {"p50": float(np.median(step_ms)), "p99": float(np.percentile(step_ms, 99))},
        "accuracy": {"rel_l2_pot": err_pot, "rel_l2_acc": err_acc, "targets": 1024,
                     "reference": "FP64 direct sum on the GPU"},
        "phases_ms": phases,
        "work": {"m2l_pairs": nm2l, "p2p_cell_pairs": np2p, "p2p_body_pairs": body_pairs,
                 "p2p_tflops": p2p_tflops, "p2p_frac_of_fp32_peak": p2p_tflops / peak},
        "fp64_gpu": fp64,
        "e2e": {"value": e2e_value, "unit": "particles/s", "h2d_bytes_per_step": 32 * n,
                "d2h_bytes_per_step": 32 * n, "ms_per_step": e2e_total / len(e2e_ms)},
        "roofline": {"kernel": "M2L (k_m2l_reg<float,10>)", "bound": "fp32",
                     "achieved": m2l_tflops, "peak": peak, "unit": "TFLOP/s",
                     "frac": m2l_tflops / peak, "traffic": traffic,
                     "peak_source": "fmm_b200_fp32_peak: FMA probe measured on this GPU in this run"},
        "cpu_baseline": cpu,
        "autotune_ncrit": autotune,
        "batched": batched,
        "serving": serving,
        "clocks": clk,
        "gpu_launches": int(launches),
    }
    print(json.dumps(line))
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
