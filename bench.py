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
* roofline: the M2L kernel (the largest phase), FP32-pipe bound.  achieved = the algorithmic
  flops of the reference's M2L loop, 8 sum_{j<P} (j+1)(P-j)^2 per cell pair (a complex
  multiply-add = 8 flops; 9,680 at P = 10), times the run's M2L pairs, over the M2L phase's
  event-timed duration; peak = the nominal FP32 rate 148 SMs x 128 lanes x 2 flops x the SM
  clock sampled during the timed solves (the FMA throughput measured by fmm_b200_fp32_peak
  is reported beside it).  The flops the kernel actually executes (the contraction in the
  source's azimuthal frame: 4 sum (j+1)(P-j)^2 + 14 (P(P+1)/2 - P) + 2 P = 5,490 per pair
  at P = 10) are reported as executed_tflops.
* cpu_baseline: the reference exafmm-dev CPU FMM (oracle/_ref/perf, compiled from the
  reference's sources) on the same workload (N = 2^20) with all host threads, median of 3
  runs, per phase.
* --impl reference: that reference CPU FMM as the timed arm (rank 0 only), same workload.
* cartesian (rank 0): BASELINE config 3, Cartesian P = 5, theta = 0.5, ncrit = 32, 4,194,304
  bodies on the unit sphere surface, FP32: device time, phases, M2L / P2P work and roofline,
  accuracy vs FP64 direct, and the reference CPU build on the same config.
* multi-GPU (torchrun): replicas only; every rank solves its own instance, no collective
  on the data path (a barrier and a max-reduction of the timings only).
* --strong (torchrun): one headline solve per step over all ranks through
  exafmm-dev_b200.distributed (all_gather of the bodies, a partitioned solve per GPU,
  reduce_scatter of the results), "scaling": "strong", value = N / step time (max over
  ranks).  The default multi-rank run stays replicas.
* partitioned (rank 0): the headline solve split by target parts for 2, 4 and 8 GPUs of a
  node (exafmm-dev_b200.distributed), the parts run in turn on this GPU: per-part device
  time, the slowest part plus the collectives' estimate, and the parts' sum checked bit for
  bit against the whole solve.
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
REF_N = 1 << 20                   # the reference arm runs the headline workload itself
CART = dict(dist="sphere", n=1 << 22, basis="cartesian", P=5, theta=0.5, ncrit=32, nspawn=1000,
            use_rmax=1, use_ropt=0)
CART_NAME = "sphere_N4194304_cartesian_P5_theta0.5_ncrit32_fp32"
CART_REF_CONFIG = "cart_p5_f32"
SMS, FP32_LANES = 148, 128         # B200: SMs, FP32 lanes per SM


def m2l_flops_per_pair(P, basis="spherical"):
    """Algorithmic M2L flops per cell pair: spherical 8 sum_{j<P} (j+1)(P-j)^2 (the reference
    loop, LaplaceSphericalCPU.cxx:156-190, one complex multiply-add = 8 flops); Cartesian 2
    per multiply-add of the truncated tensor contraction (420 at P = 5)."""
    if basis == "spherical":
        return 8 * sum((j + 1) * (P - j) ** 2 for j in range(P))
    nt = lambda p: p * (p + 1) * (p + 2) // 6
    return 2 * sum(((o + 1) * (o + 2) // 2) * nt(P - o) for o in range(P))


def m2l_executed_flops_per_pair(P):
    """Flops the spherical M2L kernel executes per pair: the contraction in the source's
    azimuthal frame (two real multiply-adds per term) plus the source and output rotations."""
    rot = P * (P + 1) // 2 - P
    return 4 * sum((j + 1) * (P - j) ** 2 for j in range(P)) + 14 * rot + 2 * P


def nominal_fp32_tflops(sm_mhz):
    return SMS * FP32_LANES * 2 * sm_mhz * 1e6 / 1e12


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


def run_reference(ref, x, q, wl, threads):
    """One reference CPU solve of workload wl (same parameters as the GPU arm): wall seconds
    and the reference's own per-phase times."""
    t0 = time.perf_counter()
    run = ref.run(x, q, ncrit=wl["ncrit"], nspawn=wl["nspawn"], theta=wl["theta"],
                  use_rmax=wl["use_rmax"], use_ropt=wl["use_ropt"], record=False, threads=threads)
    wall = time.perf_counter() - t0
    return wall, run.times()


def reference_median(ref, x, q, wl, threads, runs=3):
    """Median of `runs` reference solves: wall seconds and per-phase seconds (each phase's
    own median)."""
    walls, phases = [], []
    for _ in range(runs):
        w, t = run_reference(ref, x, q, wl, threads)
        walls.append(w)
        phases.append(t)
    med = {k: float(np.median([t[k] for t in phases])) for k in phases[0]}
    return float(np.median(walls)), med


# use_ropt = 0 for the mixed workloads: the cube solves carry zero net charge, for which the
# error-optimised radius (a / |M0_root|^(1/3)) grows without bound and every pair fails the
# acceptance test, turning those solves into direct sums (the reference does the same)
BATCH = dict(solves=256, n_min=1000, n_max=200000, P=8, theta=0.4, ncrit=64, nspawn=1000,
             use_ropt=0)
# the same batch at the opening angle that holds every solve to rel-L2 <= 1e-4
BATCH_THETA_1E4 = 0.3
# serving: the opening angle per order that holds every request to rel-L2 <= 1e-4 of potential
# and gradient (measured on zero-net-charge cubes and Plummer spheres of 1e3..1e6 bodies with
# the reference's FP32 + Kahan build: worst 4.1e-5 at P = 6, 2.6e-5 at P = 8, 2.1e-5 at P = 10)
SERVE = dict(requests=48, n_min=1000, n_max=1000000, orders=(6, 8, 10),
             theta={6: 0.22, 8: 0.30, 10: 0.35}, ncrit=64, use_ropt=0, workers=3, max_batch=64,
             hbm_budget_gb=60.0, load=(0.3, 0.6, 0.9), passes=3, warmup_passes=4,
             acc_min_n=10000)


def log_uniform_sizes(rng, count, lo, hi):
    return np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), count))).astype(int)


def rel_err(got, ref):
    pot = float(np.sqrt(((got[:, 0] - ref[:, 0]) ** 2).sum() / (ref[:, 0] ** 2).sum()))
    acc = float(np.sqrt(((got[:, 1:] - ref[:, 1:]) ** 2).sum() / (ref[:, 1:] ** 2).sum()))
    return pot, acc


def bench_batched(fmm, datasets, torch, dev, stream, flush, device, steps):
    """256 independent solves (N log-uniform in [1e3, 2e5], cube / Plummer / sphere surface
    by i mod 3, spherical P = 8, theta = 0.4, FP32 + compensation) in one batched call
    (a forest of independent trees) against the same solves one call each; accuracy of every
    solve against an FP64 direct sum; the same batch again at theta = 0.3, the angle at which
    every solve meets rel-L2 <= 1e-4."""
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
    # FP64 direct sums of 256 stride-sampled targets of every solve (the accuracy reference)
    samples = [datasets.sample_targets(int(counts[i]), 256) for i in range(len(counts))]
    direct = [fmm.direct(xs[i][samples[i]], xs[i], qs[i], device=device)
              for i in range(len(counts))]

    def timed(fn):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def accuracy():
        res = out.cpu().numpy().astype(np.float64)
        errs = [rel_err(res[offs[i]:offs[i + 1]][samples[i]], direct[i])
                for i in range(len(counts))]
        pot = [e[0] for e in errs]
        acc = [e[1] for e in errs]
        worst = int(np.argmax(np.maximum(pot, acc)))
        return {"max_rel_l2_pot": max(pot), "max_rel_l2_acc": max(acc),
                "median_rel_l2_acc": float(np.median(acc)),
                "solves_over_1e-4": int(sum(max(a, b) > 1e-4 for a, b in errs)),
                "worst_solve": {"index": worst, "n": int(counts[worst]),
                                "dist": dists[worst % 3]},
                "sample": "256 stride-sampled targets of every one of the %d solves, FP64 "
                          "direct sum on the GPU" % len(counts)}

    def run_batch(theta, one_by_one_too):
        kw = dict(basis="spherical", P=BATCH["P"], theta=theta, ncrit=BATCH["ncrit"],
                  nspawn=BATCH["nspawn"], use_rmax=1, use_ropt=BATCH["use_ropt"])
        s = fmm.Solver(precision="f32", device=device, **kw)
        s.set_stream(stream.cuda_stream)
        batch = lambda: s.solve_batch_device(counts, bodies.data_ptr(), out.data_ptr())
        for _ in range(3):
            timed(batch)
        ms = [timed(batch) for _ in range(max(3, steps // 2))]
        tuned = None
        if one_by_one_too:
            # the ncrit autotuner on the batch itself (the forest the last call built); the
            # timed batches run at the ncrit it picks
            best, tms = s.autotune_ncrit(candidates=(32, 48, 64, 96, 128), repeats=3)
            tuned = {"best_ncrit": best, "median_ms": {str(k): v for k, v in tms.items()}}
            for _ in range(2):
                timed(batch)
            ms = [timed(batch) for _ in range(max(3, steps // 2))]
        r = {"theta": theta, "ncrit": s.cfg.ncrit, "autotune_ncrit": tuned,
             "value": total / (float(np.median(ms)) * 1e-3),
             "unit": "particles/s",
             "ms_per_batch": {"p50": float(np.median(ms)), "p99": float(np.percentile(ms, 99))},
             "phases_ms": s.timings()}
        nm2l, np2p, body_pairs = s.list_counts()
        r["work"] = {"m2l_pairs": nm2l, "p2p_cell_pairs": np2p, "p2p_body_pairs": body_pairs}
        r["accuracy"] = accuracy()
        if one_by_one_too:
            def one_by_one():
                for i in range(len(counts)):
                    s.solve_device(int(counts[i]), bodies.data_ptr() + 16 * int(offs[i]),
                                   out.data_ptr() + 16 * int(offs[i]))
            timed(one_by_one)
            seq_ms = [timed(one_by_one) for _ in range(2)]
            r["one_call_per_solve"] = {"ms": float(np.median(seq_ms)),
                                       "value": total / (float(np.median(seq_ms)) * 1e-3)}
            r["speedup_vs_one_call_per_solve"] = float(np.median(seq_ms)) / float(np.median(ms))
        del s
        return r

    main = run_batch(BATCH["theta"], True)
    at_bound = run_batch(BATCH_THETA_1E4, False)
    del bodies, out
    main.update({
        "workload": "batched: %d solves, N log-uniform [%d, %d] (seed 44), cube/plummer/sphere "
                    "by i mod 3, spherical P=%d theta=%.2f ncrit=%d use_rmax=1 use_ropt=%d, fp32 + "
                    "compensation" % (BATCH["solves"], BATCH["n_min"], BATCH["n_max"], BATCH["P"],
                                      BATCH["theta"], BATCH["ncrit"], BATCH["use_ropt"]),
        "bodies": total, "at_theta_for_1e-4": at_bound,
        "l2": "256 MB flush before each timed batch"})
    return main


def bench_serving(fmm, datasets, device):
    """Continuous batching: Poisson arrivals of solves with N log-uniform in [1e3, 1e6],
    P uniform over {6, 8, 10} (each order at the opening angle that holds it to rel-L2 <=
    1e-4), cube or Plummer bodies (FP32 + compensation), submitted through the host C ABI:
    bursts (every request at t = 0) for the capacity, then three loads (fractions of it);
    accuracy of every request of at least 1e4 bodies against an FP64 direct sum."""
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
    srv = fmm.Server(theta=0.4, ncrit=SERVE["ncrit"], use_ropt=SERVE["use_ropt"],
                     workers=SERVE["workers"],
                     max_batch=SERVE["max_batch"], hbm_budget_gb=SERVE["hbm_budget_gb"],
                     device=device)
    for P, theta in SERVE["theta"].items():
        srv.set_theta(P, theta)

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

    # each request alone (its own handle per order, same host-buffer path, after a warm-up):
    # the latency a request would have on an idle GPU, the denominator of its slowdown
    alone = np.zeros(R)
    solo = {}
    for i, (x, q, P) in enumerate(reqs):
        s1 = solo.setdefault(P, fmm.Solver(P=P, theta=SERVE["theta"][P], ncrit=SERVE["ncrit"],
                                           use_ropt=SERVE["use_ropt"], device=device))
        s1.solve(x, q)
        t0 = time.perf_counter()
        s1.solve(x, q)
        alone[i] = time.perf_counter() - t0
    del solo
    decades = np.floor(np.log10(sizes)).astype(int)

    def row(load, lam, lat, que, wall):
        slow = lat / alone
        by_size = {"1e%d" % d: {"requests": int((decades == d).sum()),
                                "p50_ms": 1e3 * float(np.median(lat[decades == d])),
                                "p99_ms": 1e3 * float(np.percentile(lat[decades == d], 99))}
                   for d in sorted(set(decades.tolist()))}
        return {"load": load, "lambda_rps": lam, "p50_ms": 1e3 * float(np.median(lat)),
                "p99_ms": 1e3 * float(np.percentile(lat, 99)),
                "slowdown_p50": float(np.median(slow)), "slowdown_p99": float(np.percentile(slow, 99)),
                "latency_by_size": by_size,
                "queue_p50_ms": 1e3 * float(np.median(que)), "particles_per_s": total / wall}

    b0 = srv.stats()["batches"]
    # warm-up bursts: every worker's handle per order grows to the largest batch it meets
    # (the batches of a pass differ with the arrival timing, so this takes a few passes)
    warm_allocs = []
    for _ in range(SERVE["warmup_passes"]):
        a0 = fmm.device_allocations()
        run(np.zeros(R))
        warm_allocs.append(fmm.device_allocations() - a0)
    bursts, caps, outs = [], [], None
    for _ in range(SERVE["passes"]):  # bursts: every request at t = 0
        a0 = fmm.device_allocations()
        outs, lat, que, wall = run(np.zeros(R))
        caps.append(R / wall)
        bursts.append(row("burst", None, lat, que, wall))
        bursts[-1]["device_allocations"] = fmm.device_allocations() - a0
    capacity = float(np.median(caps))
    sweep = list(bursts)
    for f in SERVE["load"]:
        lam = f * capacity
        gaps = rng.exponential(1.0 / lam, R)
        gaps[0] = 0.0
        a0 = fmm.device_allocations()
        _, lat, que, wall = run(gaps)
        sweep.append(row(f, lam, lat, que, wall))
        sweep[-1]["device_allocations"] = fmm.device_allocations() - a0
    st = srv.stats()
    prof = srv.profile()
    srv.close()
    errs = {}
    for i in range(R):
        if sizes[i] < SERVE["acc_min_n"]:
            continue
        x, q, P = reqs[i]
        idx = datasets.sample_targets(len(q), 256)
        errs.setdefault(P, []).append(rel_err(outs[i][idx], fmm.direct(x[idx], x, q,
                                                                        device=device)))
    accuracy = {str(P): {"theta": SERVE["theta"][P], "requests": len(e),
                         "max_rel_l2_pot": max(v[0] for v in e),
                         "max_rel_l2_acc": max(v[1] for v in e)} for P, e in sorted(errs.items())}
    return {
        "workload": "serving: %d requests, N log-uniform [%d, %d] (seed 45), P in %s, "
                    "cube/plummer, theta per order %s, ncrit=%d use_rmax=1 use_ropt=%d, fp32 + "
                    "compensation; %d workers, max batch %d, HBM budget %.0f GB; host double "
                    "buffers through the C ABI" % (
                        R, SERVE["n_min"], SERVE["n_max"], list(SERVE["orders"]),
                        json.dumps({str(k): v for k, v in SERVE["theta"].items()}),
                        SERVE["ncrit"], SERVE["use_ropt"], SERVE["workers"],
                        SERVE["max_batch"], SERVE["hbm_budget_gb"]),
        "bodies_per_pass": total, "capacity_rps": capacity,
        "warmup_device_allocations": warm_allocs,
        "capacity_rps_per_burst": caps,
        "capacity_spread": (max(caps) - min(caps)) / capacity,
        "sweep": sweep,
        "batches": st["batches"] - b0,
        "worker_seconds_all_passes": prof,
        "accuracy": accuracy,
        "accuracy_sample": "256 stride-sampled targets of every request of >= %d bodies (last "
                           "burst), FP64 direct sum on the GPU" % SERVE["acc_min_n"],
        "alone_ms": {"p50": 1e3 * float(np.median(alone)), "max": 1e3 * float(alone.max())},
        "latency": "submit to result ready, host clock; Poisson gaps at load x capacity; "
                   "slowdown = latency / the same request solved alone through the host C ABI"}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def bench_reference(args, datasets):
    """--impl reference: the reference CPU FMM on the headline workload itself (N = 2^20,
    same bodies, parameters and float + Kahan + MASS arithmetic), rank 0 only."""
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
    x, q = datasets.make(WORKLOAD["dist"], n, seed=43, precision="f32")
    for _ in range(args.warmup):
        run_reference(ref, x, q, WORKLOAD, threads)
    walls, phases = [], []
    for _ in range(args.steps):
        w, t = run_reference(ref, x, q, WORKLOAD, threads)
        walls.append(w)
        phases.append(t)
    total = sum(walls)
    value = n * args.steps / total
    sample = "Plummer N=%d, the GPU arm's bodies and parameters, %s build, %d threads, %s" % (
        n, REF_CONFIG, threads, cpu_model())
    print(json.dumps({
        "metric": METRIC, "impl": "reference", "value": value, "unit": "particles/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Plummer, q = 1/N)",
        "config": {"workload": WORKLOAD_NAME, "n_bodies": n},
        "latency_ms": {"p50": 1e3 * float(np.median(walls)),
                       "p99": 1e3 * float(np.percentile(walls, 99))},
        "phases_ms_median": {k: 1e3 * float(np.median([t[k] for t in phases]))
                             for k in phases[0]},
        "cpu_baseline": {"value": value, "unit": "particles/s", "cores": threads,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "particles/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}))


def bench_partitioned(fmm, torch, stream, flush, device, n, bodies, whole, whole_ms, kw,
                      parts=(2, 4, 8), reps=5):
    """The headline solve split by target parts (fmm_b200_set_partition), the parts of a
    node of `parts` GPUs run one after another on this GPU: each part's device time is what
    its GPU would spend (it builds the whole tree and upward pass and computes its part's
    targets), so the slowest part plus the all_gather of the bodies and the reduce_scatter
    of the results bounds the solve on that many GPUs.  The parts' results summed must equal
    the whole solve bit for bit."""
    s = fmm.Solver(precision="f32", device=device, **kw)
    s.set_stream(stream.cuda_stream)
    o = torch.empty_like(bodies)
    acc = torch.empty_like(bodies)
    res = {}
    for R in parts:
        acc.zero_()
        part_ms, part_bodies, part_phases = [], [], []
        for r in range(R):
            s.set_partition(r, R)
            s.solve_device(n, bodies.data_ptr(), o.data_ptr())  # sizes the part's buffers
            t = []
            for _ in range(reps):
                with torch.cuda.stream(stream):
                    flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                s.solve_device(n, bodies.data_ptr(), o.data_ptr())
                e1.record(stream)
                torch.cuda.synchronize()
                t.append(e0.elapsed_time(e1))
            part_ms.append(float(np.median(t)))
            part_phases.append({k: round(v, 4) for k, v in s.timings().items()})
            _, _, b, e = s.partition()
            part_bodies.append(e - b)
            with torch.cuda.stream(stream):
                acc.add_(o)
            torch.cuda.synchronize()
        worst = max(part_ms)
        coll_ms = 2 * 16.0 * n / 770e9 * 1e3
        res[str(R)] = {
            "part_ms": part_ms, "max_ms": worst, "mean_ms": float(np.mean(part_ms)),
            "imbalance": worst / float(np.mean(part_ms)), "bodies_per_part": part_bodies,
            "slowest_part_phases_ms": part_phases[int(np.argmax(part_ms))],
            "sum_equals_whole_solve": bool(torch.equal(acc, whole)),
            "collectives_est_ms": coll_ms,
            "solve_ms_bound": worst + coll_ms,
            "speedup_vs_one_gpu": whole_ms / (worst + coll_ms)}
    s.set_partition(0, 1)
    return {"method": "target parts of one tree; parts run in turn on one GPU (median of %d "
                      "solves each, 256 MB L2 flush before each); collectives estimated as "
                      "2 x 16 B/body at the pool's measured 770 GB/s NVLink peer copy" % reps,
            "parts": res}


def bench_cartesian(fmm, datasets, torch, dev, stream, flush, device, steps, clk_mhz,
                    cpu_baseline):
    """Cartesian P = 5, theta = 0.5, ncrit = 32, N = 4,194,304 bodies on
    the unit sphere surface (charges uniform in [0, 1]), FP32 expansions: device time and
    phases, work and roofline of M2L and P2P, accuracy against an FP64 direct sum on 1024
    targets, and the reference CPU build (cart_p5_f32) on the same bodies."""
    n = CART["n"]
    x, q = datasets.make(CART["dist"], n, seed=46, precision="f32")
    kw = {k: CART[k] for k in ("basis", "P", "theta", "ncrit", "nspawn", "use_rmax", "use_ropt")}
    s = fmm.Solver(precision="f32", device=device, **kw)
    s.set_stream(stream.cuda_stream)
    bodies = torch.tensor(np.concatenate([x, q[:, None]], axis=1), dtype=torch.float32, device=dev)
    out = torch.empty_like(bodies)
    # the P2P lanes per target picked on this workload's own lists
    s.solve_device(n, bodies.data_ptr(), out.data_ptr())
    torch.cuda.synchronize()
    lanes, lanes_ms = s.autotune_p2p(repeats=3)
    ms, phase_sum = [], None
    for it in range(3 + max(3, steps // 2)):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.solve_device(n, bodies.data_ptr(), out.data_ptr())
        e1.record(stream)
        torch.cuda.synchronize()
        if it >= 3:
            ms.append(e0.elapsed_time(e1))
            t = s.timings()
            phase_sum = t if phase_sum is None else {k: phase_sum[k] + t[k] for k in t}
    phases = {k: v / len(ms) for k, v in phase_sum.items()}
    nm2l, np2p, body_pairs = s.list_counts()
    idx = datasets.sample_targets(n, 1024)
    trg = out.cpu().numpy().astype(np.float64)
    err = rel_err(trg[idx], fmm.direct(x[idx], x, q, device=device))
    del s, bodies, out
    peak = nominal_fp32_tflops(clk_mhz)
    m2l_tf = nm2l * m2l_flops_per_pair(CART["P"], "cartesian") / (phases["m2l"] * 1e-3) / 1e12
    p2p_tf = 20.0 * body_pairs / (phases["p2p"] * 1e-3) / 1e12
    res = {"workload": CART_NAME, "n_bodies": n, "steps": len(ms), "warmup": 3,
           "value": n / (float(np.median(ms)) * 1e-3), "unit": "particles/s",
           "ms_per_step": float(np.median(ms)), "phases_ms": phases,
           "work": {"m2l_pairs": nm2l, "p2p_cell_pairs": np2p, "p2p_body_pairs": body_pairs},
           "autotune_p2p_lanes": {"best": {"lanes4_max": lanes[0], "lanes2_max": lanes[1]},
                                  "p2p_median_ms": {"%d/%d" % k: v for k, v in lanes_ms.items()}},
           "roofline": {"m2l_tflops": m2l_tf, "m2l_frac": m2l_tf / peak,
                        "m2l_flops_per_pair": m2l_flops_per_pair(CART["P"], "cartesian"),
                        "p2p_tflops": p2p_tf, "p2p_frac": p2p_tf / peak, "peak": peak,
                        "peak_source": "nominal FP32 at the sampled SM clock"},
           "accuracy": {"rel_l2_pot": err[0], "rel_l2_acc": err[1], "targets": 1024,
                        "reference": "FP64 direct sum on the GPU"},
           "l2": "256 MB flush before each timed solve"}
    if cpu_baseline:
        oracle, _ = reference_lib()
        if oracle.have_reference(CART_REF_CONFIG, "perf"):
            ref = oracle.Reference(CART_REF_CONFIG, "perf")
            threads = os.cpu_count() or 1
            wall, ph = reference_median(ref, x, q, CART, threads)
            res["reference_cpu"] = {
                "value": n / wall, "unit": "particles/s", "cores": threads,
                "wall_s_median_of_3": wall, "phases_s_median": ph,
                "kind": "reference", "build": CART_REF_CONFIG + " (float, OpenMP, -O3)",
                "cpu": cpu_model()}
            res["speedup_vs_reference_cpu"] = res["value"] / res["reference_cpu"]["value"]
    return res


def bench_strong(args, fmm, datasets, torch, pg, world, rank, local):
    """--strong: one headline solve per step over all ranks (exafmm-dev_b200.distributed):
    each rank owns a contiguous 1/world of the bodies; a step is the all_gather of the
    bodies, the rank's partitioned solve and the reduce_scatter of the results, timed with
    CUDA events on the rank's stream, max over ranks.  value = N / step time."""
    dmod = importlib.import_module("exafmm-dev_b200.distributed")
    dev = torch.device("cuda", local)
    n = args.n
    x, q = datasets.make(WORKLOAD["dist"], n, seed=43, precision="f32")
    lo, hi = rank * n // world, (rank + 1) * n // world
    mine = torch.tensor(np.concatenate([x[lo:hi], q[lo:hi, None]], axis=1),
                        dtype=torch.float32, device=dev)
    kw = {k: WORKLOAD[k] for k in ("basis", "P", "theta", "ncrit", "nspawn", "use_rmax",
                                   "use_ropt")}
    if pg is None:  # one rank: a process group of one, so that the same collectives run
        import torch.distributed as dist
        if "RANK" in os.environ:  # under torchrun: its rendezvous
            dist.init_process_group("nccl", device_id=dev)
        else:
            import socket
            with socket.socket() as so:
                so.bind(("127.0.0.1", 0))
                port = so.getsockname()[1]
            dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0,
                                    world_size=1, device_id=dev)
        pg = dist
    ds = dmod.DistributedSolver(precision="f32", device=local, **kw)
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev)
    out = None
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            out = ds.solve(mine)
    torch.cuda.synchronize()
    pg.barrier()
    torch.cuda.synchronize()
    ms = []
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            out = ds.solve(mine)
            e1.record(stream)
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
    pg.barrier()
    t = torch.tensor([float(np.mean(ms))], device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    step_ms = float(t.item())
    idx = datasets.sample_targets(hi - lo, min(1024, hi - lo))
    trg = out.cpu().numpy().astype(np.float64)
    dref = fmm.direct(x[lo:hi][idx], x, q, device=local)
    err_pot = float(np.sqrt(((trg[idx, 0] - dref[:, 0]) ** 2).sum() / (dref[:, 0] ** 2).sum()))
    err_acc = float(np.sqrt(((trg[idx, 1:] - dref[:, 1:]) ** 2).sum() / (dref[:, 1:] ** 2).sum()))
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": n / (step_ms * 1e-3), "unit": "particles/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded Plummer sphere (a=1, r<10a, recentred), q = 1/N",
            "config": {"workload": WORKLOAD_NAME, "n_bodies": n, "parallelism":
                       "target parts of one tree over %d GPUs (all_gather, partitioned solve, "
                       "reduce_scatter)" % world,
                       "l2": "256 MB flush before each timed step"},
            "accuracy": {"rel_l2_pot": err_pot, "rel_l2_acc": err_acc,
                         "targets": len(idx), "reference": "FP64 direct sum on the GPU"}}))
    pg.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=WORKLOAD["n"])
    ap.add_argument("--ref-n", type=int, default=REF_N)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-solves line")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop line")
    ap.add_argument("--strong", action="store_true",
                    help="one headline solve over all ranks (target parts), not replicas")
    ap.add_argument("--no-partition", action="store_true",
                    help="skip the solve split by target parts (one node of GPUs, emulated)")
    ap.add_argument("--no-cart", action="store_true",
                    help="skip the Cartesian P = 5, N = 4,194,304 line")
    ap.add_argument("--profile", action="store_true",
                    help="warm-ups, then one solve between cudaProfilerStart/Stop (for ncu "
                         "--profile-from-start off), then exit")
    ap.add_argument("--profile-precision", default="f32", choices=["f32", "f64"],
                    help="working precision of the --profile solve")
    ap.add_argument("--profile-workload", default="headline", choices=["headline", "cartesian"],
                    help="--profile solve: the headline workload, or the Cartesian P = 5 one")
    ap.add_argument("--profile-parts", type=int, default=1,
                    help="--profile solve: part 0 of this many target parts (one GPU's share "
                         "of a solve split over a node)")
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
    if args.strong:
        return bench_strong(args, fmm, datasets, torch, pg, world, rank, local)
    dev = torch.device("cuda", local)
    n = args.n
    wl = CART if args.profile and args.profile_workload == "cartesian" else WORKLOAD
    if wl is CART and n == WORKLOAD["n"]:
        n = CART["n"]
    x, q = datasets.make(wl["dist"], n, seed=43 + rank, precision="f32")
    kw = {k: wl[k] for k in ("basis", "P", "theta", "ncrit", "nspawn", "use_rmax", "use_ropt")}
    prec = args.profile_precision if args.profile else "f32"
    solver = fmm.Solver(precision=prec, device=local, **kw)
    if args.profile and args.profile_parts > 1:
        solver.set_partition(0, args.profile_parts)
    stream = torch.cuda.Stream(device=dev)
    solver.set_stream(stream.cuda_stream)
    bodies = torch.tensor(np.concatenate([x, q[:, None]], axis=1),
                          dtype=torch.float32 if prec == "f32" else torch.float64, device=dev)
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
            print(json.dumps({"profile": CART_NAME if wl is CART else WORKLOAD_NAME,
                              "n_bodies": n, "precision": prec,
                              "parts": args.profile_parts,
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
    launches = (fmm.kernel_launches() - launches0) // args.steps
    # keep the GPU under the same load until the sampler has a few readings
    t_extra = time.perf_counter()
    while len(clocks.rows) < 5 and time.perf_counter() - t_extra < 3.0:
        step(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        torch.cuda.synchronize()
    clk = clocks.stop()
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
                "ms_per_step": float(np.mean(ms64)), "phases_ms": s64.timings(),
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
    # P2P threads per target group on the headline tree (ncrit = 64): leaf-size thresholds
    # for 4 and 2 lanes per target
    tuner.autotune_ncrit(x, q, candidates=(WORKLOAD["ncrit"],), repeats=1)  # back to 64
    tuner.solve(x, q)
    g, gms = tuner.autotune_p2p(repeats=5)
    autotune["p2p_lanes"] = {"best": {"lanes4_max": g[0], "lanes2_max": g[1]},
                             "p2p_median_ms": {"%d/%d" % k: v for k, v in gms.items()}}
    del tuner

    partitioned = None if args.no_partition else bench_partitioned(
        fmm, torch, stream, flush, local, n, bodies, out, total_ms / args.steps, kw)
    batched = None if args.no_batch else bench_batched(fmm, datasets, torch, dev, stream, flush,
                                                       local, args.steps)
    serving = None if args.no_serve else bench_serving(fmm, datasets, local)
    clk_mhz = clk["sm_mhz"] or 1965.0
    cart = None if args.no_cart else bench_cartesian(fmm, datasets, torch, dev, stream, flush,
                                                     local, args.steps, clk_mhz,
                                                     not args.no_cpu_baseline)

    # roofline of M2L (the largest phase): algorithmic flops per pair of the reference's loop
    # over the phase's event time, against the nominal FP32 rate at the sampled SM clock
    probe = fmm.fp32_peak_tflops(local)
    peak = nominal_fp32_tflops(clk_mhz)
    m2l_tflops = nm2l * m2l_flops_per_pair(WORKLOAD["P"]) / (phases["m2l"] * 1e-3) / 1e12
    m2l_exec = nm2l * m2l_executed_flops_per_pair(WORKLOAD["P"]) / (phases["m2l"] * 1e-3) / 1e12
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
            xr, qr = (x, q) if args.ref_n == n else datasets.make(
                WORKLOAD["dist"], args.ref_n, seed=43, precision="f32")
            wall, ph = reference_median(ref, xr, qr, WORKLOAD, threads)
            cpu = {"value": args.ref_n / wall, "unit": "particles/s", "cores": threads,
                   "kind": "reference",
                   "sample": "the headline workload itself (Plummer N=%d, same bodies and "
                             "parameters), reference %s build, median of 3, %s" % (
                                 args.ref_n, REF_CONFIG, cpu_model()),
                   "phases_s_median": ph}

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
                 "p2p_tflops": p2p_tflops, "p2p_frac_of_fp32_peak": p2p_tflops / peak,
                 "p2p_flops_per_pair": 20,
                 "m2l_flops_per_pair": m2l_flops_per_pair(WORKLOAD["P"]),
                 "m2l_executed_flops_per_pair": m2l_executed_flops_per_pair(WORKLOAD["P"])},
        "fp64_gpu": fp64,
        "e2e": {"value": e2e_value, "unit": "particles/s", "h2d_bytes_per_step": 32 * n,
                "d2h_bytes_per_step": 32 * n, "ms_per_step": e2e_total / len(e2e_ms)},
        "roofline": {"kernel": "M2L (k_m2l_reg<float,10>)", "bound": "fp32",
                     "achieved": m2l_tflops, "peak": peak, "unit": "TFLOP/s",
                     "frac": m2l_tflops / peak, "traffic": traffic,
                     "flops_per_pair": m2l_flops_per_pair(WORKLOAD["P"]),
                     "executed_tflops": m2l_exec, "probe_tflops": probe,
                     "frac_of_probe": m2l_tflops / probe,
                     "peak_source": "nominal FP32: 148 SMs x 128 lanes x 2 flops x %.0f MHz "
                                    "(SM clock sampled during the timed solves); "
                                    "MEASURED_PEAKS.json has no FP32 figure; probe_tflops = "
                                    "FMA throughput measured on this GPU in this run" % clk_mhz},
        "cpu_baseline": cpu,
        "autotune_ncrit": autotune,
        "partitioned": partitioned,
        "batched": batched,
        "serving": serving,
        "cartesian": cart,
        "clocks": clk,
        "gpu_launches": int(launches),
    }
    print(json.dumps(line))
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
