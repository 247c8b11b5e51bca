#!/usr/bin/env python
"""bench.py -- OIFT + relaxation throughput of liboift_b200 on B200.

Workload (one step): the 256^3 int16 ellipsoid volume (ellipsoid (90,70,60) at 1200 on
200, bias 1+0.1 sin(2 pi x/256), noise sigma 80), 6-adjacency, uint16 [0,4095]
gradient arc weights, polarity alpha = -0.3, seeds = sphere r=6 (object) + distance<=2
boundary shell (background); arc-weight build + oriented f_max OIFT + 50 FP32
relaxation sweeps + argmax labels/mask, inputs resident in HBM.

Metric: Gvox/s = voxels / step time (whole job over all ranks: every rank processes
its own volume, weak scaling, no data-path collective -- one volume does not shard).
`e2e` is the same metric through the public host entry point oift_b200_run_host with
pinned host buffers: H2D of the int32 image and seeds, D2H of the labels, every step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

`--impl reference` times the reference's own CPU implementation (gft OIFT_Multi +
ORelax_1_Multi compiled from the reference sources into oracle/_ref) on all host
cores: P independent processes, each on a 160^3 sample of the same generator.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "OIFT+relax Gvox/s at 256^3 (exact cut energy) vs plain GPU & CPU; batched vol/s; HBM GB/s"
UNIT = "Gvox/s"
CPU_SAMPLE = 160  # edge of the bounded CPU sample (same generator, semi-axes scaled)


def workload_case(size=256, seed=2, sweeps=50):
    from roift_b200 import synth
    return synth.ellipsoid3d(seed=seed, size=size, sweeps=sweeps)


def workload_name(c):
    Z, Y, X = c.shape
    return (f"ellipsoid {X}x{Y}x{Z} int16, 6-adj, uint16 gradient weights [0,4095], "
            f"alpha={c.pol}, OIFT f_max + {c.sweeps} FP32 relaxation sweeps + argmax")


# ------------------------------------------------------------------ clocks ----
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"roift_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in open(self.path):
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        try:
            os.remove(self.path)
        except OSError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ CPU baseline ----
def _ref_worker_init(size):
    global _REF_CASE
    import oracle as O
    c = workload_case(size=size, seed=2)
    img = c.image.astype(np.int32)
    img -= min(0, int(img.min()))  # the CLI's shift to >= 0 (oiftrelax.cpp:263-268)
    _REF_CASE = (O, c, img)


def _ref_worker_step(_):
    O, c, img = _REF_CASE
    t = time.perf_counter()
    lab = O.ref_oift_multi(img, 6, c.seeds, c.seed_labels, pol=c.pol)
    O.ref_orelax_multi(img, 6, c.seeds, lab, c.sweeps, pol=c.pol)
    return time.perf_counter() - t, c.n


def _ref_job(job):
    """One (volume, seed set) job of the batch mix through the reference CPU path."""
    import oracle as O
    img, shape, seeds, labels, pol, sweeps = job
    img = img.astype(np.int32).reshape(shape)
    img -= min(0, int(img.min()))  # the CLI's shift to >= 0 (oiftrelax.cpp:263-268)
    t = time.perf_counter()
    lab = O.ref_oift_multi(img, 6, seeds, labels, pol=pol)
    O.ref_orelax_multi(img, 6, seeds, lab, sweeps, pol=pol)
    return time.perf_counter() - t, int(img.size)


def cpu_reference_batch(jobs, procs: int):
    """The first `procs` jobs of a batch, one per process on `procs` host cores, through the
    reference CPU path (gft OIFT_Multi + ORelax_1_Multi); returns (seed sets/s, Gvox/s, the
    jobs' voxels)."""
    import multiprocessing as mp
    import oracle as O
    if not O.ref_available():
        raise RuntimeError("oracle/_ref/libgft_ref.so is missing (build with make -C oracle ref)")
    sample = jobs[:procs]
    with mp.get_context("spawn").Pool(len(sample)) as pool:
        t = time.perf_counter()
        res = pool.map(_ref_job, sample, chunksize=1)
        dt = time.perf_counter() - t
    vox = sum(r[1] for r in res)
    return len(sample) / dt, vox / dt / 1e9, vox


def cpu_reference_throughput(procs: int, steps: int, warmup: int, size=CPU_SAMPLE):
    """Reference CPU path on `procs` processes (one sample each); returns per-step Gvox/s."""
    import multiprocessing as mp
    import oracle as O
    kind = "reference" if O.ref_available() else "port"
    if kind != "reference":
        raise RuntimeError("oracle/_ref/libgft_ref.so is missing (build with make -C oracle ref)")
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs, initializer=_ref_worker_init, initargs=(size,)) as pool:
        vals = []
        for i in range(warmup + steps):
            t = time.perf_counter()
            res = pool.map(_ref_worker_step, range(procs), chunksize=1)
            dt = time.perf_counter() - t
            vox = sum(r[1] for r in res)
            if i >= warmup:
                vals.append(vox / dt / 1e9)
    return vals, kind


def run_reference_arm(args, rank):
    if rank != 0:
        return
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    procs = max(1, min(cores, 32))
    c = workload_case(size=CPU_SAMPLE)
    try:
        vals, kind = cpu_reference_throughput(procs, args.steps, args.warmup)
    except Exception as e:  # pragma: no cover - only when the reference did not build
        print(json.dumps({"impl": "reference", "unavailable": str(e)}))
        return
    v = statistics.mean(vals)
    sample = (f"{procs} concurrent processes, each gft::ift::OIFT_Multi + ORelax_1_Multi "
              f"({c.sweeps} sweeps) on a {CPU_SAMPLE}^3 sample of the workload generator")
    out = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": procs * c.n / v / 1e6,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32/fp32",
           "data": "synthetic", "impl": "reference",
           "config": {"workload": workload_name(workload_case(size=256)), "sample": sample},
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": procs, "kind": kind,
                            "sample": sample},
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


# ---------------------------------------------------------------- our arm ----
def read_traffic(kernel: str, workload: str):
    """DRAM bytes per launch from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    if not os.path.exists(path):
        return None
    for ln in open(path):
        parts = ln.split()
        if len(parts) >= 3 and parts[0] == kernel and parts[1] == workload:
            return float(parts[2])
    return None


def replica_seed(rank: int) -> int:
    """Each rank segments its own volume (replicas, weak scaling): same generator and
    shape, a different seed per rank."""
    return 2 + rank


def reduce_step_time(ms_local: float, dist, device) -> float:
    """Max over ranks of a per-rank time (every rank calls it, in the same order)."""
    import torch
    t = torch.tensor([ms_local], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_gvox(world: int, voxels_per_rank: int, ms_step: float) -> float:
    """Throughput of the whole job: every rank's voxels over the slowest rank's time."""
    return world * voxels_per_rank / (ms_step * 1e-3) / 1e9


def run_batch_workload(args):
    """Many-volume batch: `nvol` int16 volumes (axes from {96..256}), 2-8 seed sets each,
    6-adj uint16 gradient weights, alpha ~ U(-0.5, 0.5), 20 sweeps, a mask per seed set.
    Times the per-volume path (run_device on one job at a time, whole GPU) and the batched
    driver (team-batched OIFT) at its autotuned and at each scanned team count."""
    import torch
    import roift_b200 as rb
    from roift_b200 import synth
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    mix = synth.batch_mix(seed=4, nvol=args.nvol, sweeps=20)
    keep, jobs_py = [], []
    for case, sets in mix:
        img = torch.from_numpy(case.image.copy()).to(dev)
        keep.append(img)
        for sd, sl in sets:
            st = torch.from_numpy(sd).to(dev)
            lt = torch.from_numpy(sl).to(dev)
            mask = torch.empty(case.n, dtype=torch.uint8, device=dev)
            keep += [st, lt, mask]
            jobs_py.append((case, img, st, lt, mask, len(sd)))
    jobs = (rb.Job * len(jobs_py))()
    for i, (case, img, st, lt, mask, ns) in enumerate(jobs_py):
        Z, Y, X = case.shape
        jobs[i] = rb.Job(img.data_ptr(), X, Y, Z, st.data_ptr(), lt.data_ptr(), ns,
                         float(np.float32(case.pol * 100.0)), None, None, mask.data_ptr(), 0)
    vox = sum(j[0].n for j in jobs_py)
    common = rb.make_params((1, 1, 1), adjacency=6, weight_mode="grad_q", wq=4095, sweeps=20)
    ctx = rb.Context(0)
    while ctx.run_batch(common, jobs, teams=0).tuning:   # warm-up: the autotuner explores
        pass
    tuned = ctx.run_batch(common, jobs, teams=0).teams

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0, r

    sampler = ClockSampler(0)
    sampler.start()
    scan, parts = {}, {}
    for teams in [int(t) for t in args.team_scan.split(",")]:
        scan[teams], st = timed(lambda: ctx.run_batch(common, jobs, teams=teams))
        parts[teams] = {"oift_ms": st.ms_oift, "relax_ms": st.ms_relax}
    batched_s, _ = timed(lambda: ctx.run_batch(common, jobs, teams=0))
    # the same batch recorded once into a CUDA graph and replayed
    graph = ctx.batch_graph(common, jobs, teams=0)
    graph.launch()
    graph_runs = [timed(graph.launch) for _ in range(3)]
    graph_s = statistics.median(r[0] for r in graph_runs)
    graph_dev_ms = statistics.median(r[1] for r in graph_runs)
    graph.close()
    # the per-volume path: the single-volume API, one job after the other on the whole GPU
    single = rb.Context(0)

    def per_volume():
        for case, img, st, lt, mask, ns in jobs_py:
            prm = rb.make_params(case.shape, adjacency=6, weight_mode="grad_q", wq=4095,
                                 pol=case.pol, sweeps=20)
            single.run_device(prm, img.data_ptr(), st.data_ptr(), lt.data_ptr(), ns,
                              mask=mask.data_ptr())
    per_volume()                                     # warm-up (scratch growth)
    per_volume_s, _ = timed(per_volume)
    clocks = sampler.stop()
    best_s = min(batched_s, graph_s)
    # the reference's own plain-GPU OIFT (gpu/oift_fmax_gpu.cu, built from its source for
    # sm_100a), one job after the other through its entry point with host buffers, beside our
    # batched OIFT (weights + team launch, device time) and our drop-in of the same entry
    plain = None
    if not args.no_plain_gpu:
        import oracle as O
        if O.ref_gpu_available():
            ref_s = ours_s = 0.0
            for case, img, st, lt, mask, ns in jobs_py:
                img32 = case.image.astype(np.int32).reshape(-1)
                img32 -= min(0, int(img32.min()))
                sd, sl = st.cpu().numpy(), lt.cpu().numpy()
                per = float(np.float32(case.pol * 100.0))
                pc = np.array([-per, per], np.float32)
                t0 = time.perf_counter()
                O.ref_oift_fmax_gpu_run(img32.reshape(case.shape), sd, sl, pc)
                ref_s += time.perf_counter() - t0
                lab = np.full(case.n, -1, np.int32)
                lab[sd] = sl
                Z, Y, X = case.shape
                t0 = time.perf_counter()
                rb.oift_fmax_gpu_run(img32, lab, X, Y, Z, pc, sd)
                ours_s += time.perf_counter() - t0
            ours_batched_s = min(p["oift_ms"] for p in parts.values()) / 1e3
            plain = {"scope": "OIFT only, every seed set of the mix one after the other",
                     "reference_oift_fmax_gpu_run_s": ref_s,
                     "ours_oift_fmax_gpu_run_s": ours_s,
                     "ours_batched_oift_s": ours_batched_s,
                     "batched_vs_reference_per_volume": ref_s / ours_batched_s}
    # the reference CPU path on the host cores: the mix's first P seed sets, one per process
    cpu = None
    if not args.no_cpu_baseline:
        cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
        procs = max(1, min(cores, 32, len(jobs_py)))
        ref_jobs = [(case.image.reshape(-1), case.shape, st.cpu().numpy(), lt.cpu().numpy(),
                     case.pol, 20) for case, img, st, lt, mask, ns in jobs_py[:procs]]
        try:
            sets_s, cpu_gvox, cvox = cpu_reference_batch(ref_jobs, procs)
            cpu = {"value": sets_s * args.nvol / len(jobs_py), "unit": "vol/s", "cores": procs,
                   "kind": "reference", "gvox_s": cpu_gvox,
                   "sample": f"the mix's first {procs} seed sets ({cvox} voxels), one per process "
                             f"on {procs} host cores, each gft OIFT_Multi + ORelax_1_Multi (20 "
                             "sweeps, the reference's exact gradient weights, equal to the "
                             "quantised ones on these intensities); vol/s = seed sets/s x "
                             f"{args.nvol} volumes / {len(jobs_py)} seed sets"}
        except Exception as e:  # pragma: no cover - only when the reference did not build
            cpu = {"unavailable": str(e)}
    out = {"metric": "batched vol/s (64-volume mix, OIFT + 20 sweeps per seed set)",
           "value": args.nvol / best_s, "unit": "vol/s", "n_gpus": 1,
           "higher_is_better": True, "data": "synthetic", "dtype": "int32/fp32",
           "config": {"workload": f"{args.nvol} int16 volumes, axes from {{96..256}}, "
                                  f"{len(jobs_py)} seed sets, 6-adj uint16 gradient weights, "
                                  "20 FP32 sweeps", "voxels_per_pass": vox},
           "jobs": len(jobs_py), "teams": tuned,
           "team_scan_s": {str(k): v for k, v in scan.items()},
           "team_scan_parts_ms": {str(k): v for k, v in parts.items()},
           "per_volume_path": {"s": per_volume_s, "vol_s": args.nvol / per_volume_s,
                               "gvox_s": vox / per_volume_s / 1e9},
           "batched": {"s": batched_s, "vol_s": args.nvol / batched_s,
                       "gvox_s": vox / batched_s / 1e9},
           "graph_replay": {"s": graph_s, "device_ms": graph_dev_ms,
                            "vol_s": args.nvol / graph_s, "gvox_s": vox / graph_s / 1e9},
           "speedup_vs_per_volume": per_volume_s / best_s,
           "plain_gpu_reference": plain, "cpu_baseline": cpu, "clocks": clocks}
    print(json.dumps(out))
    single.close()
    ctx.close()


def run_threeobj_workload(args):
    """Three objects in 512x512x384 int16 (negative intensities allowed), 26-adjacency,
    Gaussian-RBF weights (sigma 150, quantised to [0, 4095]), 2-level coarse-to-fine cascade
    with 30 FP32 sweeps per level, conditional dilation off (multi-label).  Each step is one
    synchronous run_pyramid_device call (shift, 2 blurs, coarse pass, glue, fine pass) on
    inputs resident in HBM; the L2 is flushed between steps."""
    import torch
    import roift_b200 as rb
    from roift_b200 import synth
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    c = synth.three_ellipsoids(seed=3, shape=(args.z3, args.size3, args.size3), sweeps=30)
    N = c.n
    lab0 = np.full(N, -1, np.int32)
    lab0[c.seeds] = c.seed_labels
    d_img = torch.from_numpy(c.image.reshape(-1).copy()).to(dev)
    d_lab = torch.from_numpy(lab0).to(dev)
    d_sd = torch.from_numpy(c.seeds).to(dev)
    out = torch.empty(N, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    ctx = rb.Context(0)
    prm = rb.make_params(c.shape, adjacency=26, weight_mode="rbf_q", wq=4095, rbf_sigma=150.0,
                         pol=c.pol, sweeps=30)

    def step():
        return ctx.run_pyramid_device(prm, d_img.data_ptr(), d_lab.data_ptr(), d_sd.data_ptr(),
                                      len(c.seeds), out.data_ptr(), 2, -1.0)
    for _ in range(args.warmup):
        step()
    sampler = ClockSampler(0)
    sampler.start()
    walls, stats = [], []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        stats.append(step())
        torch.cuda.synchronize()
        walls.append(time.perf_counter() - t0)
    clocks = sampler.stop()
    ms = 1000.0 * statistics.median(walls)
    res = {"metric": "cascade Gvox/s (three objects 512x512x384, 26-adj RBF, 2 levels x 30 sweeps)",
           "value": N / (ms * 1e-3) / 1e9, "unit": "Gvox/s", "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "int32/fp32", "data": "synthetic",
           "config": {"workload": f"three ellipsoids {c.shape[2]}x{c.shape[1]}x{c.shape[0]} int16, "
                                  "26-adj, RBF sigma 150 -> uint16 [0,4095], 2-level pyramid, "
                                  "30 FP32 sweeps per level, 2 blurs", "voxels": N,
                      "seeds": int(len(c.seeds)), "l2": "flushed between timed steps"},
           "device_ms_total": statistics.median(s.ms_total for s in stats),
           "fine_ms_oift_kernel": statistics.median(s.ms_oift_kernel for s in stats),
           "fine_ms_sweeps": statistics.median(s.ms_sweeps for s in stats),
           "levels_both_passes": stats[-1].levels, "nclasses": stats[-1].nclasses,
           "clocks": clocks, "gpu_launches": sum(s.kernels for s in stats)}
    if not args.no_cpu_baseline:
        import oracle as O
        if O.ref_available():
            small = synth.three_ellipsoids(seed=3, shape=(48, 64, 64), sweeps=30)
            img = small.image.astype(np.int32)
            img -= min(0, int(img.min()))
            f = O.ref_gaussian_blur(O.ref_gaussian_blur(img).reshape(small.shape)).reshape(small.shape)
            lab = np.full(small.n, -1, np.int32)
            lab[small.seeds] = small.seed_labels
            t0 = time.perf_counter()
            O.ref_coarse_to_fine(f, 26, small.pol, 30, -1.0, small.seeds, lab)
            dt = time.perf_counter() - t0
            res["cpu_baseline"] = {"value": small.n / dt / 1e9, "unit": "Gvox/s", "cores": 1,
                                   "kind": "reference",
                                   "sample": "the reference cascade (exp_coarse_to_fine steps: "
                                             "OIFT_Multi + ORelax_1_Multi per level, exact "
                                             "gradient weights, 26-adj) on a 64x64x48 instance "
                                             "of the same generator, one thread"}
    print(json.dumps(res))
    ctx.close()


def run_diff_workload(args):
    """Sixteen 192^3 ellipsoid volumes with ground-truth masks: one training step computes,
    for every volume, the loss = soft-Dice of the membership after 40 RBF relaxation sweeps
    + soft-Dice of the cost-map confidence, and its gradient with respect to (sigma, alpha,
    beta): through the relaxation adjoint (checkpoint every 7 sweeps) and through the
    bottleneck arcs of the fixed OIFT forest; then one Adam update.  The OIFT (labels, cost)
    and its bottleneck arcs are computed once per volume (fixed forest)."""
    import torch
    import roift_b200 as rb
    from roift_b200 import synth
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    vols = synth.diff_set(nvol=args.nvol_diff, size=args.size_diff)
    ctx = rb.Context(0)
    data = []
    for c in vols:
        img = torch.from_numpy(c.image.reshape(-1).copy()).to(dev)
        sd = torch.from_numpy(c.seeds).to(dev)
        sl = torch.from_numpy(c.seed_labels).to(dev)
        lab = torch.empty(c.n, dtype=torch.int32, device=dev)
        cost = torch.empty(c.n, dtype=torch.int32, device=dev)
        arcs = torch.empty(c.n, dtype=torch.int64, device=dev)
        prm = rb.make_params(c.shape, adjacency=6, weight_mode="grad_q", wq=4095, pol=c.pol,
                             sweeps=0)
        ctx.run_device(prm, img.data_ptr(), sd.data_ptr(), sl.data_ptr(), len(c.seeds),
                       oift_label=lab.data_ptr(), cost=cost.data_ptr())
        ctx.bottleneck_arcs(prm, img.data_ptr(), cost.data_ptr(), lab.data_ptr(), sd.data_ptr(),
                            len(c.seeds), arcs.data_ptr())
        tr = torch.from_numpy(c.truth.reshape(-1).astype(np.uint8)).to(dev)
        data.append((c, img, sd, sl, lab, tr, arcs))
    theta = np.array([150.0, -0.3, 1.0])
    mom, vel, b1, b2, lr = np.zeros(3), np.zeros(3), 0.9, 0.999, np.array([5.0, 0.02, 0.02])

    def step(it):
        nonlocal mom, vel, theta
        total, grad = 0.0, np.zeros(3)
        for c, img, sd, sl, lab, tr, arcs in data:
            l, g = ctx.adjoint(c.shape, img.data_ptr(), lab.data_ptr(), sd.data_ptr(),
                               sl.data_ptr(), len(c.seeds), tr.data_ptr(), sigma=theta[0],
                               alpha=theta[1], beta=theta[2], sweeps=40, checkpoint=7)
            lc, gc = ctx.cost_adjoint(c.shape, img.data_ptr(), lab.data_ptr(), arcs.data_ptr(),
                                      tr.data_ptr(), sigma=theta[0], alpha=theta[1],
                                      beta=theta[2])
            total += l + lc
            grad += g + gc
        mom = b1 * mom + (1 - b1) * grad
        vel = b2 * vel + (1 - b2) * grad * grad
        mh, vh = mom / (1 - b1 ** (it + 1)), vel / (1 - b2 ** (it + 1))
        theta = theta - lr * mh / (np.sqrt(vh) + 1e-12)
        theta[1] = min(max(theta[1], -1.0), 1.0)
        theta[2] = min(max(theta[2], 0.0), 1.0)
        theta[0] = max(theta[0], 1.0)
        return total / len(data)
    losses = [step(i) for i in range(args.warmup)]
    sampler = ClockSampler(0)
    sampler.start()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(args.steps):
        losses.append(step(args.warmup + i))
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / args.steps
    clocks = sampler.stop()
    vox = sum(d[0].n for d in data)
    print(json.dumps({
        "metric": "adjoint training steps/s (16 x 192^3, 40 RBF sweeps, checkpoint 7, cost-map term, Adam)",
        "value": 1.0 / dt, "unit": "steps/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32 (fp64 gradient sums)",
        "data": "synthetic",
        "config": {"workload": f"{len(data)} ellipsoid volumes {args.size_diff}^3 int16 with "
                               "ground truth, OIFT forest fixed, soft-Dice of the membership "
                               "after 40 sweeps (checkpoint every 7) + soft-Dice of the "
                               "cost-map confidence (bottleneck arcs), Adam on "
                               "(sigma, alpha, beta)",
                   "voxels": vox},
        "gvox_per_s_forward_backward": vox / dt / 1e9,
        "loss_first_last": [losses[0], losses[-1]], "theta": theta.tolist(),
        "clocks": clocks}))
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain-gpu", action="store_true")
    ap.add_argument("--workload", default="ellipsoid256",
                    choices=["ellipsoid256", "batch64", "threeobj512", "diff16"])
    ap.add_argument("--nvol-diff", type=int, default=16)
    ap.add_argument("--size-diff", type=int, default=192)
    ap.add_argument("--size3", type=int, default=512, help="x/y extent of threeobj512")
    ap.add_argument("--z3", type=int, default=384, help="z extent of threeobj512")
    ap.add_argument("--team-scan", default="1,4,16,37,74,148",
                    help="team counts timed by the batch64 workload")
    ap.add_argument("--nvol", type=int, default=64)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    if args.workload == "batch64":
        if rank == 0:
            run_batch_workload(args)
        return
    if args.workload == "diff16":
        if rank == 0:
            run_diff_workload(args)
        return
    if args.workload == "threeobj512":
        if rank == 0:
            run_threeobj_workload(args)
        return

    import torch
    import roift_b200 as rb

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    dev = torch.device("cuda", local_rank)

    c = workload_case(size=args.size, seed=replica_seed(rank))
    N = c.n
    img_t = torch.from_numpy(c.image.copy()).to(dev)
    s_t = torch.from_numpy(c.seeds).to(dev)
    l_t = torch.from_numpy(c.seed_labels).to(dev)
    lab_t = torch.empty(N, dtype=torch.int32, device=dev)
    mask_t = torch.empty(N, dtype=torch.uint8, device=dev)
    cost_t = torch.empty(N, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    ctx = rb.Context(local_rank)
    prm = rb.make_params(c.shape, adjacency=6, weight_mode="grad_q", wq=4095, pol=c.pol,
                         sweeps=c.sweeps)

    def step():
        return ctx.run_device(prm, img_t.data_ptr(), s_t.data_ptr(), l_t.data_ptr(),
                              len(c.seeds), cost=cost_t.data_ptr(), label=lab_t.data_ptr(),
                              mask=mask_t.data_ptr())

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler = ClockSampler(local_rank)
    sampler.start()
    torch.cuda.synchronize()
    stats = []
    for _ in range(args.steps):
        flush.fill_(1)  # L2 flush between timed steps (outside the CUDA-event window)
        torch.cuda.synchronize()
        stats.append(step())
    torch.cuda.synchronize()
    clocks = sampler.stop()
    if dist:
        dist.barrier()
    tot_ms = sum(s.ms_total for s in stats)
    ms_step = reduce_step_time(tot_ms, dist, dev) / args.steps
    value = whole_job_gvox(world, N, ms_step)

    # ---- end to end through the host entry point (pinned buffers) ----
    e2e = None
    if not args.no_e2e:
        img32 = torch.from_numpy(c.image.astype(np.int32)).pin_memory()
        lab_pin = torch.empty(N, dtype=torch.int32).pin_memory()
        lab_init = torch.from_numpy(c.label_map())
        seeds_pin = torch.from_numpy(c.seeds.astype(np.int32)).pin_memory()
        img_np, lab_np, seeds_np = img32.numpy(), lab_pin.numpy(), seeds_pin.numpy()
        prm_h = rb.make_params(c.shape, adjacency=6, weight_mode="grad_q", wq=4095, pol=c.pol,
                               sweeps=c.sweeps)
        lab_pin.copy_(lab_init)
        ctx.run_host(prm_h, img_np, lab_np, seeds_np)  # warm the host path
        times = []
        for _ in range(max(3, args.steps // 2)):
            lab_pin.copy_(lab_init)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ctx.run_host(prm_h, img_np, lab_np, seeds_np)
            times.append(time.perf_counter() - t0)
        e2e_s = reduce_step_time(statistics.mean(times), dist, dev)
        e2e = {"value": whole_job_gvox(world, N, e2e_s * 1e3), "unit": UNIT,
               "h2d_bytes_per_step": 4 * N + 8 * len(c.seeds), "d2h_bytes_per_step": 4 * N}

    # ---- roofline of the dominant kernel (CUDA events on the launching stream) ----
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak, peak_src = json.load(open(peaks_path))["hbm_gbs"], "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    C = stats[0].nclasses
    ms_sweep = statistics.mean(s.ms_sweeps for s in stats) / c.sweeps
    ms_oiftk = statistics.mean(s.ms_oift_kernel for s in stats)
    # per sweep launch: C membership planes read + written and the int16 image, over the
    # voxels the sweep computes (the reference's growing mask; skipped tiles move nothing)
    active_per_sweep = stats[-1].relax_active_voxel_sweeps / c.sweeps
    relax_bytes = active_per_sweep * (8 * C + 2)
    oift_bytes = N * 12                  # 6 B weights + 1 B seed/label + 4 B cost + 1 B label
    if ms_sweep * c.sweeps >= ms_oiftk:
        dom, bytes_, ms_k = "relax_sweep_kernel", relax_bytes, ms_sweep
    else:
        dom, bytes_, ms_k = "oift_persistent_kernel", oift_bytes, ms_oiftk
    achieved = bytes_ / (ms_k * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_src, "kernel": dom,
                "algorithmic_bytes_per_launch": bytes_, "ms_per_launch": ms_k,
                "traffic": read_traffic(dom, f"{args.size}^3")}
    stages = {"ms_weights": statistics.mean(s.ms_weights for s in stats),
              "ms_oift": statistics.mean(s.ms_oift for s in stats),
              "ms_oift_kernel": ms_oiftk,
              "ms_relax": statistics.mean(s.ms_relax for s in stats),
              "ms_sweep": ms_sweep,
              "relax_active_fraction": active_per_sweep / N,
              "oift_levels": stats[0].levels, "oift_tile_steps": stats[0].tile_steps,
              "oift_warp_cycles": list(stats[-1].oift_cycles),
              "oift_cycles_levelwait_owner_busy_drain": list(stats[-1].oift_cycles)[0:4],
              "oift_tiles_stale_sparse_bit": list(stats[-1].oift_cycles)[7:10],
              "oift_cycles_stage_sparse_bit": list(stats[-1].oift_cycles)[4:7],
              "oift_bit_cycles_closure_layers_maskrows_expand_voxels_tail":
                  list(stats[-1].oift_cycles)[10:16],
              "oift_gbs": oift_bytes / (ms_oiftk * 1e-3) / 1e9,
              "relax_sweep_gbs": relax_bytes / (ms_sweep * 1e-3) / 1e9}

    # ---- the reference's own plain-GPU OIFT beside our drop-in of the same entry point ----
    plain = None
    if rank == 0 and world == 1 and not args.no_plain_gpu:
        import oracle as O
        if O.ref_gpu_available():
            img32 = c.image.astype(np.int32)
            img32 -= min(0, int(img32.min()))
            per = float(np.float32(c.pol * 100.0))
            pc = np.array([-per, per], np.float32)  # bg = -pol (gpu/oiftrelax_fmax_gpu.cpp:146-151)
            ref_t, ours_t = [], []
            for i in range(3):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                lab_ref, waves = O.ref_oift_fmax_gpu_run(img32, c.seeds, c.seed_labels, pc)
                ref_t.append(time.perf_counter() - t0)
                lab = c.label_map()
                t0 = time.perf_counter()
                levels = rb.oift_fmax_gpu_run(img32, lab, c.shape[2], c.shape[1], c.shape[0], pc,
                                              c.seeds)
                ours_t.append(time.perf_counter() - t0)
            plain = {"scope": "OIFT only through oift_fmax_gpu_run (host int32 buffers, "
                              "allocation and copies inside the call)",
                     "reference_ms": 1e3 * min(ref_t[1:]), "reference_waves": int(waves),
                     "ours_ms": 1e3 * min(ours_t[1:]), "ours_levels": int(levels),
                     "speedup": min(ref_t[1:]) / min(ours_t[1:]),
                     "label_mismatch_voxels": int((lab_ref != lab).sum())}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            vals, kind = cpu_reference_throughput(1, 1, 0)
            cpu = {"value": vals[0], "unit": UNIT, "cores": 1, "kind": kind,
                   "sample": f"gft OIFT_Multi + ORelax_1_Multi ({c.sweeps} sweeps), one "
                             f"thread, {CPU_SAMPLE}^3 sample of the workload generator"}
        except Exception as e:
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"unavailable: {e}"}

    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "int32/fp32", "data": "synthetic",
               "config": {"workload": workload_name(c), "voxels_per_rank": N,
                          "ranks": world, "parallelism": f"replicas{world}",
                          "l2": "flushed between timed steps (256 MiB write)"},
               "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu,
               "clocks": clocks, "gpu_launches": sum(s.kernels for s in stats),
               "plain_gpu_reference": plain,
               "stages": stages}
        print(json.dumps(out))
    ctx.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
