"""Benchmark: triangle-evaluations per second of the elastostatic layer-potential
FMM on one or more B200s.

One triangle-evaluation = one (evaluation point, source triangle, right-hand
side) interaction (elhfmm3dtria_self_iter_dr.f:270 counts points x triangles;
times the number of right-hand sides for the batched forms).

Workloads (seeded synthetic inputs, no datasets):
  hs-fault-100k-r64 : [default] the Mindlin half-space multi-RHS configuration:
                   planar fault 40 x 20 dipping 45 degrees, top edge at depth
                   1, 250 x 200 cells x 2 = 100,000 right triangles, 64 slip
                   (displacement-jump) right-hand sides i.i.d. N(0,1),
                   lambda = mu = 1, displacement + strain at the centroids,
                   iprec 3.  Direct arrival (free-space plan) + image part
                   (image plan on the reflected centroids), both near fields
                   stored on the first call and replayed as block products;
                   a step = one mixed-precision pass of all 64 right-hand
                   sides through both plans, each replayed as a CUDA graph.
                   Beside it: the plain FP64 form (one ITER call pair per
                   right-hand side), the batched FP64 form, errors of every
                   form against the FP64 direct sums on 2,000 centroids and
                   against the oracle at the CPU sample's centroids.
  hs-fault-10k-r32 : the same at 100 x 50 cells, 32 right-hand sides (the
                   small case for profiler captures).
  fault-100k-r64 / fault-10k-r32 : the same faults and right-hand sides in
                   free space (one plan).
  fault-200k-iter  : the ITER call sequence of the half-space self-evaluation
                   configuration on the free-space kernel: 500 x 200 cells
                   (200,000 triangles), iprec 2, slip = cos^2 taper + 5 %
                   N(0,1) noise (new noise per call); the timed region is the
                   whole sequence (tree + store on the first call, 9 reuses).
  hs-fault-200k-iter : the same sequence in the half space (direct arrival +
                   image part through both ITER stores).
  sphere-1.3M      : unit icosphere refined 8x (1,310,720 flat triangles) plus
                   1,000,000 targets uniform in the shell 1.05 < |x| < 3,
                   single + double layer N(0,1), iprec 2, plain FP64.
  sphere-1.3M-mixed : the same in the mixed form, errors against the FP64
                   direct sums at iprec 1, 2, 3.
  sphere-5120      : icosphere level 4 (5,120 triangles) plus 1,000 targets
                   uniform in [-2,2]^3 with |x| > 1.1, iprec 2, plain FP64.
  hs-uneven-256 / hs-uneven-32 : independent half-space faults (random
                   strike / dip / depth, triangle counts log-uniform), one
                   slip right-hand side each, mixed form.

Inputs are resident in device memory for `value`; `e2e` runs the same step
through the C ABI from pinned host buffers (elhfmm3dtria_batch_host for the
half-space batch, efmm_batch_host for the free-space batch and the mixed
sphere, elfmm3dtriatarg_ for the single ones, the ITER entry points for the
call sequences), host copies included.

--impl reference times the CPU stand-in for the reference (the oracle's direct
restatement of el3dtriadirecttarg; the Fortran reference cannot be compiled on
this image) on a bounded sample of evaluation points, all host cores.
Multi-GPU (torchrun, elfmmlib3d_b200.partition): the batched workloads split
nrhs x N right-hand-side columns on one geometry into contiguous blocks, the
uneven batch assigns nprob x N problems by a greedy n^2 balance, the
single-problem workloads run one replica per rank; no collective on the data
path; value = total evaluations / max-over-ranks time.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "hs-fault-100k-r64": dict(kind="hsbatch", nl=250, nw=200, nrhs=64, iprec=3),
    "hs-fault-10k-r32": dict(kind="hsbatch", nl=100, nw=50, nrhs=32, iprec=3),
    "fault-100k-r64": dict(kind="batch", nl=250, nw=200, nrhs=64, iprec=3),
    "fault-10k-r32": dict(kind="batch", nl=100, nw=50, nrhs=32, iprec=3),
    "fault-200k-iter": dict(kind="iter", nl=500, nw=200, calls=10, iprec=2),
    "hs-fault-200k-iter": dict(kind="hsiter", nl=500, nw=200, calls=10, iprec=2),
    "sphere-1.3M": dict(kind="single", level=8, ntarg=1_000_000, targets="shell", iprec=2),
    "sphere-5120": dict(kind="single", level=4, ntarg=1_000, targets="box", iprec=2),
    # the same sphere and shell targets in the mixed form (FP32 far field,
    # FP64 near-singular parts), errors against the FP64 direct sums at
    # iprec 1, 2, 3 (eps .5e-3, .5e-6, .5e-9)
    "sphere-1.3M-mixed": dict(kind="single_mixed", level=8, ntarg=1_000_000, targets="shell", iprec=2,
                              err_iprecs=(1, 2, 3)),
    # batched uneven geometries: independent half-space faults, random
    # strike / dip / depth, triangle counts log-uniform in [1,000, 50,000]
    "hs-uneven-256": dict(kind="uneven", nprob=256, nmin=1000, nmax=50000, iprec=3),
    "hs-uneven-32": dict(kind="uneven", nprob=32, nmin=1000, nmax=20000, iprec=3),
}


def make_fault(name, seed=1, cols=None):
    """The fault of a batched workload and its slip right-hand sides: column
    r (global index) is N(0,1) from seed 1000 seed + r; `cols` = [start,
    stop) of the global columns this rank holds (default all of nrhs)."""
    from elfmmlib3d_b200 import geometry as G
    w = WORKLOADS[name]
    tri, nrm, cen, _ = G.planar_fault(w["nl"], w["nw"])
    a, b = cols if cols is not None else (0, w["nrhs"])
    sdl = np.stack([np.random.default_rng(seed * 1000 + r).normal(size=cen.shape) for r in range(a, b)])
    return tri, nrm, cen, sdl, w["iprec"]


def rank_columns(name, world, rank):
    """This rank's block of the job's right-hand-side columns: the job is
    nrhs x world columns on one geometry, split into contiguous blocks
    (elfmmlib3d_b200.partition.rhs_columns), nrhs per rank."""
    from elfmmlib3d_b200.partition import rhs_columns
    return rhs_columns(WORKLOADS[name]["nrhs"] * world, world, rank)


def make_inputs(name, seed=1):
    from elfmmlib3d_b200 import geometry as G
    w = WORKLOADS[name]
    if w["kind"] in ("batch", "hsbatch"):
        tri, nrm, cen, sdl, iprec = make_fault(name, seed)
        return tri, nrm, cen, np.zeros((0, 3)), None, sdl[0], iprec
    if w["kind"] in ("iter", "hsiter"):
        tri, nrm, cen, us = G.planar_fault(w["nl"], w["nw"])
        sdl = G.tapered_slip(cen, us, 40.0, 20.0, 1.0, 45.0, 0.05, seed=seed)
        return tri, nrm, cen, np.zeros((0, 3)), None, sdl, w["iprec"]
    tri, nrm, cen = G.sphere_triangles(w["level"])
    if w["targets"] == "shell":
        tgt = G.shell_targets(w["ntarg"], seed + 1)
    else:
        tgt = G.box_targets(w["ntarg"], seed + 1)
    rng = np.random.default_rng(seed)
    ssl = rng.normal(size=cen.shape)
    sdl = rng.normal(size=cen.shape)
    return tri, nrm, cen, tgt, ssl, sdl, w["iprec"]


def max_over_ranks(x, world, device=None):
    """Largest x over the ranks of the process group (every rank calls it;
    a single process returns x).  Device times are reported as this max."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank, t_max_ms, world):
    """Whole-job throughput of independent replicas: all ranks' units over
    the slowest rank's time."""
    return world * units_per_rank / (t_max_ms * 1e-3)


class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                smax = float(r[1])
                for k, nm in enumerate(names):
                    if r[3 + k].lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def tf32_peak(torch, dev):
    """Measured dense TF32 tensor-core throughput: cuBLAS FP32 8192^3 with
    TF32 allowed, best of 10, CUDA events, TFLOP/s (2 N^3)."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    n = 8192
    a = torch.randn(n, n, dtype=torch.float32, device=dev)
    b = torch.randn(n, n, dtype=torch.float32, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(10):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    torch.backends.cuda.matmul.allow_tf32 = prev
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def gemm_peak(torch, dev, dtype):
    """Measured GEMM throughput (cuBLAS 8192^3, best of 5, CUDA events), in
    TFLOP/s; FP32 with TF32 disabled (plain FP32 pipe)."""
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, dtype=dtype, device=dev)
    b = torch.randn(n, n, dtype=dtype, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def host_threads():
    """Host threads this process can run at once: its CPU affinity, capped
    by a cgroup CPU quota when one is set."""
    n = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    try:
        with open("/sys/fs/cgroup/cpu.max") as fh:
            quota, period = fh.read().split()[:2]
        if quota != "max":
            n = min(n, max(1, int(quota) // int(period)))
    except (OSError, ValueError):
        pass
    return n


def cpu_oracle_sample(tri, cen, tgt, ssl, sdl, nsample, seed=0):
    """Oracle direct sum for nsample evaluation points against all triangles,
    all host cores: the first half of the sample on the centroids, the rest
    on the targets.  Returns (evals/s, seconds, cores, points, outputs), the
    outputs (u, strain at the first `rows` centroids; ut, et at the first
    `trows` targets) kept for the GPU forms' errors against the oracle."""
    from oracle import oracle as O
    O.lib()
    n = len(cen)
    half = nsample // 2
    t0 = time.perf_counter()
    if len(tgt) == 0:
        half = nsample
    half = min(half, n)
    nt = min(nsample - half, len(tgt))
    pt, st, ptt, stt = O.direct(1.0, 1.0, tri, cen, ssl, sdl, tgt, rows=(0, half), trows=(0, nt))
    dt = time.perf_counter() - t0
    ref = {"rows": half, "trows": nt, "u": pt[:half], "e": st[:half], "ut": ptt[:nt], "et": stt[:nt]}
    return (half + nt) * n / dt, dt, host_threads(), half + nt, ref


def cpu_oracle_hs_sample(tri, nrm, cen, ssl, sdl, nsample):
    """Oracle half-space self-evaluation at the first nsample centroids
    against all triangles: the direct arrival (free-space direct sum) plus
    the image part (the oracle's C image quadrature, refined by distance to
    the reflected target), all host cores.  Returns (evals/s, seconds,
    cores, points)."""
    from oracle import oracle as O
    O.lib()
    n = len(cen)
    nsample = min(nsample, n)
    t0 = time.perf_counter()
    pt, st, _, _ = O.direct(1.0, 1.0, tri, cen, ssl, sdl, None, rows=(0, nsample), trows=(0, 0))
    ui, ei = O.image_direct(1.0, 1.0, tri, nrm, ssl, sdl, cen[:nsample], level=-1)
    dt = time.perf_counter() - t0
    ref = {"rows": nsample, "trows": 0, "u": pt[:nsample] + ui, "e": st[:nsample] + ei}
    return nsample * n / dt, dt, host_threads(), nsample, ref


def uneven_sample_problems(probs):
    """The problems of an uneven batch that the CPU samples cover: about 16,
    evenly spaced in the batch (sizes drawn independently of position)."""
    return probs[::max(1, len(probs) // 16)]


def cpu_oracle_uneven_sample(probs, nsample):
    """cpu_oracle_hs_sample on the first nsample centroids of each problem of
    uneven_sample_problems.  Returns (evals/s, seconds, cores, points, the
    oracle outputs of each sampled problem)."""
    ev, dt, npts, refs = 0.0, 0.0, 0, []
    for tri, nrm, cen, ssl, sdl in uneven_sample_problems(probs):
        e, d, cores, k, ref = cpu_oracle_hs_sample(tri, nrm, cen, ssl, sdl, nsample)
        ev += e * d
        dt += d
        npts += k
        refs.append(ref)
    return ev / dt, dt, host_threads(), npts, refs


def oracle_errors(ref, u=None, e=None, ut=None, et=None):
    """Relative l2 errors of GPU outputs (numpy or torch, evaluation points
    in the order of the oracle sample) against the oracle's outputs at the
    sampled points: the first ref["rows"] centroids and ref["trows"] targets."""
    def rel(a, b):
        a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
        b = np.asarray(b)
        return float(np.linalg.norm(a - b) / np.linalg.norm(b)) if np.linalg.norm(b) > 0 else None
    out = {}
    r, t = ref["rows"], ref.get("trows", 0)
    if u is not None and r:
        out["u"] = rel(u[:r], ref["u"])
    if e is not None and r:
        out["strain"] = rel(e[:r], ref["e"])
    if ut is not None and t:
        out["u_targets"] = rel(ut[:t], ref["ut"])
    if et is not None and t:
        out["strain_targets"] = rel(et[:t], ref["et"])
    return out


def make_uneven_problems(w, world=1, rank=None):
    """The uneven batch: w["nprob"] x world half-space faults, strike
    U[0, 360), dip U[15, 90], top depth U[0.5, 5], triangle count
    log-uniform in [nmin, nmax], one slip vector N(0,1) per triangle (double
    layer).  rank given: only the problems that the greedy n^2 balance
    (elfmmlib3d_b200.partition.balance_problems) assigns to that rank."""
    from elfmmlib3d_b200.batch import fault_problem
    from elfmmlib3d_b200.partition import balance_problems
    rng = np.random.default_rng(7)
    spec = []
    for i in range(w["nprob"] * world):
        ntri = int(np.exp(rng.uniform(np.log(w["nmin"]), np.log(w["nmax"]))))
        spec.append((ntri, rng.uniform(0.0, 360.0), rng.uniform(15.0, 90.0), rng.uniform(0.5, 5.0)))
    mine = range(len(spec))
    if rank is not None:
        mine = balance_problems([float(s_[0]) ** 2 for s_ in spec], world)[rank]
    probs = []
    for i in mine:
        ntri, strike, dip, depth = spec[i]
        tri, nrm, cen, slip = fault_problem(ntri, strike, dip, depth, seed=i)
        probs.append((tri, nrm, cen, None, slip))
    return probs


# FP64 operations per near-field (point, triangle) pair of the analytic
# kernel: ncu thread-instruction counts of k_near_leaf on the sphere-5120 case,
# (dadd + dmul + 2 dfma) / pairs = (0.999e9 + 1.749e9 + 2 * 3.029e9) / 3.193e6
# (profiles/near_leaf_sphere5120.md)
NEAR_FLOPS_PER_PAIR = 2758.0


def run_ours(args, rank, world, local_rank):
    import torch
    import elfmmlib3d_b200 as E
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    tri, nrm, cen, tgt, ssl, sdl, iprec = make_inputs(args.workload, seed=1 + rank)
    n, m = len(cen), len(tgt)
    evals = (n + m) * n

    def d(a):
        return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    dtri, dnrm, dcen, dtgt, dssl, dsdl = map(d, (tri, nrm, cen, tgt, ssl, sdl))
    u = torch.empty((n, 3), dtype=torch.float64, device=dev)
    e = torch.empty((n, 3, 3), dtype=torch.float64, device=dev)
    ut = torch.empty((m, 3), dtype=torch.float64, device=dev)
    et = torch.empty((m, 3, 3), dtype=torch.float64, device=dev)
    P = E.Plan(local_rank)

    def step():
        P.set_geometry(dtri, dnrm, dcen, dtgt, iprec=iprec)
        P.evaluate(1.0, 1.0, dssl, dsdl, u, e, ut, et)

    for _ in range(args.warmup):
        step()
    near_ms = []
    l0 = E.kernel_launches()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        P.record(0)
        for _ in range(args.steps):
            step()
            near_ms.append(P.timings()["near"])
        P.record(1)
        ms = P.elapsed(0, 1)
    torch.cuda.synchronize()
    launches = E.kernel_launches() - l0
    info = P.info()
    tim = P.timings()
    setup = P.setup_timings()
    t_max = max_over_ranks(ms, world, dev)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    value = replica_value(evals * args.steps, t_max, world)

    # end to end through the Fortran ABI, pinned host buffers
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    htri, hnrm, hcen, htgt, hssl, hsdl = map(pin, (tri, nrm, cen, tgt, ssl, sdl))
    E.elfmm3dtriatarg(iprec, 1.0, 1.0, htri, hnrm, hcen, hssl, hsdl, htgt)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ier, *_ = E.elfmm3dtriatarg(iprec, 1.0, 1.0, htri, hnrm, hcen, hssl, hsdl, htgt)
        assert ier == 0, ier
    e2e_s = time.perf_counter() - t0
    e2e_t = max_over_ranks(e2e_s, world, dev)
    e2e_value = world * evals * args.steps / e2e_t
    h2d = 8 * (9 * n + 3 * n + 3 * n + 3 * m + 6 * n)
    d2h = 8 * (3 * n + 9 * n + 3 * m + 9 * m)

    if rank != 0:
        return None
    peak = gemm_peak(torch, dev, torch.float64)
    near_avg = float(np.mean(near_ms))
    flops = NEAR_FLOPS_PER_PAIR * info["near_pairs"]
    achieved = flops / (near_avg * 1e-3) / 1e12
    roof = {"kernel": "k_near_leaf", "bound": "fp64", "achieved": achieved, "peak": peak,
            "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
            "peak_source": "measured cuBLAS DGEMM 8192^3 in this run (FP64 has no entry in MEASURED_PEAKS.json)",
            "algorithmic": f"{NEAR_FLOPS_PER_PAIR:.0f} FP64 flop/pair x {info['near_pairs']} pairs"}
    cpu, oerr = None, None
    if not args.no_cpu_baseline and world == 1:
        ev, dt, cores, npts, ref = cpu_oracle_sample(tri, cen, tgt, ssl, sdl, args.cpu_sample)
        cpu = {"value": ev, "unit": "triangle-evals/s", "cores": cores, "kind": "port",
               "sample": f"oracle direct sum, {npts} evaluation points x {n} triangles ({dt:.1f} s)"}
        oerr = oracle_errors(ref, u, e, ut, et)
    out = {
        "metric": "triangle-evals/s (free-space SLP+DLP displacement+strain, FP64 FMM at iprec 2)",
        "value": value, "unit": "triangle-evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "triangles": n, "targets": m, "iprec": iprec,
                   "evals_per_step": evals, "parallelism": f"replicas{world}",
                   "l2_policy": "inputs + expansions > L2 (126 MB)",
                   "stage_ms": tim, "setup_ms": setup, "tree": {k: info[k] for k in ("nboxes", "nlev", "p", "nbox")},
                   "near_pairs": info["near_pairs"], "m2l_pairs": info["m2l_pairs"],
                   "rel_err_vs_oracle": oerr,
                   "rel_err_vs_oracle_sample": "the cpu_baseline sample's points (oracle FP64 direct sum)"},
        "e2e": {"value": e2e_value, "unit": "triangle-evals/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "timing": "host wall clock around blocking C-ABI calls"},
        "gpu_launches": launches,
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }
    return out


SINGLE_MIXED_METRIC = ("triangle-evals/s (free-space SLP+DLP displacement+strain, mixed precision, errors vs FP64 "
                       "direct sums at iprec 1/2/3)")


def run_single_mixed(args, rank, world, local_rank):
    """One right-hand side on the sphere with off-surface targets in the
    mixed form (evaluate_batch with nrhs 1, precision 1): a step =
    set_geometry + the mixed pass, as the FP64 sphere workload's step.
    Beside it: the FP64 pass at the same iprec, and the mixed form's
    relative error against the FP64 direct sums at each of err_iprecs on
    2,000 centroids and 2,000 targets (untimed)."""
    import torch
    import elfmmlib3d_b200 as E
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    w = WORKLOADS[args.workload]
    tri, nrm, cen, tgt, ssl, sdl, iprec = make_inputs(args.workload, seed=1 + rank)
    n, m = len(cen), len(tgt)
    evals = (n + m) * n

    def d(a):
        return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    dtri, dnrm, dcen, dtgt, dssl, dsdl = map(d, (tri, nrm, cen, tgt, ssl, sdl))
    z = lambda *shape: torch.zeros(shape, dtype=torch.float64, device=dev)
    u, e, ut, et = z(1, n, 3), z(1, n, 3, 3), z(1, m, 3), z(1, m, 3, 3)
    P = E.Plan(local_rank)

    def step(ip=iprec):
        P.set_geometry(dtri, dnrm, dcen, dtgt, iprec=ip)
        P.evaluate_batch(1.0, 1.0, 1, dssl[None], dsdl[None], u, e, ut, et, precision=1)

    for _ in range(args.warmup):
        step()
    l0 = E.kernel_launches()
    stage = []
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        P.record(0)
        for _ in range(args.steps):
            step()
            stage.append(P.timings())
        P.record(1)
        ms = P.elapsed(0, 1)
    torch.cuda.synchronize()
    launches = E.kernel_launches() - l0
    t_max = max_over_ranks(ms, world, dev)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    value = replica_value(evals * args.steps, t_max, world)
    info = P.info()
    tim = {k: float(np.mean([s_[k] for s_ in stage])) for k in stage[0]}
    tr_flops = float(sum(P.translation_flops(1, precision=1).values()))
    tr_ms = tim["m2m"] + tim["m2l"] + tim["l2l"]

    # end to end from pinned host buffers through the C ABI (efmm_batch_host)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    htri, hnrm, hcen, htgt = map(pin, (tri, nrm, cen, tgt))
    hssl, hsdl = pin(ssl[None]), pin(sdl[None])
    hout = (pin(np.zeros((1, n, 3))), pin(np.zeros((1, n, 3, 3))), pin(np.zeros((1, m, 3))),
            pin(np.zeros((1, m, 3, 3))))
    ier, *_ = E.batch_host(iprec, 1.0, 1.0, htri, hnrm, hcen, hssl, hsdl, htgt, precision=1, out=hout)
    assert ier == 0, ier
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ier, *_ = E.batch_host(iprec, 1.0, 1.0, htri, hnrm, hcen, hssl, hsdl, htgt, precision=1, out=hout)
        assert ier == 0, ier
    e2e_t = max_over_ranks(time.perf_counter() - t0, world, dev)
    e2e_value = world * evals * args.steps / e2e_t
    h2d = 8 * (9 * n + 3 * n + 3 * n + 3 * m + 6 * n)
    d2h = 8 * (3 * n + 9 * n + 3 * m + 9 * m)

    # the FP64 pass at the same iprec
    u64, e64, ut64, et64 = z(n, 3), z(n, 3, 3), z(m, 3), z(m, 3, 3)
    P.set_geometry(dtri, dnrm, dcen, dtgt, iprec=iprec)
    P.evaluate(1.0, 1.0, dssl, dsdl, u64, e64, ut64, et64)
    P.record(0)
    P.set_geometry(dtri, dnrm, dcen, dtgt, iprec=iprec)
    P.evaluate(1.0, 1.0, dssl, dsdl, u64, e64, ut64, et64)
    P.record(1)
    fp64_ms = P.elapsed(0, 1)

    # errors against the FP64 direct sums: the first ns centroids (on-surface)
    # and the first nk targets (a second plan holding only those targets)
    ns, nk = min(2000, n), min(2000, m)
    ud, ed = z(ns, 3), z(ns, 3, 3)
    P.evaluate_direct_subset(1.0, 1.0, ns, dssl, dsdl, ud, ed)
    Q = E.Plan(local_rank)
    Q.set_geometry(dtri, dnrm, dcen, dtgt[:nk].contiguous(), iprec=iprec)
    utd, etd = z(nk, 3), z(nk, 3, 3)
    Q.evaluate(1.0, 1.0, dssl, dsdl, None, None, utd, etd, direct=True)
    Q.close()
    rel = lambda a, b: float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
    # the oracle's FP64 direct sum at the CPU sample's points (also the timed
    # CPU baseline): errors of every form against it
    cpu, ref = None, None
    if not args.no_cpu_baseline and world == 1:
        ev, dt, cores, npts, ref = cpu_oracle_sample(tri, cen, tgt, ssl, sdl, args.cpu_sample)
        cpu = {"value": ev, "unit": "triangle-evals/s", "cores": cores, "kind": "port",
               "sample": f"oracle direct sum, {npts} evaluation points x {n} triangles ({dt:.1f} s)"}
    errs, oerr = {}, {}
    for ip in w["err_iprecs"]:
        step(ip)
        errs[f"mixed_iprec{ip}"] = {"u": rel(u[0, :ns], ud), "strain": rel(e[0, :ns], ed),
                                    "u_targets": rel(ut[0, :nk], utd), "strain_targets": rel(et[0, :nk], etd),
                                    "order_iprec": P.info()["p"],
                                    "order_mixed": P.set_mixed_floor(0.5e-7)}  # the default floor
        if ref is not None:
            oerr[f"mixed_iprec{ip}"] = oracle_errors(ref, u[0], e[0], ut[0], et[0])
    errs[f"fp64_iprec{iprec}"] = {"u": rel(u64[:ns], ud), "strain": rel(e64[:ns], ed),
                                  "u_targets": rel(ut64[:nk], utd), "strain_targets": rel(et64[:nk], etd)}
    if ref is not None:
        oerr[f"fp64_iprec{iprec}"] = oracle_errors(ref, u64, e64, ut64, et64)
    P.close()
    if rank != 0:
        return None
    achieved = tr_flops / (tr_ms * 1e-3) / 1e12
    peak32 = gemm_peak(torch, dev, torch.float32)
    roof = {"kernel": "translations (k_translate_rot_s, parity-split factored M2M + M2L + L2L, FP32)",
            "bound": "fp32", "achieved": achieved, "peak": peak32, "unit": "TFLOP/s",
            "frac": achieved / peak32 if peak32 else None, "traffic": None,
            "peak_source": "measured cuBLAS SGEMM 8192^3 with TF32 off (best of 5) in this run; the FP32 FMA "
                           "pipe (MEASURED_PEAKS.json has no FP32 entry)",
            "algorithmic": f"{tr_flops:.4g} useful FP32 flop per step (per box pair and column: two Ry of "
                           f"sum_n (n+1)^2 + n^2, the z shift's re / im blocks, two Rz; per-offset orders) in "
                           f"{tr_ms:.1f} ms of translation stages"}
    return {
        "metric": SINGLE_MIXED_METRIC,
        "value": value, "unit": "triangle-evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": args.workload, "triangles": n, "targets": m, "iprec": iprec,
                   "evals_per_step": evals, "parallelism": f"replicas{world}",
                   "l2_policy": "inputs + expansions > L2 (126 MB)",
                   "step": "set_geometry + mixed pass (one right-hand side, single and double layer)",
                   "fp64_ms_per_step": fp64_ms, "fp64_value": evals / (fp64_ms * 1e-3),
                   "rel_err_vs_direct": errs,
                   "rel_err_sample": f"{ns} centroids (on-surface) and {nk} targets",
                   "rel_err_vs_oracle": oerr or None,
                   "rel_err_vs_oracle_sample": "the cpu_baseline sample's centroids and targets (oracle FP64 "
                                               "direct sum)",
                   "stage_ms": tim, "tree": {k: info[k] for k in ("nboxes", "nlev", "p", "nbox")}},
        "e2e": {"value": e2e_value, "unit": "triangle-evals/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "timing": "host wall clock around blocking efmm_batch_host calls (pinned host arrays)"},
        "gpu_launches": launches // max(1, args.steps),
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }


def run_batch(args, rank, world, local_rank):
    """The batched workload: mixed-precision batched form timed as `value`,
    plain FP64 and batched FP64 forms beside it, errors vs the direct sum."""
    import torch
    import elfmmlib3d_b200 as E
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    cols = rank_columns(args.workload, world, rank)
    tri, nrm, cen, sdl, iprec = make_fault(args.workload, cols=cols)
    R, n = sdl.shape[0], len(cen)
    evals = n * n * R

    def d(a):
        return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    dtri, dnrm, dcen, dsdl = map(d, (tri, nrm, cen, sdl))
    u = torch.zeros((R, n, 3), dtype=torch.float64, device=dev)
    e = torch.zeros((R, n, 3, 3), dtype=torch.float64, device=dev)
    P = E.Plan(local_rank)

    def step(precision=1):
        P.set_geometry(dtri, dnrm, dcen, None, iprec=iprec)
        P.evaluate_batch(1.0, 1.0, R, None, dsdl, u, e, precision=precision)

    for _ in range(args.warmup):
        step()
    l0 = E.kernel_launches()
    stage = []
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        torch.cuda.nvtx.range_push("timed")  # profiler captures select this range
        P.record(0)
        for _ in range(args.steps):
            step()
            stage.append(P.timings())
        P.record(1)
        ms = P.elapsed(0, 1)
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    launches = E.kernel_launches() - l0
    t_max = max_over_ranks(ms, world, dev)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    value = replica_value(evals * args.steps, t_max, world)
    info = P.info()
    fl = P.flops_per_column()
    setup = P.setup_timings()
    tim = {k: float(np.mean([s_[k] for s_ in stage])) for k in stage[0]}
    u_mixed, e_mixed = u.clone(), e.clone()

    # end to end from pinned host buffers through the C ABI (efmm_batch_host)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    htri, hnrm, hcen, hsdl = map(pin, (tri, nrm, cen, sdl))
    hout = (pin(np.zeros((R, n, 3))), pin(np.zeros((R, n, 3, 3))), pin(np.zeros((R, 1, 3))),
            pin(np.zeros((R, 1, 3, 3))))
    ier, *_ = E.batch_host(iprec, 1.0, 1.0, htri, hnrm, hcen, None, hsdl, precision=1, out=hout)
    assert ier == 0, ier
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ier, *_ = E.batch_host(iprec, 1.0, 1.0, htri, hnrm, hcen, None, hsdl, precision=1, out=hout)
        assert ier == 0, ier
    e2e_s = time.perf_counter() - t0
    e2e_t = max_over_ranks(e2e_s, world, dev)
    e2e_value = world * evals * args.steps / e2e_t
    h2d = 8 * (9 * n + 3 * n + 3 * n + 3 * n * R)
    d2h = 8 * (3 * n * R + 9 * n * R)

    # the other forms, same inputs: plain FP64 = one full evaluation per
    # right-hand side (set_geometry + evaluate each); batched FP64
    u1 = torch.zeros((R, n, 3), dtype=torch.float64, device=dev)
    e1 = torch.zeros((R, n, 3, 3), dtype=torch.float64, device=dev)
    P.set_geometry(dtri, dnrm, dcen, None, iprec=iprec)
    P.evaluate(1.0, 1.0, None, dsdl[0], u1[0], e1[0])
    P.record(0)
    for r in range(R):
        P.set_geometry(dtri, dnrm, dcen, None, iprec=iprec)
        P.evaluate(1.0, 1.0, None, dsdl[r], u1[r], e1[r])
    P.record(1)
    plain_ms = P.elapsed(0, 1)
    step(0)
    P.record(0)
    step(0)
    P.record(1)
    b64_ms = P.elapsed(0, 1)
    u64, e64 = u.clone(), e.clone()
    ns = min(2000, n)
    ud = torch.zeros((ns, 3), dtype=torch.float64, device=dev)
    ed = torch.zeros((ns, 3, 3), dtype=torch.float64, device=dev)
    rel = lambda a, b: float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
    errs = {"plain_fp64": [0.0, 0.0], "batched_fp64": [0.0, 0.0], "mixed_batched": [0.0, 0.0]}
    for r in (0, R - 1):
        P.evaluate_direct_subset(1.0, 1.0, ns, None, dsdl[r], ud, ed)
        for key, (uu, ee) in (("plain_fp64", (u1, e1)), ("batched_fp64", (u64, e64)),
                              ("mixed_batched", (u_mixed, e_mixed))):
            errs[key][0] = max(errs[key][0], rel(uu[r, :ns], ud))
            errs[key][1] = max(errs[key][1], rel(ee[r, :ns], ed))
    if rank != 0:
        return None
    # roofline: the translation kernel (k_translate<float>: M2M + M2L + L2L)
    C = 4 * R
    tr_flops = (fl["m2m"] + fl["m2l"] + fl["l2l"]) * C
    tr_ms = tim["m2m"] + tim["m2l"] + tim["l2l"]
    achieved = tr_flops / (tr_ms * 1e-3) / 1e12
    peak32 = gemm_peak(torch, dev, torch.float32)
    roof = {"kernel": "k_translate_rot_s (parity-split M2M+M2L+L2L, FP32)", "bound": "fp32", "achieved": achieved,
            "peak": peak32, "unit": "TFLOP/s", "frac": achieved / peak32, "traffic": None,
            "peak_source": "measured cuBLAS SGEMM 8192^3 (FP32 pipe, TF32 off) in this run; "
                           "MEASURED_PEAKS.json has no FP32 entry",
            "algorithmic": f"parity-split factored translations (Rz, Ry, shift along z, Ry back, Rz back): "
                           f"{tr_flops:.4g} flop per step over {info['m2l_pairs']} M2L pairs x {C} columns"}
    stage_tf = {k: fl[k] * C / (tim[k] * 1e-3) / 1e12 for k in ("p2m", "m2m", "m2l", "l2l", "l2t") if tim[k] > 0}
    cpu, oerr = None, None
    if not args.no_cpu_baseline and world == 1:
        ev, dt, cores, npts, ref = cpu_oracle_sample(tri, cen, np.zeros((0, 3)), None, sdl[0], args.cpu_sample)
        cpu = {"value": ev, "unit": "triangle-evals/s", "cores": cores, "kind": "port",
               "sample": f"oracle direct sum, {npts} centroids x {n} triangles x 1 right-hand side "
                         f"({dt:.1f} s)"}
        oerr = {k: oracle_errors(ref, uu[0], ee[0]) for k, (uu, ee) in
                (("plain_fp64", (u1, e1)), ("batched_fp64", (u64, e64)), ("mixed_batched", (u_mixed, e_mixed)))}
    plain_value = evals / (plain_ms * 1e-3)
    b64_value = evals / (b64_ms * 1e-3)
    return {
        "metric": "triangle-evals/s at <=1e-6 rel err (mixed-precision batched form; plain FP64 beside it)",
        "value": value, "unit": "triangle-evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": args.workload, "triangles": n, "rhs": R, "targets": 0, "iprec": iprec,
                   "green": "free space", "evals_per_step": evals,
                   "parallelism": (f"rhs-columns{world}: {R * world} right-hand sides on one geometry, columns "
                                   f"{cols[0]}..{cols[1] - 1} on rank {rank}, geometry and plans replicated, no "
                                   "exchange") if world > 1 else "1 GPU",
                   "l2_policy": "expansions (2 x 3.5 GB FP32) and pair data > L2 (126 MB)",
                   "forms": {"mixed_batched": value / world, "batched_fp64": b64_value,
                             "plain_fp64": plain_value, "mixed_over_plain": value / world / plain_value,
                             "plain_fp64_ms": plain_ms, "batched_fp64_ms": b64_ms},
                   "rel_err_vs_direct": {k: {"u": v[0], "strain": v[1]} for k, v in errs.items()},
                   "rel_err_sample": f"{ns} centroids, right-hand sides 0 and {R - 1}",
                   "rel_err_vs_oracle": oerr,
                   "rel_err_vs_oracle_sample": "right-hand side 0 at the cpu_baseline sample's centroids "
                                               "(oracle FP64 direct sum)",
                   "stage_ms": tim, "stage_tflops": stage_tf, "setup_ms": setup,
                   "tree": {k: info[k] for k in ("nboxes", "nlev", "p", "nbox")},
                   "near_pairs": info["near_pairs"], "m2l_pairs": info["m2l_pairs"]},
        "e2e": {"value": e2e_value, "unit": "triangle-evals/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "timing": "host wall clock around blocking efmm_batch_host calls"},
        "gpu_launches": launches,
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }


def run_hsbatch(args, rank, world, local_rank):
    """The half-space batched workload: the direct arrival (free-space plan on
    the centroids) plus the image part (image plan on the reflected
    centroids), both with their near fields stored on the first call of the
    sequence and replayed for every batch of 64 slip vectors; mixed precision
    timed as `value`, the plain FP64 form (one ITER call pair per right-hand
    side) and the batched FP64 form beside it; errors against the direct
    sums (free space + image) on 2,000 centroids."""
    import torch
    import elfmmlib3d_b200 as E
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    cols = rank_columns(args.workload, world, rank)
    tri, nrm, cen, sdl, iprec = make_fault(args.workload, cols=cols)
    R, n = sdl.shape[0], len(cen)
    evals = n * n * R

    def d(a):
        return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    dtri, dnrm, dcen, dsdl = map(d, (tri, nrm, cen, sdl))
    dcenr = d(cen * np.array([1.0, 1.0, -1.0]))
    F, I = E.Plan(local_rank), E.Plan(local_rank)
    F.set_geometry(dtri, dnrm, dcen, None, iprec=iprec, iter=True)
    I.set_geometry(dtri, dnrm, dcen, dcenr, iprec=iprec, iter=True, mindlin=True)
    uf = torch.zeros((R, n, 3), dtype=torch.float64, device=dev)
    ef = torch.zeros((R, n, 3, 3), dtype=torch.float64, device=dev)
    ui, ei = torch.zeros_like(uf), torch.zeros_like(ef)

    def step(precision=1, mode=2, graph=False):
        graph = graph and not args.no_graph
        F.evaluate_batch(1.0, 1.0, R, None, dsdl, uf, ef, precision=precision, mode=mode, graph=graph)
        I.evaluate_image(1.0, 1.0, R, None, dsdl, ui, ei, precision=precision, mode=mode, graph=graph)

    # mixed form's truncation floor: orders for max(eps(iprec), floor), by
    # default the library's 5e-8 (the FP32 rounding of the result)
    mixed_floor = args.mixed_floor
    p_mixed = F.set_mixed_floor(mixed_floor)
    I.set_mixed_floor(mixed_floor)
    t0 = time.perf_counter()
    step(mode=1)  # first call of the sequence: near fields stored
    store_s = time.perf_counter() - t0
    for _ in range(args.warmup):
        step()
    # stage times and the product launches' events come from plain passes
    # (a graph replay has no per-stage events); the timed steps replay the
    # whole pass of each plan as one CUDA graph (captured in the warm-up)
    stages = []
    torch.cuda.synchronize()
    pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pe0.record()
    for _ in range(args.steps):
        step()
        stages.append((F.timings(), I.timings(), F.product_stats(), I.product_stats(), F.near_stats()))
    pe1.record()
    pe1.synchronize()
    nograph_ms = pe0.elapsed_time(pe1) / args.steps
    for _ in range(max(args.warmup, 2)):
        step(graph=True)
    l0 = E.kernel_launches()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        torch.cuda.nvtx.range_push("timed")  # profiler captures select this range
        ev0.record()
        for _ in range(args.steps):
            step(graph=True)
        ev1.record()
        ev1.synchronize()
        torch.cuda.nvtx.range_pop()
    ms = ev0.elapsed_time(ev1)
    launches = E.kernel_launches() - l0
    t_max = max_over_ranks(ms, world, dev)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    value = replica_value(evals * args.steps, t_max, world)
    tf = {k: float(np.mean([s_[0][k] for s_ in stages])) for k in stages[0][0]}
    ti = {k: float(np.mean([s_[1][k] for s_ in stages])) for k in stages[0][1]}
    u_mixed, e_mixed = (uf + ui).clone(), (ef + ei).clone()

    # the mixed form at the iprec orders (no truncation floor), beside the
    # headline: plain passes timed with events
    F.set_mixed_floor(0.0)
    I.set_mixed_floor(0.0)
    for _ in range(2):
        step()
    torch.cuda.synchronize()
    pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pe0.record()
    for _ in range(args.steps):
        step()
    pe1.record()
    pe1.synchronize()
    mixed_iprec_ms = pe0.elapsed_time(pe1) / args.steps
    u_mi, e_mi = (uf + ui).clone(), (ef + ei).clone()
    # and at a coarser floor (5e-7: orders 26 at iprec 3), to show the
    # order / time trade-off; plain passes timed with events
    coarse_floor = 5e-7
    p_coarse = F.set_mixed_floor(coarse_floor)
    I.set_mixed_floor(coarse_floor)
    for _ in range(2):
        step()
    torch.cuda.synchronize()
    pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pe0.record()
    for _ in range(args.steps):
        step()
    pe1.record()
    pe1.synchronize()
    mixed_coarse_ms = pe0.elapsed_time(pe1) / args.steps
    u_mc, e_mc = (uf + ui).clone(), (ef + ei).clone()
    F.set_mixed_floor(mixed_floor)
    I.set_mixed_floor(mixed_floor)

    # plain FP64: one ITER call pair (direct arrival + image) per right-hand side
    u1 = torch.zeros((R, n, 3), dtype=torch.float64, device=dev)
    e1 = torch.zeros((R, n, 3, 3), dtype=torch.float64, device=dev)
    ui1 = torch.zeros((1, n, 3), dtype=torch.float64, device=dev)
    ei1 = torch.zeros((1, n, 3, 3), dtype=torch.float64, device=dev)
    F.evaluate(1.0, 1.0, None, dsdl[0], u1[0], e1[0], mode=2)
    torch.cuda.synchronize()
    pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pe0.record()
    for r in range(R):
        F.evaluate(1.0, 1.0, None, dsdl[r], u1[r], e1[r], mode=2)
        I.evaluate_image(1.0, 1.0, 1, None, dsdl[r:r + 1], ui1, ei1, precision=0, mode=2)
        u1[r] += ui1[0]
        e1[r] += ei1[0]
    pe1.record()
    pe1.synchronize()
    plain_ms = pe0.elapsed_time(pe1)
    be0, be1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step(0)
    be0.record()
    step(0)
    be1.record()
    be1.synchronize()
    b64_ms = be0.elapsed_time(be1)
    u64, e64 = (uf + ui).clone(), (ef + ei).clone()
    # errors against the direct sums (free space + image) on 2,000 centroids
    ns = min(2000, n)
    ud = torch.zeros((ns, 3), dtype=torch.float64, device=dev)
    ed = torch.zeros((ns, 3, 3), dtype=torch.float64, device=dev)
    rel = lambda a, b: float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
    errs = {"plain_fp64": [0.0, 0.0], "batched_fp64": [0.0, 0.0], "mixed_batched": [0.0, 0.0],
            "mixed_batched_iprec_orders": [0.0, 0.0], "mixed_batched_floor_5e-7": [0.0, 0.0]}
    for r in (0, R - 1):
        F.evaluate_direct_subset(1.0, 1.0, ns, None, dsdl[r], ud, ed)
        ier, uid, eid = E.hs_image_direct(1.0, 1.0, tri, nrm, None, sdl[r], cen[:ns])
        assert ier == 0, ier
        udt = ud + torch.from_numpy(uid).to(dev)
        edt = ed + torch.from_numpy(eid).to(dev)
        for key, (uu, ee) in (("plain_fp64", (u1, e1)), ("batched_fp64", (u64, e64)),
                              ("mixed_batched", (u_mixed, e_mixed)),
                              ("mixed_batched_iprec_orders", (u_mi, e_mi)),
                              ("mixed_batched_floor_5e-7", (u_mc, e_mc))):
            errs[key][0] = max(errs[key][0], rel(uu[r, :ns], udt))
            errs[key][1] = max(errs[key][1], rel(ee[r, :ns], edt))
    trf = F.translation_flops(R, 1)
    tri_ = I.translation_flops(R, 1)
    fi, ii = F.info(), I.info()
    stored = {"free": F.stored_bytes(), "image": I.stored_bytes()}
    F.close()  # the C-ABI call below holds its own plans and stores
    I.close()
    del uf, ef, ui, ei
    torch.cuda.empty_cache()

    # end to end through the C ABI (elhfmm3dtria_batch_host): the 64 slip
    # vectors from pinned host memory, both plans' passes (stored near
    # fields replayed, each pass one CUDA graph), the total displacement and
    # strain back to pinned host memory, every step; the store call
    # (icomp_type 2) and one replay before the timed calls are untimed
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    htri, hnrm, hcen, hsdl = map(pin, (tri, nrm, cen, sdl))
    hout = (pin(np.zeros((R, n, 3))), pin(np.zeros((R, n, 3, 3))))
    ws = np.zeros(8)
    t0 = time.perf_counter()
    ier, _, _ = E.hs_batch_host(iprec, 1.0, 1.0, htri, hnrm, hcen, None, hsdl, precision=1, icomp_type=2,
                                wsave=ws, out=hout)
    assert ier == 0, ier
    e2e_store_s = time.perf_counter() - t0
    ier, _, _ = E.hs_batch_host(iprec, 1.0, 1.0, htri, hnrm, hcen, None, hsdl, precision=1, icomp_type=3,
                                wsave=ws, out=hout)
    assert ier == 0, ier
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ier, _, _ = E.hs_batch_host(iprec, 1.0, 1.0, htri, hnrm, hcen, None, hsdl, precision=1, icomp_type=3,
                                    wsave=ws, out=hout)
        assert ier == 0, ier
    e2e_s = time.perf_counter() - t0
    E.iter_release(ws)
    e2e_t = max_over_ranks(e2e_s, world, dev)
    e2e_value = world * evals * args.steps / e2e_t
    h2d = 8 * 3 * n * R
    d2h = 8 * (3 * n * R + 9 * n * R)
    e2e_vs_value = {"u": rel(torch.from_numpy(hout[0]).to(dev), u_mixed),
                    "strain": rel(torch.from_numpy(hout[1]).to(dev), e_mixed)}
    if rank != 0:
        return None
    # roofline: the P2M products of both plans (k_gemm_tc, the largest
    # kernel), timed with CUDA events around each product launch on the
    # plans' streams; useful FP32 flops from the product shapes, tensor-pipe
    # flops = 3 x useful (the head/tail split issues three TF32 MMAs)
    prod_ms = float(np.mean([s_[2][0] + s_[3][0] for s_ in stages]))
    prod_flops = float(np.mean([s_[2][1] + s_[3][1] for s_ in stages]))
    useful = prod_flops / (prod_ms * 1e-3) / 1e12
    achieved = 3.0 * useful
    # MEASURED_PEAKS.json has no TF32 entry: the dense TF32 tensor rate is
    # measured here with cuBLAS, the same method (8192^3, best of 10)
    peak = tf32_peak(torch, dev)
    peak_source = "measured cuBLAS TF32 GEMM 8192^3 (best of 10) in this run; MEASURED_PEAKS.json has no TF32 entry"
    try:
        bf16 = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("bf16_tflops")
        peak_source += f" (its bf16_tflops is {bf16})"
    except (OSError, ValueError, TypeError):
        pass
    roof_tc = {"kernel": "k_tc_bulk<64, float> (P2M products: split unit multipoles x split densities streamed "
                         "by bulk copies, tcgen05.mma kind::tf32, free-space and image plans)",
               "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
               "frac": (achieved / peak) if peak else None, "traffic": None, "peak_source": peak_source,
               "useful_fp32_tflops": useful,
               "algorithmic": f"{prod_flops:.4g} useful FP32 flop per step (unit multipoles x densities) in "
                              f"{prod_ms:.1f} ms of product launches; 3 TF32 MMAs per FP32 product"}
    # the stored free-space near field's product (k_tc_bulk<64, double>):
    # the split store (TF32 head + tail per element), the split densities and
    # the FP64 products it writes, against the measured HBM copy rate
    nms = float(np.mean([s_[4][0] for s_ in stages]))
    nbytes = float(np.mean([s_[4][1] for s_ in stages]))
    roof_near = None
    if nms > 0 and nbytes > 0:
        try:
            hbm = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs")
        except (OSError, ValueError):
            hbm = None
        nach = nbytes / (nms * 1e-3) / 1e9
        roof_near = {"kernel": "k_tc_bulk<64, double> (replay of the stored free-space near field from its split: "
                               "pre-split tiles streamed by bulk copies into the tensor cores, FP64 K-tile sums)",
                     "bound": "hbm", "achieved": nach, "peak": hbm, "unit": "GB/s",
                     "frac": nach / hbm if hbm else None, "traffic": None,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if hbm else "MEASURED_PEAKS.json absent",
                     "algorithmic": f"{nbytes:.4g} bytes per replay (split store 8 bytes per stored element, split "
                                    f"densities, FP64 products) in {nms:.2f} ms (CUDA events around the launch)"}
    # the dominant kernels of the step (ncu launch shares): the factored
    # translations in the parity-split form (k_translate_rot_s, FP32 FMA
    # pipe), useful flops per pair and column, time = the M2M + M2L + L2L
    # stage events of both plans, against the measured SGEMM rate
    tr_flops = sum(trf.values()) + sum(tri_.values())
    tr_ms = float(np.mean([sum(s_[0][k] + s_[1][k] for k in ("m2m", "m2l", "l2l")) for s_ in stages]))
    peak32 = gemm_peak(torch, dev, torch.float32)
    tr_ach = tr_flops / (tr_ms * 1e-3) / 1e12
    roof = {"kernel": "k_translate_rot_s (parity-split factored M2M / M2L / L2L: Rz, the re / im blocks of "
                      "Ry and of the z shift, Ry back, Rz back; paired FP32 FMAs, both plans; the largest share "
                      "of the step's launch time) with the image U-kernel M2L (k_translate_us, parity split)",
            "bound": "fp32", "achieved": tr_ach, "peak": peak32, "unit": "TFLOP/s",
            "frac": tr_ach / peak32 if peak32 else None, "traffic": None,
            "peak_source": "measured cuBLAS SGEMM 8192^3 with TF32 off (best of 5) in this run; the FP32 FMA "
                           "pipe (MEASURED_PEAKS.json has no FP32 entry)",
            "algorithmic": f"{tr_flops:.4g} useful FP32 flop per step (per box pair and column: two Ry of "
                           f"sum_n (n+1)^2 + n^2, the z shift's re / im blocks, two Rz; the U-kernel M2L's re / "
                           f"im blocks; per-offset orders) in {tr_ms:.1f} ms of translation stages",
            "flops_by_stage": {"free": trf, "image": tri_}}
    cpu, oerr = None, None
    if not args.no_cpu_baseline and world == 1:
        ev, dt, cores, npts, ref = cpu_oracle_hs_sample(tri, nrm, cen, None, sdl[0], args.cpu_sample)
        cpu = {"value": ev, "unit": "triangle-evals/s", "cores": cores, "kind": "port",
               "sample": f"oracle half-space self-evaluation (free-space direct sum + image quadrature with "
                         f"distance refinement), {npts} centroids x {n} triangles x 1 right-hand side "
                         f"({dt:.1f} s)"}
        oerr = {k: oracle_errors(ref, uu[0], ee[0]) for k, (uu, ee) in
                (("plain_fp64", (u1, e1)), ("batched_fp64", (u64, e64)), ("mixed_batched", (u_mixed, e_mixed)),
                 ("mixed_batched_iprec_orders", (u_mi, e_mi)))}
        oerr["e2e_c_abi"] = oracle_errors(ref, hout[0][0], hout[1][0])
    plain_value = evals / (plain_ms * 1e-3)
    b64_value = evals / (b64_ms * 1e-3)
    return {
        "metric": "triangle-evals/s at <=1e-6 rel err (mixed-precision batched form; plain FP64 beside it)",
        "value": value, "unit": "triangle-evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": args.workload, "triangles": n, "rhs": R, "targets": "centroids", "iprec": iprec,
                   "green": "Mindlin half space (free space + image)", "evals_per_step": evals,
                   "parallelism": (f"rhs-columns{world}: {R * world} right-hand sides on one geometry, columns "
                                   f"{cols[0]}..{cols[1] - 1} on rank {rank}, geometry, plans and stored near "
                                   "fields replicated, no exchange") if world > 1 else "1 GPU",
                   "l2_policy": "expansions (FP32, several GB) and stored near field (~49 GB) > L2 (126 MB)",
                   "step": "free-space batch + image batch, near fields replayed (stored on the first call, "
                           f"{store_s * 1e3:.0f} ms, untimed), "
                           + ("plain passes (--no-graph)" if args.no_graph else
                              "each plan's pass replayed as one CUDA graph"),
                   "ms_per_step_without_graph": nograph_ms,
                   "forms": {"mixed_batched": value / world, "batched_fp64": b64_value,
                             "plain_fp64": plain_value, "mixed_over_plain": value / world / plain_value,
                             "plain_fp64_ms": plain_ms, "batched_fp64_ms": b64_ms,
                             "mixed_batched_iprec_orders": evals / (mixed_iprec_ms * 1e-3),
                             "mixed_iprec_orders_ms": mixed_iprec_ms,
                             "mixed_batched_floor_5e-7": evals / (mixed_coarse_ms * 1e-3),
                             "mixed_floor_5e-7_ms": mixed_coarse_ms, "mixed_floor_5e-7_order": p_coarse},
                   "orders": {"iprec": fi["p"], "mixed": p_mixed, "mixed_floor": mixed_floor,
                              "rule": "mixed form: expansions and translations truncated at max(eps(iprec), "
                                      "floor), by default the library's floor 5e-8 (the FP32 rounding of the "
                                      "result); plain and batched FP64 forms at eps(iprec); the forms at the "
                                      "iprec orders and at the floor 5e-7 are timed beside it (plain passes)"},
                   "rel_err_vs_direct": {k: {"u": v[0], "strain": v[1]} for k, v in errs.items()},
                   "rel_err_sample": f"{ns} centroids, right-hand sides 0 and {R - 1}",
                   "rel_err_vs_oracle": oerr,
                   "rel_err_vs_oracle_sample": "right-hand side 0 at the cpu_baseline sample's centroids (oracle "
                                               "FP64 free-space direct sum + image quadrature)",
                   "stage_ms_free": tf, "stage_ms_image": ti,
                   "tree_free": {k: fi[k] for k in ("nboxes", "nlev", "p", "nbox")},
                   "tree_image": {k: ii[k] for k in ("nboxes", "nlev", "p", "nbox")},
                   "stored_bytes": stored,
                   "tuner": {"lines": E.tune_dump(),
                             "format": "knob (0 M2M, 1 M2L, 2 L2L) p nbox C prec kind (0 free, 1 image) decided "
                                       "(0 tensor cores, 1 CUDA cores) ms_tensor ms_cuda"}},
        "e2e": {"value": e2e_value, "unit": "triangle-evals/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "timing": "host wall clock around blocking elhfmm3dtria_batch_host calls (icomp_type 3: pinned "
                          "slip vectors to the device, both plans' stored-near-field passes as CUDA graphs, the "
                          "total displacement + strain back to pinned host memory)",
                "store_call_s": e2e_store_s, "outputs_vs_value_step": e2e_vs_value},
        "gpu_launches": launches,
        "roofline": roof,
        "roofline_tc": roof_tc,
        "roofline_near": roof_near,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }


def run_iter(args, rank, world, local_rank):
    """The ITER workload: store on the first call, reuse on the others."""
    import torch
    import elfmmlib3d_b200 as E
    from elfmmlib3d_b200 import geometry as G
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    w = WORKLOADS[args.workload]
    L, Wd, depth, dip = 40.0, 20.0, 1.0, 45.0
    tri, nrm, cen, us = G.planar_fault(w["nl"], w["nw"], L, Wd, dip, depth)
    n, ncall, iprec = len(cen), w["calls"], w["iprec"]
    slips = [G.tapered_slip(cen, us, L, Wd, depth, dip, 0.05, seed=100 * (rank + 1) + c) for c in range(ncall)]
    evals = n * n * ncall

    def d(a):
        return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    dtri, dnrm, dcen = map(d, (tri, nrm, cen))
    dsl = [d(x) for x in slips]
    u = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    e = torch.zeros((n, 3, 3), dtype=torch.float64, device=dev)
    P = E.Plan(local_rank)

    def sequence(calls):
        P.set_geometry(dtri, dnrm, dcen, None, iprec=iprec, iter=True)
        P.evaluate(1.0, 1.0, None, dsl[0], u, e, mode=1)
        for c in range(1, calls):
            P.evaluate(1.0, 1.0, None, dsl[c], u, e, mode=2)

    sequence(max(args.warmup, 2))
    replay_ms = []
    l0 = E.kernel_launches()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        torch.cuda.nvtx.range_push("timed")
        P.record(0)
        P.set_geometry(dtri, dnrm, dcen, None, iprec=iprec, iter=True)
        P.evaluate(1.0, 1.0, None, dsl[0], u, e, mode=1)
        store_tim = P.timings()
        for c in range(1, ncall):
            P.evaluate(1.0, 1.0, None, dsl[c], u, e, mode=2)
            replay_ms.append(P.timings())
        P.record(1)
        ms = P.elapsed(0, 1)
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    launches = E.kernel_launches() - l0
    t_max = max_over_ranks(ms, world, dev)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    value = replica_value(evals, t_max, world)
    info = P.info()
    stored = P.stored_bytes()
    u_last, e_last = u.clone(), e.clone()
    # error of the last call against the FP64 direct sum on 2,000 centroids
    ns = min(2000, n)
    ud = torch.zeros((ns, 3), dtype=torch.float64, device=dev)
    ed = torch.zeros((ns, 3, 3), dtype=torch.float64, device=dev)
    P.evaluate_direct_subset(1.0, 1.0, ns, None, dsl[ncall - 1], ud, ed)
    rel = lambda a, b: float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
    err = {"u": rel(u_last[:ns], ud), "strain": rel(e[:ns], ed)}
    # plain form: full calls (tree + analytic near field), two of them timed
    P.record(2)
    for c in range(2):
        P.set_geometry(dtri, dnrm, dcen, None, iprec=iprec)
        P.evaluate(1.0, 1.0, None, dsl[c], u, e)
    P.record(3)
    plain_call_ms = P.elapsed(2, 3) / 2
    # end to end: the reference's ITER entry from host arrays (store, then reuse)
    ws = np.zeros(8)
    hs = [torch.from_numpy(np.ascontiguousarray(x)).pin_memory().numpy() for x in slips]
    htri, hnrm, hcen = (torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy() for a in (tri, nrm, cen))
    t0 = time.perf_counter()
    ier, *_ = E.elfmm3dtriaiter(iprec, 1.0, 1.0, htri, hnrm, hcen, None, hs[0], icomp_type=2, wsave=ws)
    assert ier == 0, ier
    for c in range(1, ncall):
        ier, *_ = E.elfmm3dtriaiter(iprec, 1.0, 1.0, htri, hnrm, hcen, None, hs[c], icomp_type=3, wsave=ws)
        assert ier == 0, ier
    e2e_s = time.perf_counter() - t0
    E.iter_release(ws)
    if rank != 0:
        return None
    rep_near = float(np.mean([t["near"] for t in replay_ms]))
    rep_tot = float(np.mean([t["total"] for t in replay_ms]))
    gbs = stored / (rep_near * 1e-3) / 1e9
    peak = None
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs")
    except (OSError, ValueError):
        pass
    roof = {"kernel": "k_near_replay", "bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
            "frac": (gbs / peak) if peak else None, "traffic": None,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peak else "MEASURED_PEAKS.json absent",
            "algorithmic": f"stored near field read once per call: {stored / 1e9:.2f} GB"}
    cpu, oerr = None, None
    if not args.no_cpu_baseline and world == 1:
        ev, dt, cores, npts, ref = cpu_oracle_sample(tri, cen, np.zeros((0, 3)), None, slips[ncall - 1],
                                                     args.cpu_sample)
        cpu = {"value": ev, "unit": "triangle-evals/s", "cores": cores, "kind": "port",
               "sample": f"oracle direct sum, {npts} centroids x {n} triangles ({dt:.1f} s)"}
        oerr = oracle_errors(ref, u_last, e_last)
    return {
        "metric": "triangle-evals/s over the ITER call sequence (store once, reuse)",
        "value": value, "unit": "triangle-evals/s", "n_gpus": world, "steps": ncall, "warmup": max(args.warmup, 2),
        "ms_per_step": t_max / ncall, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "triangles": n, "calls": ncall, "iprec": iprec, "green": "free space",
                   "evals_per_sequence": evals, "parallelism": f"replicas{world}",
                   "l2_policy": f"stored near field {stored / 1e9:.1f} GB > L2 (126 MB)",
                   "first_call_ms": store_tim["total"], "replay_call_ms": rep_tot, "replay_near_ms": rep_near,
                   "plain_call_ms": plain_call_ms, "sequence_over_plain": plain_call_ms * ncall / t_max,
                   "rel_err_vs_direct_last_call": err, "stored_bytes": stored,
                   "rel_err_vs_oracle_last_call": oerr,
                   "rel_err_vs_oracle_sample": "the cpu_baseline sample's centroids (oracle FP64 direct sum)",
                   "tree": {k: info[k] for k in ("nboxes", "nlev", "p", "nbox")}, "near_pairs": info["near_pairs"]},
        "e2e": {"value": world * evals / e2e_s, "unit": "triangle-evals/s",
                "h2d_bytes_per_step": 8 * (9 * n + 3 * n + 3 * n + 3 * n), "d2h_bytes_per_step": 8 * (3 * n + 9 * n),
                "timing": "host wall clock around the elfmm3dtriaiter_ sequence (icomp 2, then 3)"},
        "gpu_launches": launches,
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }


def run_hsiter(args, rank, world, local_rank):
    """The half-space ITER call sequence: each call = the direct arrival
    (free-space plan, ITER) + the image part (image plan, ITER), the first
    call building both trees and storing both near fields, the other nine
    reusing them with new slip."""
    import torch
    import elfmmlib3d_b200 as E
    from elfmmlib3d_b200 import geometry as G
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    w = WORKLOADS[args.workload]
    L, Wd, depth, dip = 40.0, 20.0, 1.0, 45.0
    tri, nrm, cen, us = G.planar_fault(w["nl"], w["nw"], L, Wd, dip, depth)
    n, ncall, iprec = len(cen), w["calls"], w["iprec"]
    slips = [G.tapered_slip(cen, us, L, Wd, depth, dip, 0.05, seed=100 * (rank + 1) + c) for c in range(ncall)]
    evals = n * n * ncall

    def d(a):
        return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    dtri, dnrm, dcen = map(d, (tri, nrm, cen))
    dcenr = d(cen * np.array([1.0, 1.0, -1.0]))
    dsl = [d(x)[None] for x in slips]
    u = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    e = torch.zeros((n, 3, 3), dtype=torch.float64, device=dev)
    ui = torch.zeros((1, n, 3), dtype=torch.float64, device=dev)
    ei = torch.zeros((1, n, 3, 3), dtype=torch.float64, device=dev)
    F, I = E.Plan(local_rank), E.Plan(local_rank)

    def call(c, mode):
        if mode == 1:
            F.set_geometry(dtri, dnrm, dcen, None, iprec=iprec, iter=True)
            I.set_geometry(dtri, dnrm, dcen, dcenr, iprec=iprec, iter=True, mindlin=True)
        F.evaluate(1.0, 1.0, None, dsl[c][0], u, e, mode=mode)
        I.evaluate_image(1.0, 1.0, 1, None, dsl[c], ui, ei, precision=0, mode=mode)

    for _ in range(max(args.warmup, 2)):
        call(0, 1)
        call(1, 2)
    l0 = E.kernel_launches()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    rep = []
    with ClockSampler(local_rank) as clk:
        torch.cuda.nvtx.range_push("timed")
        ev0.record()
        t0 = time.perf_counter()
        call(0, 1)
        first_s = time.perf_counter() - t0
        for c in range(1, ncall):
            call(c, 2)
            rep.append((F.timings()["total"], I.timings()["total"], F.timings()["near"]))
        ev1.record()
        ev1.synchronize()
        torch.cuda.nvtx.range_pop()
    ms = ev0.elapsed_time(ev1)
    launches = E.kernel_launches() - l0
    t_max = max_over_ranks(ms, world, dev)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    value = replica_value(evals, t_max, world)
    stored = (F.stored_bytes(), I.stored_bytes())
    ut, et = (u + ui[0]).clone(), (e + ei[0]).clone()
    ns = min(2000, n)
    ud = torch.zeros((ns, 3), dtype=torch.float64, device=dev)
    ed = torch.zeros((ns, 3, 3), dtype=torch.float64, device=dev)
    F.evaluate_direct_subset(1.0, 1.0, ns, None, dsl[ncall - 1][0], ud, ed)
    ier, uid, eid = E.hs_image_direct(1.0, 1.0, tri, nrm, None, slips[ncall - 1], cen[:ns])
    assert ier == 0, ier
    rel = lambda a, b: float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
    err = {"u": rel(ut[:ns], ud + torch.from_numpy(uid).to(dev)),
           "strain": rel(et[:ns], ed + torch.from_numpy(eid).to(dev))}
    # plain form: full calls (trees, analytic / refined near fields), two of them timed
    pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pe0.record()
    for c in range(2):
        F.set_geometry(dtri, dnrm, dcen, None, iprec=iprec)
        I.set_geometry(dtri, dnrm, dcen, dcenr, iprec=iprec, mindlin=True)
        F.evaluate(1.0, 1.0, None, dsl[c][0], u, e)
        I.evaluate_image(1.0, 1.0, 1, None, dsl[c], ui, ei, precision=0, mode=0)
    pe1.record()
    pe1.synchronize()
    plain_call_ms = pe0.elapsed_time(pe1) / 2
    F.close()  # the library's ITER slots below hold their own stores
    I.close()
    # end to end: the reference's ITER entries from host arrays (store, then reuse)
    wf, wi = np.zeros(8), np.zeros(8)
    hs = [torch.from_numpy(np.ascontiguousarray(x)).pin_memory().numpy() for x in slips]
    htri, hnrm, hcen = (torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy() for a in (tri, nrm, cen))
    t0 = time.perf_counter()
    for c in range(ncall):
        ic = 2 if c == 0 else 3
        ier, *_ = E.elfmm3dtriaiter(iprec, 1.0, 1.0, htri, hnrm, hcen, None, hs[c], icomp_type=ic, wsave=wf)
        assert ier == 0, ier
        ier, *_ = E.elhfmm3dtriatargiter(iprec, 1.0, 1.0, htri, hnrm, hcen, None, hs[c], target=hcen,
                                         icomp_type=ic, wsave=wi)
        assert ier == 0, ier
    e2e_s = time.perf_counter() - t0
    E.iter_release(wf)
    E.iter_release(wi)
    if rank != 0:
        return None
    rep_f = float(np.mean([r[0] for r in rep]))
    rep_i = float(np.mean([r[1] for r in rep]))
    rep_near = float(np.mean([r[2] for r in rep]))
    gbs = stored[0] / (rep_near * 1e-3) / 1e9
    peak = None
    try:
        peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs")
    except (OSError, ValueError):
        pass
    roof = {"kernel": "k_near_replay (free-space stored near field)", "bound": "hbm", "achieved": gbs, "peak": peak,
            "unit": "GB/s", "frac": (gbs / peak) if peak else None, "traffic": None,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peak else "MEASURED_PEAKS.json absent",
            "algorithmic": f"stored near field read once per call: {stored[0] / 1e9:.2f} GB"}
    cpu, oerr = None, None
    if not args.no_cpu_baseline and world == 1:
        ev, dt, cores, npts, ref = cpu_oracle_hs_sample(tri, nrm, cen, None, slips[ncall - 1], args.cpu_sample)
        cpu = {"value": ev, "unit": "triangle-evals/s", "cores": cores, "kind": "port",
               "sample": f"oracle half-space self-evaluation (free-space direct sum + image quadrature with "
                         f"distance refinement), {npts} centroids x {n} triangles ({dt:.1f} s)"}
        oerr = oracle_errors(ref, ut, et)
    return {
        "metric": "triangle-evals/s over the ITER call sequence (store once, reuse)",
        "value": value, "unit": "triangle-evals/s", "n_gpus": world, "steps": ncall, "warmup": max(args.warmup, 2),
        "ms_per_step": t_max / ncall, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "triangles": n, "calls": ncall, "iprec": iprec,
                   "green": "Mindlin half space (free space + image)", "evals_per_sequence": evals,
                   "parallelism": f"replicas{world}",
                   "l2_policy": f"stored near fields {sum(stored) / 1e9:.1f} GB > L2 (126 MB)",
                   "first_call_s": first_s, "replay_call_ms": {"free": rep_f, "image": rep_i},
                   "rel_err_vs_oracle_last_call": oerr,
                   "rel_err_vs_oracle_sample": "the cpu_baseline sample's centroids (oracle FP64 free-space direct "
                                               "sum + image quadrature)",
                   "plain_call_ms": plain_call_ms, "sequence_over_plain": plain_call_ms * ncall / t_max,
                   "rel_err_vs_direct_last_call": err, "stored_bytes": {"free": stored[0], "image": stored[1]}},
        "e2e": {"value": world * evals / e2e_s, "unit": "triangle-evals/s",
                "h2d_bytes_per_step": 8 * (9 * n + 3 * n + 3 * n + 3 * n) * 2,
                "d2h_bytes_per_step": 8 * (3 * n + 9 * n) * 2,
                "timing": "host wall clock around elfmm3dtriaiter_ + elhfmm3dtriatargiter_ per call (icomp 2, then 3)"},
        "gpu_launches": launches,
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }


def run_reference(args, rank):
    """The reference arm: the oracle's CPU restatement of the reference's
    path on all host cores, each step a bounded sample of the workload
    (ref_sample evaluation points against all triangles).  Half-space
    workloads time the direct arrival plus the image part."""
    if rank != 0:
        return None
    w = WORKLOADS[args.workload]
    kind = w["kind"]
    batch = kind in ("batch", "hsbatch")
    hs = kind in ("hsbatch", "hsiter", "uneven")
    if kind == "uneven":
        probs = make_uneven_problems(w)
        n = int(sum(len(p[2]) for p in probs))
        cfg = {"problems": len(probs), "triangles_total": n, "iprec": w["iprec"]}
        sample = lambda: cpu_oracle_uneven_sample(probs, args.ref_sample)
        desc = (f"oracle half-space self-evaluation (free-space direct sum + image quadrature with distance "
                f"refinement) at {args.ref_sample} centroids of each of {len(uneven_sample_problems(probs))} "
                f"evenly spaced problems, against all of their problem's triangles, per step")
        metric = "triangle-evals/s (batched uneven half-space geometries, mixed precision)"
    else:
        tri, nrm, cen, tgt, ssl, sdl, iprec = make_inputs(args.workload)
        n = len(cen)
        cfg = {"triangles": n, "targets": len(tgt), "iprec": iprec}
        if batch:
            cfg.update({"rhs": w["nrhs"], "green": "Mindlin half space" if hs else "free space"})
        if hs:
            sample = lambda: cpu_oracle_hs_sample(tri, nrm, cen, ssl, sdl, args.ref_sample)
            desc = (f"oracle half-space self-evaluation (free-space direct sum + image quadrature with "
                    f"distance refinement), {args.ref_sample} centroids x {n} triangles per step")
        else:
            sample = lambda: cpu_oracle_sample(tri, cen, tgt, ssl, sdl, args.ref_sample)
            desc = (f"oracle direct sum (el3dtriadirecttarg restated), {args.ref_sample} evaluation points x "
                    f"{n} triangles per step")
        if batch:
            metric = "triangle-evals/s at <=1e-6 rel err (mixed-precision batched form; plain FP64 beside it)"
        elif kind in ("iter", "hsiter"):
            metric = "triangle-evals/s over the ITER call sequence (store once, reuse)"
        elif kind == "single_mixed":
            metric = SINGLE_MIXED_METRIC
        else:
            metric = "triangle-evals/s (free-space SLP+DLP displacement+strain, FP64 FMM at iprec 2)"
    for _ in range(args.warmup):
        sample()
    evs, secs = 0.0, 0.0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ev, dt, cores, npts = sample()[:4]
        evs += ev * dt
        secs += dt
    tot = time.perf_counter() - t0
    value = evs / secs
    return {
        "impl": "reference",
        "metric": metric,
        "value": value, "unit": "triangle-evals/s", "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, **cfg},
        "cpu_baseline": {"value": value, "unit": "triangle-evals/s", "cores": host_threads(), "kind": "port",
                         "sample": desc},
        "e2e": {"value": value, "unit": "triangle-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_uneven(args, rank, world, local_rank):
    """Batched uneven geometries: nprob independent half-space faults (strike
    U[0, 360), dip U[15, 90], top depth U[0.5, 5] degrees / units, triangle
    count log-uniform in [nmin, nmax], one slip vector N(0,1) each), each a
    half-space self-evaluation at its centroids (direct arrival + image part)
    in the mixed form.  Engine "forest" (default): all problems in one forest
    (elfmmlib3d_b200.Forest: one free-space and one image plan over every
    problem, each stage one launch over all problems' boxes); "plans": worker
    threads owning a plan pair each (elfmmlib3d_b200.batch.halfspace_many).
    A step = all problems, set-up (trees, lists) included.  value: inputs
    resident on the device, CUDA events around each step; e2e: host arrays
    in and out through elhfmm3dtria_many_host.  Errors of the timed results
    against the FP64 direct sums on 200 centroids of every 8th problem and
    against the oracle on the CPU sample (untimed)."""
    import torch
    import elfmmlib3d_b200 as E
    from elfmmlib3d_b200.batch import halfspace_many, _check
    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    w = WORKLOADS[args.workload]
    probs = make_uneven_problems(w, world, rank)
    sizes = np.array([len(p[2]) for p in probs])
    counts = sizes.astype(np.int32)
    off = np.concatenate([[0], np.cumsum(sizes)])
    evals = float(np.sum(sizes.astype(np.float64) ** 2))
    engine = args.uneven_engine
    workers = args.uneven_workers or max(4, min(16, host_threads()))
    h_tri = np.ascontiguousarray(np.concatenate([p[0].reshape(-1, 9) for p in probs]))
    h_nrm = np.ascontiguousarray(np.concatenate([p[1] for p in probs]))
    h_cen = np.ascontiguousarray(np.concatenate([p[2] for p in probs]))
    h_sdl = np.ascontiguousarray(np.concatenate([p[4] for p in probs]))
    d = lambda a: torch.tensor(a, dtype=torch.float64, device=dev)
    tri, nrm, cen, sdl = d(h_tri), d(h_nrm), d(h_cen), d(h_sdl)
    u = torch.zeros((len(h_cen), 3), dtype=torch.float64, device=dev)
    e = torch.zeros((len(h_cen), 3, 3), dtype=torch.float64, device=dev)
    F = E.Forest(local_rank) if engine == "forest" else None
    if F is not None:
        F.set_leaf(args.free_leaf, args.image_leaf)
        F.set_mixed_floor(args.mixed_floor)

    split = {}

    def step():
        if F is not None:
            t0 = time.perf_counter()
            F.set_geometry(counts, tri, nrm, cen, iprec=w["iprec"])
            t1 = time.perf_counter()
            F.evaluate(1.0, 1.0, None, sdl, u, e, precision=1)
            split.update(set_geometry_ms=(t1 - t0) * 1e3, evaluate_ms=(time.perf_counter() - t1) * 1e3)
        else:
            res, _ = halfspace_many(probs, iprec=w["iprec"], precision=1, workers=workers, device=local_rank,
                                    engine="plans")
            u.copy_(torch.from_numpy(np.concatenate([r[0] for r in res])))
            e.copy_(torch.from_numpy(np.concatenate([r[1] for r in res])))

    for _ in range(max(1, args.warmup)):
        step()
    torch.cuda.synchronize()
    l0 = E.kernel_launches()
    times = []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            ev0.record()
            step()
            ev1.record()
            torch.cuda.synchronize()
            times.append(ev0.elapsed_time(ev1) * 1e-3)
    launches = E.kernel_launches() - l0
    t = float(np.mean(times))
    t_max = max_over_ranks(t, world, dev)
    value = world * evals / t_max
    stages = None
    if F is not None:
        # device ms of the last step's passes by stage, host ms of its set-up by phase
        stages = {name: {"evaluate": F.plan(k).timings(), "set_up": F.plan(k).setup_timings(),
                         "info": F.plan(k).info()} for k, name in ((0, "free"), (1, "image"))}
        stages["host_ms"] = dict(split)
    uh, eh = u.cpu().numpy(), e.cpu().numpy()
    res = [(uh[off[i]:off[i + 1]], eh[off[i]:off[i + 1]]) for i in range(len(probs))]
    print(f"uneven: {t * 1e3:.1f} ms per step on the device ({evals / t:.3e} triangle-evals/s)", file=sys.stderr)
    if F is not None:
        F.close()  # the host entry point builds its own forest
        F = None
    del tri, nrm, cen, sdl, u, e
    torch.cuda.empty_cache()
    # e2e: host arrays through the C ABI, host wall clock
    e2e_t = []
    if engine == "forest":
        E.set_many_host_mixed_floor(args.mixed_floor)
        for _ in range(args.steps):
            t0 = time.perf_counter()
            ier, uu, ee = E.hs_many_host(w["iprec"], 1.0, 1.0, counts, h_tri, h_nrm, h_cen, None, h_sdl, precision=1)
            e2e_t.append(time.perf_counter() - t0)
            if ier:
                raise E.ElfmmError(ier, "elhfmm3dtria_many_host")
        e2e_err = float(max(np.linalg.norm(uu - uh) / np.linalg.norm(uh), np.linalg.norm(ee - eh) / np.linalg.norm(eh)))
    checked = list(range(0, len(probs), 8))
    errs = np.array([_check(probs[i], *res[i], min(200, int(sizes[i])), 1.0, 1.0, dev) for i in checked])
    e2e_v = world * evals / max_over_ranks(float(np.mean(e2e_t)), world, dev) if e2e_t else value
    if rank != 0:
        return None
    cpu, oerr = None, None
    if not args.no_cpu_baseline and world == 1:
        ev, dt, cores, npts, refs = cpu_oracle_uneven_sample(probs, args.cpu_sample)
        cpu = {"value": ev, "unit": "triangle-evals/s", "cores": cores, "kind": "port",
               "sample": f"oracle half-space self-evaluation (free-space direct sum + image quadrature with "
                         f"distance refinement) at {npts} centroids of {len(uneven_sample_problems(probs))} "
                         f"evenly spaced problems, against all of their problem's triangles ({dt:.1f} s)"}
        # per-problem errors of the timed results against the oracle at those centroids
        sidx = list(range(len(probs)))[::max(1, len(probs) // 16)]
        per = [oracle_errors(ref, res[i][0], res[i][1]) for ref, i in zip(refs, sidx)]
        oerr = {"problems": len(per), "triangles": [int(sizes[i]) for i in sidx],
                "u": [x.get("u") for x in per], "strain": [x.get("strain") for x in per],
                "u_max": max(x.get("u") or 0.0 for x in per), "strain_max": max(x.get("strain") or 0.0 for x in per)}
    forest_step = ("one forest of all problems: the problems moved side by side in x and y, one per column of "
                   "boxes of a common root; set_geometry of its free-space and image plan (trees, lists, "
                   "work lists), the mixed pass of each over all problems' boxes (one right-hand side)")
    plans_step = ("every problem: set_geometry of a free-space and an image plan, the mixed batch pass of each "
                  "(one right-hand side), results to host; worker threads over one queue (largest first)")
    return {
        "metric": "triangle-evals/s (batched uneven half-space geometries, mixed precision)",
        "value": value, "unit": "triangle-evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": args.workload, "problems": len(probs), "triangles_total": int(sizes.sum()),
                   "triangles_min_median_max": [int(sizes.min()), int(np.median(sizes)), int(sizes.max())],
                   "evals_per_step": evals, "iprec": w["iprec"], "engine": engine,
                   "leaf_capacity": {"free": args.free_leaf or "iprec table", "image": args.image_leaf or "half the iprec table"},
                   "workers": workers if engine == "plans" else None,
                   "step": forest_step if engine == "forest" else plans_step,
                   "l2": "inputs (geometry > 300 MB) larger than L2",
                   "stage_ms": stages,
                   "rel_err_vs_direct": {"problems_checked": len(checked), "centroids_each": 200,
                                         "u_max": float(errs[:, 0].max()),
                                         "u_median": float(np.median(errs[:, 0])),
                                         "strain_max": float(errs[:, 1].max()),
                                         "strain_median": float(np.median(errs[:, 1]))},
                   "rel_err_vs_oracle": oerr,
                   "rel_err_vs_oracle_sample": "per sampled problem, the cpu_baseline sample's centroids",
                   "parallelism": (f"problems{world}: {w['nprob']} x {world} problems, greedy n^2 balance "
                                   "across ranks, no exchange") if world > 1 else "1 GPU"},
        "e2e": {"value": e2e_v, "unit": "triangle-evals/s", "h2d_bytes_per_step": int(sizes.sum() * 8 * (9 + 3 + 3 + 3)),
                "d2h_bytes_per_step": int(sizes.sum() * 8 * 12),
                "timing": ("host wall clock around elhfmm3dtria_many_host: geometry and slip vectors from host "
                           f"memory, results back (max relative difference from the device-resident step "
                           f"{e2e_err:.1e})") if e2e_t else "the device-resident step (plans engine copies "
                           "every problem from the host already)"},
        "gpu_launches": launches // max(1, args.steps),
        "roofline": None,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="hs-fault-100k-r64", choices=list(WORKLOADS))
    # CPU samples: one evaluation point per host thread by default, so that
    # every core has work (the oracle shares the points among its threads)
    ncpu = min(256, max(8, host_threads()))
    ap.add_argument("--cpu-sample", type=int, default=ncpu)
    ap.add_argument("--ref-sample", type=int, default=ncpu)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--uneven-engine", default="forest", choices=["forest", "plans"],
                    help="uneven batch: one forest of all problems, or worker threads over per-problem plans")
    ap.add_argument("--free-leaf", type=int, default=0,
                    help="uneven forest: leaf capacity of the free-space plan (0: the iprec table)")
    ap.add_argument("--image-leaf", type=int, default=0,
                    help="uneven forest: leaf capacity of the image plan (0: half the iprec table)")
    ap.add_argument("--uneven-workers", type=int, default=0,
                    help="uneven batch: host worker threads (default: the host threads, 4 to 16)")
    ap.add_argument("--mixed-floor", type=float, default=5e-8,
                    help="half-space workloads: tolerance floor of the mixed form's expansion orders (default: "
                         "the library's, 5e-8, the FP32 rounding of the result)")
    ap.add_argument("--no-graph", action="store_true",
                    help="half-space batch: time plain passes instead of CUDA-graph replays (profiling)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank)
    else:
        if world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        if WORKLOADS[args.workload]["kind"] == "batch":
            out = run_batch(args, rank, world, local_rank)
        elif WORKLOADS[args.workload]["kind"] == "hsbatch":
            out = run_hsbatch(args, rank, world, local_rank)
        elif WORKLOADS[args.workload]["kind"] == "iter":
            out = run_iter(args, rank, world, local_rank)
        elif WORKLOADS[args.workload]["kind"] == "hsiter":
            out = run_hsiter(args, rank, world, local_rank)
        elif WORKLOADS[args.workload]["kind"] == "uneven":
            out = run_uneven(args, rank, world, local_rank)
        elif WORKLOADS[args.workload]["kind"] == "single_mixed":
            out = run_single_mixed(args, rank, world, local_rank)
        else:
            out = run_ours(args, rank, world, local_rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
