"""Benchmark: triangle-evaluations per second of the elastostatic layer-potential
FMM on one or more B200s.

A step is one complete elfmm3dtriatarg evaluation (tree + lists + four-pass
Laplace far field + analytic near field) of the workload below, with inputs
resident in device memory; `e2e` runs the same evaluation through the
reference-compatible C ABI (elfmm3dtriatarg_) from pinned host buffers, host
copies included.  One triangle-evaluation = one (evaluation point, source
triangle) interaction; the evaluation points are the centroids plus the
off-surface targets (elhfmm3dtria_self_iter_dr.f:270 counts the same product).

Workloads (seeded synthetic inputs, no datasets):
  sphere-1.3M : unit icosphere refined 8x (1,310,720 flat triangles) plus
                1,000,000 targets uniform in the shell 1.05 < |x| < 3,
                single + double layer densities i.i.d. N(0,1), lambda = mu = 1,
                iprec 2 (tolerance 0.5e-6), plain FP64.   [default]
  sphere-5120 : icosphere level 4 (5,120 triangles) plus 1,000 targets uniform
                in [-2,2]^3 with |x| > 1.1 (the CPU-runnable configuration).

--impl reference times the CPU stand-in for the reference (the oracle's direct
restatement of el3dtriadirecttarg; the Fortran reference cannot be compiled on
this image) on a bounded sample of evaluation points, all host cores.
Multi-GPU (torchrun): independent replicas, one per rank, no collectives on the
data path; value = total evaluations / max-over-ranks time.
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
    "sphere-1.3M": dict(level=8, ntarg=1_000_000, targets="shell", iprec=2),
    "sphere-5120": dict(level=4, ntarg=1_000, targets="box", iprec=2),
}


def make_inputs(name, seed=1):
    from elfmmlib3d_b200 import geometry as G
    w = WORKLOADS[name]
    tri, nrm, cen = G.sphere_triangles(w["level"])
    if w["targets"] == "shell":
        tgt = G.shell_targets(w["ntarg"], seed + 1)
    else:
        tgt = G.box_targets(w["ntarg"], seed + 1)
    rng = np.random.default_rng(seed)
    ssl = rng.normal(size=cen.shape)
    sdl = rng.normal(size=cen.shape)
    return tri, nrm, cen, tgt, ssl, sdl, w["iprec"]


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


def fp64_gemm_peak(torch, dev):
    """Measured FP64 throughput (cuBLAS DGEMM 8192^3, best of 5, CUDA events)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
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


def cpu_oracle_sample(tri, cen, tgt, ssl, sdl, nsample, seed=0):
    """Oracle direct sum for nsample evaluation points against all triangles,
    all host cores.  Returns (evals/s, seconds, cores, points)."""
    from oracle import oracle as O
    O.lib()
    n = len(cen)
    half = nsample // 2
    t0 = time.perf_counter()
    O.direct(1.0, 1.0, tri, cen, ssl, sdl, tgt, rows=(0, half), trows=(0, nsample - half))
    dt = time.perf_counter() - t0
    cores = os.cpu_count()
    return nsample * n / dt, dt, cores, nsample


# FP64 operations per near-field (point, triangle) pair of the analytic
# kernel: ncu thread-instruction counts of k_near_leaf on the sphere-5120 case,
# (dadd + dmul + 2 dfma) / pairs = (0.984e9 + 1.749e9 + 2 * 3.029e9) / 3.194e6
# (profiles/near_leaf_sphere5120.md)
NEAR_FLOPS_PER_PAIR = 2752.0


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
    t_max = ms
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
        dist.barrier()
    value = world * evals * args.steps / (t_max * 1e-3)

    # end to end through the Fortran ABI, pinned host buffers
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    htri, hnrm, hcen, htgt, hssl, hsdl = map(pin, (tri, nrm, cen, tgt, ssl, sdl))
    E.elfmm3dtriatarg(iprec, 1.0, 1.0, htri, hnrm, hcen, hssl, hsdl, htgt)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ier, *_ = E.elfmm3dtriatarg(iprec, 1.0, 1.0, htri, hnrm, hcen, hssl, hsdl, htgt)
        assert ier == 0, ier
    e2e_s = time.perf_counter() - t0
    e2e_t = e2e_s
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_t = float(tt.item())
    e2e_value = world * evals * args.steps / e2e_t
    h2d = 8 * (9 * n + 3 * n + 3 * n + 3 * m + 6 * n)
    d2h = 8 * (3 * n + 9 * n + 3 * m + 9 * m)

    if rank != 0:
        return None
    peak = fp64_gemm_peak(torch, dev)
    near_avg = float(np.mean(near_ms))
    flops = NEAR_FLOPS_PER_PAIR * info["near_pairs"]
    achieved = flops / (near_avg * 1e-3) / 1e12
    roof = {"kernel": "k_near_leaf", "bound": "fp64", "achieved": achieved, "peak": peak,
            "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
            "peak_source": "measured cuBLAS DGEMM 8192^3 in this run (FP64 has no entry in MEASURED_PEAKS.json)",
            "algorithmic": f"{NEAR_FLOPS_PER_PAIR:.0f} FP64 flop/pair x {info['near_pairs']} pairs"}
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        ev, dt, cores, npts = cpu_oracle_sample(tri, cen, tgt, ssl, sdl, args.cpu_sample)
        cpu = {"value": ev, "unit": "triangle-evals/s", "cores": cores, "kind": "port",
               "sample": f"oracle direct sum, {npts} evaluation points x {n} triangles ({dt:.1f} s)"}
    out = {
        "metric": "triangle-evals/s (free-space SLP+DLP displacement+strain, FP64 FMM at iprec 2)",
        "value": value, "unit": "triangle-evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "triangles": n, "targets": m, "iprec": iprec,
                   "evals_per_step": evals, "parallelism": f"replicas{world}",
                   "l2_policy": "inputs + expansions > L2 (126 MB)",
                   "stage_ms": tim, "setup_ms": setup, "tree": {k: info[k] for k in ("nboxes", "nlev", "p", "nbox")},
                   "near_pairs": info["near_pairs"], "m2l_pairs": info["m2l_pairs"]},
        "e2e": {"value": e2e_value, "unit": "triangle-evals/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "timing": "host wall clock around blocking C-ABI calls"},
        "gpu_launches": launches,
        "roofline": roof,
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }
    return out


def run_reference(args, rank):
    if rank != 0:
        return None
    tri, nrm, cen, tgt, ssl, sdl, iprec = make_inputs(args.workload)
    n = len(cen)
    for _ in range(args.warmup):
        cpu_oracle_sample(tri, cen, tgt, ssl, sdl, args.ref_sample)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ev, dt, cores, npts = cpu_oracle_sample(tri, cen, tgt, ssl, sdl, args.ref_sample)
    tot = time.perf_counter() - t0
    value = args.steps * args.ref_sample * n / tot
    return {
        "impl": "reference",
        "metric": "triangle-evals/s (free-space SLP+DLP displacement+strain, FP64 FMM at iprec 2)",
        "value": value, "unit": "triangle-evals/s", "n_gpus": 0, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "triangles": n, "targets": len(tgt), "iprec": iprec},
        "cpu_baseline": {"value": value, "unit": "triangle-evals/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"oracle direct sum (el3dtriadirecttarg restated), {args.ref_sample} "
                                   f"evaluation points x {n} triangles per step"},
        "e2e": {"value": value, "unit": "triangle-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sphere-1.3M", choices=list(WORKLOADS))
    ap.add_argument("--cpu-sample", type=int, default=16)
    ap.add_argument("--ref-sample", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
        out = run_ours(args, rank, world, local_rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
