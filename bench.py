#!/usr/bin/env python
"""Factor + solve throughput of the B200 recursive-skeletonization solver.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload star16k|stokes65k|ellipse1k]

One step = QuadTree build + skeletonize + solve of one boundary integral
problem (the reference's SkelFactorization::skeletonize + linear_solve,
skel_factorization.cpp:94-403).  The default workload is the Laplace star
r = 1 + 0.3 cos 5t with N = 16384 nodes, 64-point leaves and ID tolerance
1e-10 (FP64).  The metric is unknowns / (factor + solve time).

`value` times ki_factor (geometry from host memory: the quadtree is built on
the host) + ki_solve_device with the right-hand side resident in HBM; `e2e`
times the public host-buffer path ki_factor + ki_solve with pinned inputs
and the solution copied back.  Both are CUDA-event times on the stream the
library launches on, L2 flushed (256 MiB write) between steps.  With N > 1
GPUs (torchrun) every rank factors its own replica of the problem (one
problem does not shard); the time is the max over ranks.
`--impl reference` times the reference solver compiled from its own sources
(oracle/_ref) on the host cores for the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "kern-interp-old_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

import ki_geometry as G  # noqa: E402

METRIC = "factor+solve unknowns/s at 1e-10 rel err"
WORKLOADS = {
    "star16k": (lambda: G.star_case(),
                "Laplace double layer, star r=1+0.3cos5t, N=16384 nodes, leaf 64 pts, "
                "id_tol 1e-10, FP64"),
    "stokes65k": (lambda: G.stokes_holes_case(),
                  "Stokes double layer, unit disk with 8 holes, 32768 nodes (65536 dofs), "
                  "leaf 64 pts, id_tol 1e-10, FP64, multiply-connected"),
    "ellipse1k": (lambda: G.ellipse_case(),
                  "Laplace double layer, ellipse (1.0,0.6), N=1024, leaf 64 pts, id_tol 1e-10, FP64"),
}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_from_profile(workload):
    """DRAM bytes per ID launch (read + write, averaged over the ID launches of
    one factorization) from the committed ncu summary of this workload."""
    import re
    path = os.path.join(ROOT, "profiles", "id_kernel_%s.txt" % workload)
    try:
        with open(path) as f:
            m = re.search(r"^dram_bytes_per_id_launch:\s*([0-9.eE+]+)", f.read(), re.M)
        return float(m.group(1)) if m else None
    except OSError:
        return None


def fp64_peak_tflops(dev):
    """FP64 compute roof measured on this GPU: cuBLAS DGEMM 4096^3 (2 n^3
    flops), best of 5, CUDA events.  The B200's FP64 FMA pipe and its FP64
    tensor path have the same nominal rate; tcgen05 has no FP64 kind."""
    import torch
    n = 4096
    a = torch.randn(n, n, device=dev, dtype=torch.float64)
    b = torch.randn(n, n, device=dev, dtype=torch.float64)
    c = torch.empty_like(a)
    for _ in range(2):
        torch.matmul(a, b, out=c)
    best = float("inf")
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b, c
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(dev), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "reasons": sorted(reasons), "samples": len(sm)}


def run_reference(args, pr, units):
    """Reference arm: the reference solver built from its own sources."""
    import kioracle as K
    kind = "reference" if K.ref_available() else "port"
    cores = os.cpu_count() or 1
    Solver = K.RefSolver if kind == "reference" else K.PortSolver

    def step():
        t0 = time.perf_counter()
        s = Solver(pr, threads=cores)
        mu, alpha = s.solve(pr.f)
        dt = time.perf_counter() - t0
        s.close()
        return dt

    for _ in range(args.warmup):
        step()
    times = [step() for _ in range(args.steps)]
    total = sum(times)
    value = units * args.steps / total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "unknowns/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload][1], "n_dofs": units,
                       "parallelism": "host threads", "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": value, "unit": "unknowns/s", "cores": cores,
                             "kind": kind,
                             "sample": "%d full factor+solve runs of the workload "
                                       "(OpenBLAS 0.3.15, 1 BLAS thread, %d OpenMP box "
                                       "threads)" % (args.steps, cores)},
            "e2e": {"value": value, "unit": "unknowns/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline(pr, units, budget_s=12.0):
    import kioracle as K
    kind = "reference" if K.ref_available() else "port"
    Solver = K.RefSolver if kind == "reference" else K.PortSolver
    cores = os.cpu_count() or 1
    n, t = 0, 0.0
    while t < budget_s and n < 40:
        t0 = time.perf_counter()
        s = Solver(pr, threads=cores)
        s.solve(pr.f)
        t += time.perf_counter() - t0
        s.close()
        n += 1
    return {"value": units * n / t, "unit": "unknowns/s", "cores": cores, "kind": kind,
            "sample": "%d full factor+solve runs of the same workload (%.1f s)" % (n, t)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="star16k", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pr = WORKLOADS[args.workload][0]()
    units = pr.n_dofs

    if args.impl == "reference":
        if rank == 0:
            run_reference(args, pr, units)
        return

    import torch
    import kinterp
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    # a dedicated (non-default) stream: the library launches on it and the
    # events bracket exactly that stream's work
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    f_dev = torch.tensor(pr.f, device=dev, dtype=torch.float64)
    mu_dev = torch.empty_like(f_dev)
    nb = 3 * pr.holes.shape[0] if pr.pde == G.STOKES else pr.holes.shape[0]
    al_dev = torch.empty(max(nb, 1), device=dev, dtype=torch.float64)

    def device_step(timed):
        s = kinterp.Solver(pr, stream=sh, timed=timed)
        s.solve_device(f_dev.data_ptr(), mu_dev.data_ptr(), al_dev.data_ptr() if nb else None)
        return s

    for _ in range(args.warmup):
        device_step(False).close()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = Clocks(local)
    launches0 = kinterp.kernel_launches()
    total_ms = 0.0
    id_ms = id_flops = id_bytes = id_launch = 0.0
    factor_ms = []
    kinds = {}
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s = device_step(True)
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
        st = s.stats()
        factor_ms.append(st["factor_ms"])
        id_ms += st["id_ms"]
        id_flops += st["id_flops"]
        id_bytes += st["id_bytes"]
        id_launch += st["id_launches"]
        for row in s.launch_log():
            kinds[int(row[1])] = kinds.get(int(row[1]), 0.0) + row[6]
        s.close()
    torch.cuda.synchronize()
    launches = kinterp.kernel_launches() - launches0
    clk = clocks.stop()

    # e2e: public host-buffer API, pinned inputs, result read back every step
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).pin_memory().numpy()
    import copy
    pe = copy.copy(pr)
    pe.points, pe.normals = pin(pr.points), pin(pr.normals)
    pe.curvatures, pe.weights, pe.f = pin(pr.curvatures), pin(pr.weights), pin(pr.f)
    e2e_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s = kinterp.Solver(pe, stream=sh)
        mu_h, al_h = s.solve(pe.f)
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
        s.close()

    t_max = total_ms
    e2e_max = e2e_ms
    if dist:
        t = torch.tensor([total_ms, e2e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max, e2e_max = float(t[0]), float(t[1])

    if rank == 0:
        # parity of the timed path against the FP64 oracle, and the analytic error
        import kioracle as K
        o = K.PortSolver(pr, threads=os.cpu_count() or 1)
        mo, ao = o.solve(pr.f)
        rel_oracle = float(np.linalg.norm(mu_h - mo) / np.linalg.norm(mo))
        s = kinterp.Solver(pr)
        u = s.eval_targets(pr.targets, mu_h, al_h)
        analytic = float(np.linalg.norm(u - pr.exact) / np.linalg.norm(pr.exact))
        s.close()
        hbm_peak, hbm_kind = peaks()
        fp64_peak = fp64_peak_tflops(dev)
        achieved = (id_flops / (id_ms * 1e-3)) / 1e12 if id_ms > 0 else None
        traffic = traffic_from_profile(args.workload)
        h2d = 8 * (6 * pr.n_points + units)
        d2h = 8 * (units + nb)
        value = world * units * args.steps / (t_max * 1e-3)
        line = {
            "metric": METRIC, "value": value, "unit": "unknowns/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload][1], "n_dofs": units,
                       "leaf_dofs": pr.max_leaf_dofs, "id_tol": pr.id_tol,
                       "parallelism": "replicas" if world > 1 else "single GPU",
                       "l2": "flushed between steps (256 MiB device write)"},
            "factor_ms": float(np.mean(factor_ms)),
            "solve_ms": t_max / args.steps - float(np.mean(factor_ms)),
            "rel_err_vs_fp64_oracle": rel_oracle, "analytic_rel_err": analytic,
            "phase_ms_per_step": {"id": kinds.get(0, 0.0) / args.steps,
                                  "decouple": kinds.get(1, 0.0) / args.steps,
                                  "top": kinds.get(2, 0.0) / args.steps},
            "roofline": {"kernel": "ID kernels (id_onchip_kernel / id_kernel: entry generation, "
                                   "pivoted QR, T)",
                         "bound": "tensor", "pipe": "fp64 (no tcgen05 FP64 kind; FP64 FMA)",
                         "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                         "frac": (achieved / fp64_peak) if achieved else None,
                         "peak_source": "measured live on this GPU: cuBLAS DGEMM 4096^3 "
                                        "(no FP64 figure in MEASURED_PEAKS.json)",
                         "flops_per_launch": id_flops / max(id_launch, 1),
                         "algorithmic_hbm_bytes_per_launch": id_bytes / max(id_launch, 1),
                         "hbm_frac_of_measured": ((id_bytes / (id_ms * 1e-3)) / 1e9 / hbm_peak)
                         if id_ms > 0 else None,
                         "hbm_peak_gbs": hbm_peak, "hbm_peak_source": hbm_kind,
                         "launches_per_step": id_launch / args.steps,
                         "ms_per_step": id_ms / args.steps,
                         "traffic": traffic},
            "e2e": {"value": world * units * args.steps / (e2e_max * 1e-3),
                    "unit": "unknowns/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(pr, units)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
