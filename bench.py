#!/usr/bin/env python
"""Factor + solve throughput of the B200 recursive-skeletonization solver.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload star16k|stokes65k|ellipse1k|batch256]
                    [--no-cpu-baseline] [--no-adjoint]

One step = QuadTree build + skeletonize + solve of the workload (the
reference's SkelFactorization::skeletonize + linear_solve,
skel_factorization.cpp:94-403) to 1e-10 relative error.  The metric is
unknowns / (factor + solve time), for two methods on the same GPU:

  * mixed + refine (`value`): the factorization at ID tolerance 3e-7
    (3e-8 for stokes65k) in
    preconditioner mode (tall ID matrices reduced by a sparse row sketch)
    used by FP64 refinement / GMRES on the operator with on-the-fly FP64
    entries, stopped at relative residual 1e-12 (ki_factor_ex +
    ki_solve_refined_device; residuals below 5e-8 are updated with the
    correction product, FP32 far field / FP64 near field, and the true FP64
    residual of the result is reported beside it);
  * FP64 (`fp64`): the reference method, factorization at ID tolerance
    1e-10 and one direct solve (ki_factor + ki_solve_device).

The default workload is the Stokes disk with 8 holes (65,536 dofs, 64-point
leaves, multiply connected); `star16k` is the Laplace star r = 1 + 0.3 cos 5t,
N = 16384 nodes; `batch256` is 256 random stars of 512-8192 nodes factored
together (ki_factor_batch).  Errors are reported against the FP64 oracle (the
reference algorithm restated on the CPU) at ID tolerance 1e-10 and, as the
converged reference, at 1e-13.

Timing: CUDA events on the stream the library launches on, the right-hand
side resident in HBM, geometry in pinned host memory, the L2 flushed (256
MiB write) before every step, no per-launch instrumentation inside the timed
steps (the per-kernel figures come from one instrumented factorization and
the refinement's parts timed alone afterwards); `e2e` is the mixed method
through the host-buffer API (pinned geometry and data in, solution out) in
the same way.  With N > 1 GPUs (torchrun) every
rank solves its own replica (one problem does not shard): weak scaling, time
= max over ranks.  Unless --no-adjoint, a single-problem workload also times the
adjoint of the target-potential objective on the 8192-node Fourier star
(forward solve + targets, backward transposed solve + kernel-derivative
contractions).  `--impl reference` times the reference solver compiled from
its own sources (oracle/_ref) on the host cores for the same workload.
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
MIXED_TOL = 3e-7      # ID tolerance of the preconditioning factorization (default)
# per workload: the tolerance with the smallest factor + refinement time at
# the residual bar, measured on a B200 (Stokes: 3e-8 reaches it in two
# refinement products, looser tolerances need three)
MIXED_TOLS = {"stokes65k": 3e-8}
MIXED_MODE = 1        # KI_MODE_PRECONDITIONER: sketched IDs for tall boxes
REFINE_TOL = 1e-12    # true relative residual at which the refinement stops
FP64_TOL = 1e-10

WORKLOADS = {
    "star16k": (lambda: G.star_case(),
                "Laplace double layer, star r=1+0.3cos5t, N=16384 nodes, leaf 64 pts"),
    "stokes65k": (lambda: G.stokes_holes_case(),
                  "Stokes double layer, unit disk with 8 holes, 32768 nodes (65536 dofs), "
                  "leaf 64 pts, multiply-connected"),
    "ellipse1k": (lambda: G.ellipse_case(),
                  "Laplace double layer, ellipse (1.0,0.6), N=1024, leaf 64 pts"),
    "batch256": (lambda: G.random_star_cases(256, seed=4),
                 "256 Laplace random stars r=1+sum a_k cos(k t+phi_k), N log-uniform in "
                 "[512, 8192] (796,517 dofs in all), leaf 64 pts, one batched factorization"),
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
    """SM clock and clock-event reasons sampled during the timed region: NVML
    polled every 2 ms from a background thread (the timed region of a short
    run lasts well under nvidia-smi's sampling interval); `nvidia-smi -lms
    200` if NVML is unavailable.  Read-only queries."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40),
               ("sw_thermal_slowdown", 0x20), ("sw_power_cap", 0x4))

    def __init__(self, dev):
        import threading
        self.proc = None
        self.samples = []
        self.stop_ev = threading.Event()
        self.thread = None
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(dev)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))

            def poll():
                while not self.stop_ev.is_set():
                    try:
                        self.samples.append(
                            (float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)),
                             int(pynvml.nvmlDeviceGetCurrentClocksEventReasons(h))))
                    except Exception:
                        pass
                    self.stop_ev.wait(0.002)

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(dev), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.stop_ev.set()
            self.thread.join(timeout=5)
            if not self.samples:
                return None
            reasons = set()
            for _, bits in self.samples:
                for name, bit in self.REASONS:
                    if bits & bit:
                        reasons.add(name)
            return {"sm_mhz": float(np.median([c for c, _ in self.samples])),
                    "sm_max_mhz": self.max_mhz, "reasons": sorted(reasons),
                    "samples": len(self.samples), "source": "nvml"}
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
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


def max_over_ranks(times, dist, device):
    """Every rank's timings replaced by their maximum over the ranks (the
    job's time is its slowest replica's); unchanged without a process group."""
    if not dist:
        return list(times)
    import torch
    t = torch.tensor(list(times), device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


# ------------------------------------------------------------------ CPU arms
def _ref_solver():
    import kioracle as K
    kind = "reference" if K.ref_available() else "port"
    return kind, (K.RefSolver if kind == "reference" else K.PortSolver)


def _cpu_problems(workload, probs, per_step):
    """The problems one CPU step solves: the whole workload, or for the
    batch a bounded rotating sample of it."""
    if workload != "batch256":
        return lambda step: probs
    return lambda step: [probs[(step * per_step + i) % len(probs)] for i in range(per_step)]


def run_reference(args, probs):
    """Reference arm: the reference solver built from its own sources."""
    kind, Solver = _ref_solver()
    cores = os.cpu_count() or 1
    pick = _cpu_problems(args.workload, probs, 16)

    def step(i):
        t = 0.0
        u = 0
        for pr in pick(i):
            t0 = time.perf_counter()
            s = Solver(pr, id_tol=FP64_TOL, threads=cores)
            s.solve(pr.f)
            t += time.perf_counter() - t0
            s.close()
            u += pr.n_dofs
        return t, u

    for i in range(args.warmup):
        step(i)
    tot_t, tot_u = 0.0, 0
    for i in range(args.steps):
        t, u = step(args.warmup + i)
        tot_t += t
        tot_u += u
    value = tot_u / tot_t
    sample = ("%d steps, each a full FP64 factor+solve (id_tol 1e-10) of %s (OpenBLAS 0.3.15, "
              "1 BLAS thread, %d OpenMP box threads)"
              % (args.steps, "16 of the 256 problems" if args.workload == "batch256"
                 else "the workload", cores))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "unknowns/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * tot_t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload][1], "method": "FP64 direct",
                       "parallelism": "host threads", "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": value, "unit": "unknowns/s", "cores": cores,
                             "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "unknowns/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline(workload, probs, budget_s=12.0):
    kind, Solver = _ref_solver()
    cores = os.cpu_count() or 1
    pick = _cpu_problems(workload, probs, 16)
    n, t, u = 0, 0.0, 0
    while t < budget_s and n < 40:
        for pr in pick(n):
            t0 = time.perf_counter()
            s = Solver(pr, id_tol=FP64_TOL, threads=cores)
            s.solve(pr.f)
            t += time.perf_counter() - t0
            s.close()
            u += pr.n_dofs
        n += 1
    what = "16-problem samples of the batch" if workload == "batch256" else "full factor+solve runs"
    return {"value": u / t, "unit": "unknowns/s", "cores": cores, "kind": kind,
            "sample": "%d %s, FP64 id_tol 1e-10 (%.1f s)" % (n, what, t)}


def oracle_solutions(probs, idx):
    """FP64 oracle (CPU restatement) at id_tol 1e-10 and 1e-13 for the
    problems idx: (mu_1e10, mu_1e13) lists."""
    import kioracle as K
    cores = os.cpu_count() or 1
    a, b = [], []
    for i in idx:
        pr = probs[i]
        o = K.PortSolver(pr, id_tol=FP64_TOL, threads=cores)
        a.append(o.solve(pr.f)[0])
        o.close()
        o = K.PortSolver(pr, id_tol=1e-13, threads=cores)
        b.append(o.solve(pr.f)[0])
        o.close()
    return a, b


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


# ------------------------------------------------------------------ GPU arm
# algorithmic FP64 flops per (target node, source node) pair of the operator
# product: Laplace r (2), |r|^2 (3), reciprocal (1), r.n (3), scaled sum (2);
# Stokes the same pair terms plus the 2x2 tensor block (r.n, r.d, two
# outputs): 20
PAIR_FLOPS = {G.LAPLACE: 11.0, G.LAPLACE_NEUMANN: 11.0, G.STOKES: 20.0}


def pin_problem(p):
    """A copy of the problem whose geometry and data arrays are in pinned
    host memory (the arrays the factorization reads)."""
    import copy
    import torch
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).pin_memory().numpy()
    q = copy.copy(p)
    q.points, q.normals = pin(p.points), pin(p.normals)
    q.curvatures, q.weights = pin(p.curvatures), pin(p.weights)
    q.f = pin(p.f)
    return q


def event_ms(stream, fn, reps=5, flush=None):
    """Median CUDA-event time of fn() on `stream` (L2 flushed before each)."""
    import torch
    out = []
    for _ in range(reps):
        if flush is not None:
            flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        out.append(e0.elapsed_time(e1))
    return float(np.median(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="stokes65k", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--mixed-tol", type=float, default=None,
                    help="ID tolerance of the preconditioning factorization (default: per workload)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    global MIXED_TOL
    MIXED_TOL = args.mixed_tol or MIXED_TOLS.get(args.workload, MIXED_TOL)
    built = WORKLOADS[args.workload][0]()
    batch = args.workload == "batch256"
    probs = built if batch else [built]
    units = sum(p.n_dofs for p in probs)

    if args.impl == "reference":
        if rank == 0:
            run_reference(args, probs)
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
    # geometry and data in pinned host memory for every arm
    pp = [pin_problem(p) for p in probs]
    f_host = np.concatenate([p.f for p in probs])
    f_dev = torch.tensor(f_host, device=dev, dtype=torch.float64)
    mu_dev = torch.empty_like(f_dev)
    pr0 = pp[0]
    nb = 0 if batch else (3 * pr0.holes.shape[0] if pr0.pde == G.STOKES else pr0.holes.shape[0])
    al_dev = torch.empty(max(nb, 1), device=dev, dtype=torch.float64)

    def factor(tol, timed=False, mode=0):
        if batch:
            return kinterp.BatchSolver(pp, id_tol=tol, stream=sh, mode=mode)
        return kinterp.Solver(pr0, id_tol=tol, stream=sh, timed=timed, mode=mode)

    def refine(s):
        if batch:
            return s.solve_refined_device(f_dev.data_ptr(), mu_dev.data_ptr(),
                                          rel_tol=REFINE_TOL, max_iters=20)
        return s.solve_refined_device(f_dev.data_ptr(), mu_dev.data_ptr(),
                                      al_dev.data_ptr() if nb else None,
                                      rel_tol=REFINE_TOL, max_iters=20)

    def direct(s):
        if batch:
            s.solve_device(f_dev.data_ptr(), mu_dev.data_ptr())
        else:
            s.solve_device(f_dev.data_ptr(), mu_dev.data_ptr(), al_dev.data_ptr() if nb else None)

    def mixed_step(timed=False):
        s = factor(MIXED_TOL, timed, MIXED_MODE)
        it, rr = refine(s)
        return s, it, rr

    def fp64_step(timed=False):
        s = factor(FP64_TOL, timed)
        direct(s)
        return s

    def timed_loop(step_fn):
        """K steps, each: flush L2, events around one step on the library's
        stream.  Returns the total ms."""
        total = 0.0
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step_fn()
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
        return total

    # warm-up of both methods
    for _ in range(args.warmup):
        mixed_step()[0].close()
        fp64_step().close()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()

    # ---- mixed + refine (the value): no per-launch timing instrumentation
    clocks = Clocks(local)
    launches0 = kinterp.kernel_launches()
    iters, rres = [], []

    def mixed_timed():
        s, it, rr = mixed_step()
        iters.append(it)
        rres.append(rr)
        s.close()

    t_mixed = timed_loop(mixed_timed)
    launches = kinterp.kernel_launches() - launches0
    clk = clocks.stop()
    torch.cuda.synchronize()
    mu_mixed = mu_dev.cpu().numpy()
    al_mixed = al_dev.cpu().numpy()[:nb]

    # ---- FP64 direct (the reference method on the GPU)
    t_fp64 = timed_loop(lambda: fp64_step().close())
    torch.cuda.synchronize()
    mu_fp64 = mu_dev.cpu().numpy()

    # ---- e2e: public host-buffer API, pinned inputs, solution read back
    f_pin = torch.from_numpy(f_host).pin_memory().numpy()

    def e2e_step():
        if batch:
            s = kinterp.BatchSolver(pp, id_tol=MIXED_TOL, stream=sh, mode=MIXED_MODE)
        else:
            s = kinterp.Solver(pr0, id_tol=MIXED_TOL, stream=sh, mode=MIXED_MODE)
        s.solve_refined(f_pin, rel_tol=REFINE_TOL, max_iters=20)
        s.close()

    t_e2e = timed_loop(e2e_step)

    t_mixed, t_fp64, t_e2e = max_over_ranks([t_mixed, t_fp64, t_e2e], dist, dev)

    if rank == 0:
        # ---- per-kernel figures from separate, untimed passes: one
        # instrumented factorization of each method (launch durations by
        # CUDA events on the launching streams), then the refinement's parts
        # (one preconditioner application, one FP64 operator product, one
        # correction product) timed alone on the factorization it uses
        st, st64 = {}, {}
        parts = {}
        if not batch:
            s = factor(MIXED_TOL, True, MIXED_MODE)
            st = s.stats()
            n = s.n_dofs + s.n_border
            xv = torch.randn(n, device=dev, dtype=torch.float64)
            yv = torch.empty_like(xv)
            parts["solve_ms"] = event_ms(stream, lambda: direct(s), flush=flush)
            parts["matvec_ms"] = event_ms(
                stream, lambda: s.matvec_device(xv.data_ptr(), yv.data_ptr()), flush=flush)
            parts["corr_matvec_ms"] = event_ms(
                stream, lambda: s.matvec_correction_device(xv.data_ptr(), yv.data_ptr(), 1.0),
                flush=flush)
            parts["refine_ms"] = event_ms(stream, lambda: refine(s), flush=flush)
            # true FP64 residual of the timed run's solution
            xs = torch.tensor(np.concatenate([mu_mixed, al_mixed]), device=dev,
                              dtype=torch.float64)
            s.matvec_device(xs.data_ptr(), yv.data_ptr())
            torch.cuda.synchronize()
            bvec = np.concatenate([f_host, np.zeros(nb)])
            parts["true_rel_residual"] = float(np.linalg.norm(bvec - yv.cpu().numpy()) /
                                               np.linalg.norm(f_host))
            s.close()
            s = factor(FP64_TOL, True)
            st64 = s.stats()
            s.close()
        # accuracy against the FP64 oracle (at the reference's 1e-10 and,
        # as the converged solution, at 1e-13)
        idx = [0, 100, 200] if batch else [0]
        o10, o13 = oracle_solutions(probs, idx)
        offs = np.concatenate([[0], np.cumsum([p.n_dofs for p in probs])])
        err = lambda mu, ref: max(rel(mu[offs[i]:offs[i + 1]], r) for i, r in zip(idx, ref))
        analytic = None
        if not batch:
            s = kinterp.Solver(pr0)
            u = s.eval_targets(pr0.targets, mu_mixed, al_mixed)
            analytic = rel(u, pr0.exact)
            s.close()
        peak64 = fp64_peak_tflops(dev)
        hbm_peak, hbm_kind = peaks()
        h2d = sum(8 * (6 * p.n_points) for p in probs) + 8 * units
        d2h = 8 * (units + nb)
        value = world * units * args.steps / (t_mixed * 1e-3)
        fp64_value = world * units * args.steps / (t_fp64 * 1e-3)
        rooflines = {}
        if st:
            def fp64_line(kernel, flops, ms, launches=None):
                a = flops / (ms * 1e-3) / 1e12 if ms > 0 else None
                return {"kernel": kernel, "bound": "fp64", "achieved": a, "peak": peak64,
                        "unit": "TFLOP/s", "frac": a / peak64 if a else None,
                        "flops_per_step": flops, "ms_per_step": ms, "launches": launches}
            rooflines["id"] = fp64_line(
                "id_onchip_kernel / id_kernel (entry generation, pivoted QR, T)",
                st["id_flops"], st["id_ms"], st["id_launches"])
            rooflines["id"]["algorithmic_hbm_bytes"] = st["id_bytes"]
            rooflines["id"]["traffic_per_launch"] = traffic_from_profile(args.workload)
            rooflines["decouple"] = fp64_line(
                "decouple_kernel + large-box sequences (K_BN, T products, X_rr^-1, L, U, update)",
                st["dec_flops"], st["decouple_ms"])
            rooflines["top"] = fp64_line("assemble_top + lu_fused_kernel (top-level LU)",
                                         st["top_flops"], st["top_ms"])
            pairs = float(sum(p.n_points ** 2 for p in probs))
            rooflines["operator_product"] = fp64_line(
                "mv_partial_kernel + mv_finish_kernel (FP64 refinement residual)",
                PAIR_FLOPS[pr0.pde] * pairs, parts["matvec_ms"])
            sb = st["solve_bytes"]
            rooflines["solve_sweeps"] = {
                "kernel": "sweep_kernel / diag_inv_kernel / top LU solve (one preconditioner "
                          "application)", "bound": "hbm",
                "achieved": sb / (parts["solve_ms"] * 1e-3) / 1e9, "peak": hbm_peak,
                "unit": "GB/s", "frac": sb / (parts["solve_ms"] * 1e-3) / 1e9 / hbm_peak,
                "bytes": sb, "ms": parts["solve_ms"], "peak_source": hbm_kind}
        # the dominant kernel family of the mixed step
        dom = None
        if rooflines:
            shares = {"id": st["id_ms"], "decouple": st["decouple_ms"], "top": st["top_ms"],
                      "operator_product": parts["matvec_ms"],
                      "solve_sweeps": parts["solve_ms"] * max(1.0, float(np.mean(iters)))}
            dom = max(shares, key=shares.get)
        roof = None
        if dom:
            r = rooflines[dom]
            roof = {"kernel": r["kernel"], "family": dom, "bound": r["bound"],
                    "achieved": r["achieved"], "peak": r["peak"], "unit": r["unit"],
                    "frac": r["frac"],
                    "peak_source": ("measured live on this GPU: cuBLAS DGEMM 4096^3 (no FP64 "
                                    "figure in MEASURED_PEAKS.json)" if r["bound"] == "fp64"
                                    else "MEASURED_PEAKS.json hbm_gbs (%s)" % hbm_kind),
                    "traffic": traffic_from_profile(args.workload) if dom == "id" else None}
        line = {
            "metric": METRIC, "value": value, "unit": "unknowns/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_mixed / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOADS[args.workload][1], "n_dofs": units,
                       "method": "mixed+refine: factor at id_tol %g in preconditioner mode "
                                 "(sketched IDs), FP64 refinement/GMRES with on-the-fly FP64 "
                                 "operator (small residuals updated with FP32 far-field "
                                 "correction products) to rel. residual %g"
                                 % (MIXED_TOL, REFINE_TOL),
                       "leaf_dofs": pr0.max_leaf_dofs,
                       "parallelism": "replicas" if world > 1 else "single GPU",
                       "l2": "flushed between steps (256 MiB device write)",
                       "inputs": "geometry and data in pinned host memory; f resident in HBM "
                                 "for value, copied in and mu copied out for e2e"},
            "gmres_iters": float(np.mean(iters)), "rel_residual": float(max(rres)),
            "true_rel_residual": parts.get("true_rel_residual"),
            "rel_err_vs_fp64_oracle": err(mu_mixed, o10),
            "rel_err_vs_converged_oracle": err(mu_mixed, o13),
            "fp64_oracle_own_err": max(rel(a, b) for a, b in zip(o10, o13)),
            "analytic_rel_err": analytic,
            "phase_ms": None if batch else {
                "factor": st["factor_ms"], "id": st["id_ms"], "decouple": st["decouple_ms"],
                "top": st["top_ms"], "host_wait_on_ranks": st["wait_ms"],
                "refine": parts["refine_ms"], "one_solve": parts["solve_ms"],
                "fp64_operator_product": parts["matvec_ms"],
                "correction_product": parts["corr_matvec_ms"],
                "note": "one instrumented factorization and the refinement's parts timed "
                        "alone, outside the timed steps; launch durations overlap "
                        "(IDs of level l-1 run beside the decoupling of level l)"},
            "fp64": {"value": fp64_value, "ms_per_step": t_fp64 / args.steps,
                     "factor_ms": st64.get("factor_ms"),
                     "id_tol": FP64_TOL,
                     "rel_err_vs_fp64_oracle": err(mu_fp64, o10),
                     "rel_err_vs_converged_oracle": err(mu_fp64, o13)},
            "speedup_mixed_vs_fp64": value / fp64_value,
            "roofline": roof,
            "rooflines": rooflines or None,
            "e2e": {"value": world * units * args.steps / (t_e2e * 1e-3),
                    "unit": "unknowns/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        if not args.no_adjoint and not batch:
            line["adjoint"] = adjoint_bench(dev, stream)
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(args.workload, probs)
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def adjoint_bench(dev, stream, reps=5):
    """Adjoint of J = sum_t (u_t - u*_t)^2 on the 8192-node Fourier star (32
    shape coefficients, 64 targets): forward (geometry, factor at 1e-10,
    solve, targets) + backward (transposed solve, kernel-derivative
    contractions, chain rule to the coefficients), CUDA events on the
    caller's stream (device-wide synchronisation around each run); gradient
    checked against central differences (h = 1e-6) in two coefficients."""
    import torch
    import ki_autograd as KA
    pr = G.fourier_star_case(n=8192)
    coef, u_star = pr.extra["coef"], pr.extra["u_star"]
    tg = torch.tensor(pr.targets, dtype=torch.float64, device=dev)
    us = torch.tensor(u_star, dtype=torch.float64, device=dev)
    f = torch.tensor(pr.f, dtype=torch.float64, device=dev)

    def objective(c_np):
        c = torch.tensor(c_np, dtype=torch.float64, device=dev)
        pts, nrm, kap, w = KA.fourier_star_geometry(c, pr.n_points)
        u = KA.target_potential(pts, nrm, kap, w, f, tg, pr.leaf_points, FP64_TOL)
        return float(((u - us) ** 2).sum())

    times, fwd = [], []
    g = None
    for i in range(reps + 2):
        torch.cuda.synchronize()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        c = torch.tensor(coef, dtype=torch.float64, device=dev, requires_grad=True)
        pts, nrm, kap, w = KA.fourier_star_geometry(c, pr.n_points)
        u = KA.target_potential(pts, nrm, kap, w, f, tg, pr.leaf_points, FP64_TOL)
        J = ((u - us) ** 2).sum()
        e1.record(stream)
        J.backward()
        e2.record(stream)
        torch.cuda.synchronize()
        if i >= 2:
            times.append(e0.elapsed_time(e2))
            fwd.append(e0.elapsed_time(e1))
        g = c.grad.cpu().numpy()
    h = 1e-6
    fd_err = 0.0
    for q in (0, 17):
        cp, cm = coef.copy(), coef.copy()
        cp[q] += h
        cm[q] -= h
        fd = (objective(cp) - objective(cm)) / (2 * h)
        fd_err = max(fd_err, abs(fd - g[q]) / np.abs(g).max())
    return {"workload": "Laplace Fourier star, 32 shape coefficients, N=8192, leaf 64 pts, "
                        "64 targets, id_tol 1e-10",
            "ms": float(np.median(times)), "forward_ms": float(np.median(fwd)),
            "backward_ms": float(np.median(times) - np.median(fwd)),
            "grad_vs_central_fd_rel": fd_err}


if __name__ == "__main__":
    main()
