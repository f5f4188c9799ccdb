#!/usr/bin/env python
"""TVAL3 time-to-solution benchmark on B200 (one JSON line on rank 0).

Default workload: the 2D ultrasound-tomography ring - 256x256
image, 512 transducers on the inscribed circle, each emitter firing at the 256
receivers on the opposite half (131072 rays, 2.72e7 Bresenham hits),
isotropic TV, mu=2^10, beta=2^6, tol=1e-5, maxit=500 - on the on-the-fly
Bresenham projector.  A step is one reconstruction (scaleb, A^T b, the
continuation / inner loop, final scaling) through a device-resident plan whose
iteration loop is one CUDA graph with conditional nodes, run until it is
within 1e-3 (relative L2) of the FP64 solution (tests/golden, given as Ut) or
the reference's own stopping rules end it.

  value   reconstructions/s with inputs resident in HBM (CUDA events around
          each solve on the launching stream; 256 MB L2 flush between solves)
  fp64_noise_floor  how far the FP64 solution itself moves when one FP32
          rounding per stored element and iteration is added (the oracle's
          noise model, precomputed in tests/golden): an FP32 solve cannot be
          held closer than that to it
  e2e     the same problem through the host-buffer C ABI tval3g_solve
          (geometry and b from host memory, U back to host, the per-call
          operator preparation included, the reference's stopping rules);
          host clock around the blocking call
  roofline  the dominant kernel timed alone with CUDA events after an L2
          flush, algorithmic bytes / time against the measured HBM copy rate
  cpu_baseline  the reference solver itself (oracle/_ref, compiled from its
          own sources) on the CSR twin: one complete solve under its own
          stopping rules (anisotropic TV: the reference has no isotropic TV)
  aniso   the same workload with anisotropic TV on the GPU (the reference
          arm's problem): time to relerr <= 1e-3 and the full solve
  unit_weight  the literal unit-weight ring, a fixed 20 iterations, against
          the FP64 oracle's 20 iterations
  batch   the mixed batch of 64 independent 2D problems (58 GB of dense A
          drawn on the device from seeded counter-based streams): the
          batched graph against the plain one-instance-per-launch form, the
          HBM floor of its dense instances, and the relerr of each instance
          of its FP64 subset
  configs the other reference configurations in compact records (one GPU
          only): the dense 64x64 solve, the 128^3 hemisphere, the multi-RHS
          solve (joint and independent right-hand sides) and the
          differentiable unrolled solve, two timed steps each; and the
          double-data path (tval3g_solve_f64) end to end on the ring and the
          dense 64x64 problem against their FP64 solutions

--workload dense2d | hemi3d | batch | mrhs | unrolled measures the plain dense
64x64 problem, the 128^3 hemisphere, the mixed batch alone, the joint
multi-RHS solve and the differentiable unrolled solve.
--impl reference runs only the reference CPU solver (complete solves, at most
three timed) on the default workload.
Multi-GPU (torchrun): every rank solves its own replica (no collective in the
data path); value = total reconstructions / max-over-ranks time.
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
sys.path.insert(0, os.path.join(ROOT, "tval3-cpu_b200", "python"))

METRIC = "TVAL3 time-to-solution (relerr≤1e-3 vs FP64), batched vs plain, 1 B200; HBM %"
GOLDEN = os.path.join(ROOT, "tests", "golden")


def args_():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="tval3g", choices=["tval3g", "reference"])
    p.add_argument("--workload", default="ring2d",
                   choices=["ring2d", "dense2d", "hemi3d", "batch", "mrhs", "unrolled"])
    p.add_argument("--profile", action="store_true",
                   help="for ncu: build the plan, run --warmup + --steps solves, print nothing else")
    p.add_argument("--maxit", type=int, default=None, help="override maxit (profiling a short solve)")
    p.add_argument("--side", type=int, default=64,
                   help="dense2d: image side (profiling the dense normal product on wider rows; not the 64x64 "
                        "configuration then, and no FP64 comparison)")
    p.add_argument("--sampling", type=float, default=0.3, help="dense2d: rows of A per pixel (m = sampling n)")
    p.add_argument("--no-batch", action="store_true",
                   help="ring workload: leave out the mixed-batch sub-record (64 problems, 58 GB of dense A) "
                        "and the other configurations' records")
    p.add_argument("--tune", action="store_true",
                   help="single-instance workloads: operators built with the launch-shape autotuner")
    p.add_argument("--plain", action="store_true",
                   help="with --profile: run the host-driven loop (same kernels, same order) instead of the "
                        "CUDA graph, whose conditional nodes ncu cannot profile kernel by kernel")
    return p.parse_args()


def workload(name, forward3d=None, side=64, sampling=0.3):
    from tval3g import workloads as W
    if name == "ring2d":
        return W.ring2d(seed=1, side=256, T=512, tv_norm=1, maxit=500, tol=1e-5, normalize=True)
    if name == "dense2d":
        return W.dense2d(seed=0, side=side, sampling=sampling, tv_norm=1, maxit=300, tol=1e-4)
    if name == "hemi3d":
        return W.hemi3d(seed=2, side=128, T=2048, receivers=1024, tv_norm=0, maxit=400, tol=1e-5,
                        forward=forward3d)
    raise KeyError(name)


CONFIGS = {
    "ring2d": {"workload": "2D ring 256x256, 512 transducers x 256 receivers (131072 rays, 2.72e7 hits), iso TV, "
                           "mu 2^10, beta 2^6, tol 1e-5, maxit 500; hit weight scale_factor = "
                           "1/sigma_max(A) so that mu and beta act as in TVAL3",
               "operator": "on-the-fly Bresenham projector, tiled pixel-major adjoint"},
    "dense2d": {"workload": "2D dense 64x64, A 1229x4096 N(0,1/m), iso TV, mu 2^8, beta 2^5, tol 1e-4, maxit 300",
                "operator": "dense normal product in one pass over A"},
    "hemi3d": {"workload": "3D 128^3, 2048 hemisphere transducers x 1024 random receivers (2.1M rays), aniso TV, "
                           "mu 2^10, beta 2^6, tol 1e-5, maxit 400; hit weight 1/sigma_max(A)",
               "operator": "on-the-fly 3D Bresenham projector, gather adjoint"},
    "mrhs": {"workload": "dense A 4096 x 16384 N(0,1/m), 32 right-hand sides (128x128 phantoms) solved jointly as "
                         "32 layers, iso TV, mu 2^8, beta 2^5, tol 1e-4, maxit 300",
             "operator": "tcgen05 3xTF32 multi-RHS product (TMA, TMEM, stream-K over all SMs)"},
    "unrolled": {"workload": "differentiable unrolled solve: 8 phantoms of 128x128 on the ring of 256 transducers x "
                             "128 receivers (32768 rays), K = 50 iterations with per-iteration (mu_k, beta_k), "
                             "checkpoint every 10, loss 0.5 |u_K - u_true|^2, gradients w.r.t. b, mu_k, beta_k",
                 "operator": "on-the-fly Bresenham projector; hand-written adjoint of the unrolled iterations"},
    "batch": {"workload": "64 independent 2D problems, sides {64..256}, dense Gaussian (25-40 % sampling) or ring "
                          "Bresenham (128-512 transducers)",
              "operator": "mixed dense / ray, one batched plan"},
}


def fp64_reference(name):
    f = {"ring2d": "ring256_fp64.npz", "dense2d": "dense64_fp64.npz", "mrhs": "mrhs32_fp64.npz"}.get(name)
    if f and os.path.exists(os.path.join(GOLDEN, f)):
        return dict(np.load(os.path.join(GOLDEN, f)))
    return None


# --------------------------------------------------------------------------
# clocks
# --------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.rows, self.proc = gpu, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()   # the first sample before the timed region starts
            while not self.rows and time.time() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.01)
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        k, t0 = len(self.rows), time.time()   # and one taken after it ends
        while len(self.rows) == k and time.time() - t0 < 1.0 and self.proc.poll() is None:
            time.sleep(0.01)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows if len(r) >= 9 for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm)}


# --------------------------------------------------------------------------
# reference arm / CPU baseline
# --------------------------------------------------------------------------
def reference_solve(w):
    """One complete solve of the reference's own solver (float data, all host
    threads, its own stopping rules: maxit, tol, tol_inn), timed by the host
    clock around the call (its info.secs covers the same span,
    2d/tval3_cpu_2d.cpp:760,862).  Ray workloads run on their CSR twin (the
    reference's 2D projector is commented out, 2d/mat_mult.h:111-193); the
    reference has anisotropic TV only.  Returns (seconds, result) or None
    when oracle/_ref was not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.ref_available(2):
        return None
    o = dict(w["opts"])
    o["tv_norm"] = 0
    cwd = os.getcwd()
    t0 = time.perf_counter()
    if w["kind"] == "dense":
        r = O.ref_solve("dense", w["shape"], w["b"], o, dtype=0, A=w["A"], vppc=1)
    else:
        A = w["csr"]
        r = O.ref_solve("csr", w["shape"], w["b"], o, dtype=0,
                        csr=(A["m"], A["n"], A["rowptr"], A["colind"], A["val"]), vppc=1)
    secs = time.perf_counter() - t0
    os.chdir(cwd)
    return secs, r


def rel_l2(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


# the reference arm times complete solves: at most this many (and one
# warm-up), so that the arm ends within a few minutes whatever --steps asks
REF_MAX_STEPS, REF_MAX_WARMUP = 3, 1


def run_reference(a, rank):
    if rank != 0:
        return
    w = workload("ring2d")
    ref = fp64_reference("ring2d")
    steps, warm = max(1, min(a.steps, REF_MAX_STEPS)), min(a.warmup, REF_MAX_WARMUP)
    for _ in range(warm):
        if reference_solve(w) is None:
            break
    secs, r = [], None
    for _ in range(steps):
        out = reference_solve(w)
        if out is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (the reference "
                                                                  "sources were absent when building)"}))
            return
        secs.append(out[0])
        r = out[1]
    ms = float(np.mean(secs)) * 1000
    val = 1000.0 / ms
    err = rel_l2(r.U, ref["U_aniso"]) if ref is not None and "U_aniso" in ref else None
    sample = (f"complete solves of the reference solver (float data, anisotropic TV: it has no isotropic TV) "
              f"on the CSR twin of the ring operator, its own stopping rules: {r.total_iters} iterations, "
              f"relerr vs the FP64 anisotropic solution {err:.2e}" if err is not None else
              f"complete solves of the reference solver ({r.total_iters} iterations)")
    line = {"metric": METRIC, "value": val, "unit": "reconstructions/s", "n_gpus": a.gpus, "steps": steps,
            "warmup": warm, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "config": CONFIGS["ring2d"], "impl": "reference",
            "requested": {"steps": a.steps, "warmup": a.warmup,
                          "note": f"at most {REF_MAX_STEPS} timed complete solves and {REF_MAX_WARMUP} warm-up"},
            "iterations": r.total_iters, "relerr_vs_fp64_aniso": err, "tv": "anisotropic",
            "cpu_baseline": {"value": val, "unit": "reconstructions/s", "cores": os.cpu_count(), "kind": "reference",
                             "sample": sample},
            "e2e": {"value": val, "unit": "reconstructions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# --------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------
class Ctx:
    def __init__(self, torch, dev, stream, flush):
        self.torch, self.dev, self.stream, self.flush = torch, dev, stream, flush

    def event_time(self, fn, reps):
        torch = self.torch
        out, res = [], None
        for _ in range(reps):
            self.flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(self.stream)
            res = fn()
            e1.record(self.stream)
            e1.synchronize()
            out.append(e0.elapsed_time(e1))
        return out, res


def max_over_ranks(dist, values, device):
    """Each value's maximum over the ranks (the job's time is its slowest
    rank's); the values unchanged without a process group."""
    if not dist:
        return [float(v) for v in values]
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(p)) if os.path.exists(p) else {}
    if "hbm_gbs" in peaks:
        return float(peaks["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured)"
    return 6650.0, "fallback 6.65 TB/s"


def profile_traffic(name):
    prof = os.path.join(ROOT, "profiles", name)
    if os.path.exists(prof):
        for line in open(prof):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1].split()[0])
    return None


def kernel_roofline(cx, capi, spec, w, kind):
    """Time the dominant operator kernel alone (per launch, after an L2 flush)."""
    torch, dev, s = cx.torch, cx.dev, cx.stream.cuda_stream
    op = capi.Operator(spec)
    x = torch.rand(op.cols, device=dev)
    y = torch.rand(op.rows, device=dev)
    out_m = torch.empty(op.rows, device=dev)
    out_n = torch.empty(op.cols, device=dev)
    kt = {}
    dirs = {"forward": (x, out_m, 0), "adjoint": (y, out_n, 1)}
    if kind == "dense":
        dirs["normal"] = (x, out_n, 2)
    for name, (src, dst, tr) in dirs.items():
        op.apply_n(src, dst, 3, trans=tr, stream=s)
        ts, _ = cx.event_time(lambda: op.apply_n(src, dst, 1, trans=tr, stream=s), 10)
        kt[name] = float(np.mean(ts))
    nnz, n, m, index = op.nnz, op.cols, op.rows, op.adjoint_index_bytes
    op.close()
    variants = None
    if kind in ("ray2d", "ray3d"):
        # the other adjoint form: rays traced on the fly, atomic adds into the image
        opa = capi.Operator(spec, adj_atomics=True)
        opa.apply_n(y, out_n, 3, trans=1, stream=s)
        ts, _ = cx.event_time(lambda: opa.apply_n(y, out_n, 1, trans=1, stream=s), 10)
        opa.close()
        opp = capi.Operator(spec, adj_plain=True)
        opp.apply_n(y, out_n, 3, trans=1, stream=s)
        tp, _ = cx.event_time(lambda: opp.apply_n(y, out_n, 1, trans=1, stream=s), 10)
        plain_index = opp.adjoint_index_bytes
        opp.close()
        variants = {"tiled_gather_ms": kt["adjoint"], "plain_gather_ms": float(np.mean(tp)),
                    "atomics_ms": float(np.mean(ts)), "tiled_index_bytes": int(index),
                    "plain_index_bytes": int(plain_index),
                    "default": "tiled gather (deterministic)",
                    "forms": "tiled: measurements of each 2D tile / 3D brick staged in shared memory, 16-bit "
                             "positions per hit; plain: 4-byte traced-ray id per hit, measurements from L2; "
                             "atomics: rays traced on the fly, atomic adds into the image"}
    peak, src = peak_hbm()
    if kind == "ray2d":
        # tiled adjoint: its index once (tile lists, 16-bit positions, offsets),
        # the measurement vector once, the image once
        bytes_ = index + 4 * m + 4 * n
        kname, prof, direction = "k_ray_adj_tiled (ray adjoint)", "ray_adjoint_tiled_ring256.md", "adjoint"
    elif kind == "ray3d":
        # brick-tiled adjoint: its index once (brick lists, 16-bit positions,
        # offsets), the measurement vector once, the image once
        bytes_ = index + 4 * m + 4 * n
        kname, prof, direction = "k_ray_adj_tiled (3D bricks)", "ray_adjoint_brick_hemi128.md", "adjoint"
    else:
        A = w["A"]
        # the solve's normal product A^T (A u): A once, u read, Au written and
        # read back, g written
        bytes_ = 4 * A.size + 4 * (2 * A.shape[1] + 2 * A.shape[0])
        kname, prof, direction = "k_dense_normal (A^T A u, A read once)", "dense_normal_64.md", "normal"
    achieved = bytes_ / (kt[direction] * 1e-3) / 1e9
    return {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": profile_traffic(prof), "algorithmic_bytes": int(bytes_),
            "ms_per_launch": kt[direction], "peak_source": src,
            "ms_per_launch_by_direction": kt, "adjoint_variants": variants,
            "timing": "one launch per CUDA-event pair, 256 MB L2 flush before each"}


def stencil_roofline(plan, spec, w, ut):
    """The iteration's image-sized vector kernels, each timed alone (20
    launches back to back after the solve; at 128^3 each touches more than
    the L2): algorithmic bytes = the vectors each reads and writes once."""
    ms = plan.time_stencils(20)
    n, m = spec.n, int(np.asarray(w["b"]).size)
    dims = len(w["shape"])
    xT = w["kind"] == "ray2d"   # the descent also writes the transposed image for the 2D ray forward
    byts = {"getg": 4 * n * ((3 + 2 * dims) + (1 + dims)) + 12 * m,      # g, Atb, U, W, S -> g, D U; Au, b, delta
            "descend": 4 * n * (2 * (4 + dims) + (1 if xT else 0)) + 8 * m,  # U, g, g2, D U, d -> snapshots, U; Au -> Aup
            "shrink_grad": 4 * n * (3 * dims + 9 + (1 if ut else 0))}    # D U, S, Dts, g, Up, U, gp, g2p -> W, g2, d, uup
    peak, src = peak_hbm()
    out = {}
    for k, t in ms.items():
        gbs = byts[k] / (t * 1e-3) / 1e9
        out[k] = {"ms_per_launch": t, "algorithmic_bytes": int(byts[k]), "achieved_gbs": gbs, "frac": gbs / peak}
    out["peak_source"] = src
    out["timing"] = "20 launches back to back after the solve, CUDA events on the plan's stream"
    return out


def launch_shape(capi, spec):
    """The autotuner's choice for spec's operator (from its cache, filled by
    the plan): lanes per ray of the ray forward, forward / adjoint gather
    width classes (0 = built-in)."""
    op = capi.Operator(spec, tune=True)
    s = op.launch_shape()
    op.close()
    return {"forward_lanes_per_ray": s[0], "forward_gather_class": s[1], "adjoint_gather_class": s[2]}


def run_single(a, cx, capi, name, world, rank, dist, clocks, cpu=True):
    torch, dev, stream = cx.torch, cx.dev, cx.stream
    fwd3d = None
    if name == "hemi3d":   # data from the GPU operator (no host CSR twin at this size)
        def fwd3d(g, u):
            # hit weight 1/sigma_max(A), as for the ring (power iteration on A^T A)
            op = capi.Operator(capi.ray3d_problem(u.shape, g))
            x = torch.rand(op.cols, device=dev, generator=torch.Generator(device=dev).manual_seed(7))
            y = torch.empty(op.rows, device=dev)
            lam = 1.0
            for _ in range(30):
                x /= torch.linalg.vector_norm(x)
                op.apply(x, y, stream=stream.cuda_stream)
                op.apply(y, x, trans=True, stream=stream.cuda_stream)
                lam = float(torch.linalg.vector_norm(x))
            op.close()
            g["scale"] = float(np.float32(1.0 / np.sqrt(lam)))
            op = capi.Operator(capi.ray3d_problem(u.shape, g))
            op.apply(torch.tensor(u.ravel().astype(np.float32), device=dev), y, stream=stream.cuda_stream)
            op.close()
            return y.cpu().numpy()
    w = workload(name, fwd3d, a.side, a.sampling)
    custom = name == "dense2d" and (a.side, a.sampling) != (64, 0.3)
    spec = capi.problem_from_workload(w)
    opts = dict(w["opts"])
    if a.maxit is not None:
        opts["maxit"] = a.maxit
    b_host = np.ascontiguousarray(w["b"], np.float32)
    d_b = torch.tensor(b_host, device=dev)
    d_U = torch.empty(spec.n, device=dev)
    ref = None if custom else fp64_reference(name)
    d_ref = torch.tensor(ref["U"].ravel().astype(np.float32), device=dev) if ref is not None else None
    target = 1e-3 if ref is not None else 0.0
    uts = [d_ref] if d_ref is not None else None

    plan = capi.Plan([spec], [opts], graph=not (a.profile and a.plain), trace=True, tune=a.tune)
    plan.set_target(target)
    solve = lambda p: p.solve([d_b], [d_U], d_Ut=uts, stream=stream.cuda_stream)  # noqa: E731
    if a.profile:
        cx.event_time(lambda: solve(plan), a.warmup + a.steps)
        plan.close()
        return None
    cx.event_time(lambda: solve(plan), max(a.warmup, 3))
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    times, launches, infos = [], 0, None
    for _ in range(a.steps):
        t1, infos = cx.event_time(lambda: solve(plan), 1)
        times += t1
        launches += plan.stats()["kernel_launches"]
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms = max_over_ranks(dist, [float(np.mean(times))], dev)[0]
    iters = infos[0]["total_iters"]
    relerr = float(infos[0]["rel_error"]) if ref is not None else None
    curve = plan.trace(0)[:, 5] if ref is not None else []

    plan.set_target(0.0)   # the full solve under the reference's stopping rules alone
    full_t, full_info = cx.event_time(lambda: solve(plan), 2)
    stencils = stencil_roofline(plan, spec, w, ut=uts is not None)
    plan.close()

    plan_plain = capi.Plan([spec], [opts], graph=False, tune=a.tune)   # host-driven loop, same kernels
    plan_plain.set_target(target)
    cx.event_time(lambda: solve(plan_plain), 1)
    pt, _ = cx.event_time(lambda: solve(plan_plain), 2)
    plan_plain.close()

    et, ec = [], []   # end to end through the host-buffer C ABI (two untimed calls first)
    for k in range(max(1, min(a.steps, 3)) + 2):
        t0 = time.perf_counter()
        if a.tune:   # the batch entry point takes the flags (one instance)
            _, e_infos = capi.solve_batch([spec], [b_host], [opts], tune=True)
            e_info = e_infos[0]
        else:
            _, e_info = capi.solve(spec, b_host, opts)
        if k > 1:
            et.append((time.perf_counter() - t0) * 1000)
            ec.append(e_info["secs"] * 1000)
    e2e_ms = float(np.mean(et))
    in_bytes = int(b_host.nbytes + sum(x.nbytes for x in spec.keep))

    extra = ring_variants(a, cx, capi, ref) if name == "ring2d" else {}
    if name == "ring2d" and not a.no_batch:
        # the metric's "batched vs plain" on the mixed batch (cfg3(i) of the
        # reference configurations), measured in the same run
        extra["batch"] = batch_measure(a, cx, capi, dist)
        if world == 1:
            extra["configs"] = other_configs(a, cx, capi, rank, clocks)

    line = {"metric": METRIC, "value": world * 1000.0 / ms, "unit": "reconstructions/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded phantom and operator, Gaussian noise)",
            "config": dict(CONFIGS[name], instances=1, l2="256 MB write between timed solves",
                           launch_shape=launch_shape(capi, spec) if a.tune else "built-in",
                           **({"workload": f"2D dense {a.side}x{a.side}, A {spec.p.m}x{spec.p.n_cols} N(0,1/m), "
                                           f"iso TV (not the 64x64 configuration)"} if custom else {})),
            "iterations": iters, "time_to_solution_ms": ms, "relerr_vs_fp64": relerr,
            "fp64_noise_floor": float(ref["noise_floor"][0]) if ref is not None and "noise_floor" in ref else None,
            "reached_target": bool(relerr is not None and relerr <= target), "target": target,
            "relerr_curve_every_5": [round(float(x), 6) for x in curve[::5]],
            "full_solve": {"ms": float(np.mean(full_t)), "iterations": full_info[0]["total_iters"],
                           "relerr_vs_fp64": float(full_info[0]["rel_error"]) if ref is not None else None,
                           "rule": "reference stopping rules (tol, tol_inn, maxit)"},
            "plain": {"value": world * 1000.0 / float(np.mean(pt)), "unit": "reconstructions/s",
                      "ms_per_step": float(np.mean(pt)), "form": "host-driven loop, one launch per kernel"},
            "e2e": {"value": world * 1000.0 / e2e_ms, "unit": "reconstructions/s", "h2d_bytes_per_step": in_bytes,
                    "d2h_bytes_per_step": int(spec.n * 4), "ms_each": [round(x, 3) for x in et],
                    "ms_inside_library": [round(x, 3) for x in ec]},
            "roofline": dict(kernel_roofline(cx, capi, spec, w, w["kind"]), stencils=stencils),
            "clocks": clk, "gpu_launches": launches}
    line.update(extra)
    if cpu and rank == 0 and world == 1 and name != "hemi3d":
        out = reference_solve(w)
        if out:
            secs, r = out
            err = rel_l2(r.U, ref["U_aniso"]) if ref is not None and "U_aniso" in ref else None
            line["cpu_baseline"] = {"value": 1.0 / secs, "unit": "reconstructions/s", "cores": os.cpu_count(),
                                    "kind": "reference",
                                    "sample": f"one complete solve of the reference solver (anisotropic TV, float, "
                                              f"{'CSR twin' if w['kind'] != 'dense' else 'dense'}, its own stopping "
                                              f"rules): {r.total_iters} iterations"
                                              + (f", relerr vs the FP64 anisotropic solution {err:.2e}"
                                                 if err is not None else "")}
    return line


def other_configs(a, cx, capi, rank, clocks):
    """Compact records of the other reference configurations, measured in the
    default run on one GPU with their own workloads' shapes (two timed steps
    each after at least three warm-up ones): the plain dense 64x64 solve, the
    3D 128^3 hemisphere, the multi-RHS dense solve (joint and independent
    right-hand sides) and the differentiable unrolled solve."""
    import copy
    b = copy.copy(a)
    b.steps, b.warmup, b.maxit, b.side, b.sampling = 2, 3, None, 64, 0.3
    b.no_batch, b.tune, b.profile, b.plain = True, False, False, False
    keep = ("value", "unit", "ms_per_step", "iterations", "relerr_vs_fp64", "fp64_noise_floor", "reached_target",
            "full_solve", "clocks")
    out = {}
    for name in ("dense2d", "hemi3d"):
        t0 = time.perf_counter()
        r = run_single(b, cx, capi, name, 1, rank, None, clocks, cpu=False)
        rec = {k: r[k] for k in keep}
        rec["workload"] = r["config"]["workload"]
        rec["e2e"] = {k: r["e2e"][k] for k in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step")}
        rl = r["roofline"]
        rec["roofline"] = {k: rl.get(k) for k in ("bound", "kernel", "achieved", "peak", "unit", "frac",
                                                   "ms_per_launch", "peak_source")}
        rec["roofline"]["stencils"] = rl.get("stencils")
        rec["wall_s"] = round(time.perf_counter() - t0, 1)
        out["dense64" if name == "dense2d" else "hemi128"] = rec
    t0 = time.perf_counter()
    r = run_mrhs(b, cx, capi, 1, None, clocks)
    out["mrhs"] = {k: r[k] for k in ("value", "unit", "ms_per_step", "iterations", "relerr_vs_fp64",
                                     "relerr_per_rhs_max", "reached_target", "gemv_path", "tensor_over_gemv",
                                     "independent", "clocks")}
    out["mrhs"]["workload"] = r["config"]["workload"]
    out["mrhs"]["roofline"] = {k: r["roofline"][k] for k in ("kernel", "achieved", "frac", "ms_per_launch",
                                                              "tensor_tflops")}
    out["mrhs"]["wall_s"] = round(time.perf_counter() - t0, 1)
    t0 = time.perf_counter()
    r = run_unrolled(b, cx, capi, 1, None, clocks)
    out["unrolled"] = {k: r[k] for k in ("value", "unit", "ms_per_step", "forward_ms", "backward_ms", "loss",
                                         "clocks")}
    out["unrolled"]["workload"] = r["config"]["workload"]
    out["unrolled"]["wall_s"] = round(time.perf_counter() - t0, 1)
    out["f64"] = f64_records(capi)
    return out


def f64_records(capi):
    """The double-data path (tval3g_solve_f64, the FP64 build of the engine
    behind the reference's double overloads) end to end on the ring and the
    dense 64x64 workloads, host buffers, the reference's stopping rules: mean
    wall time of three calls after one, iterations and relerr against the
    FP64 oracle's solution (tests/golden)."""
    out = {}
    for name in ("ring2d", "dense2d"):
        w = workload(name)
        spec = capi.problem_from_workload(w)
        vals = np.asarray(w["A"], np.float64) if w["kind"] == "dense" else None
        b = np.asarray(w["b"], np.float64)
        ref = fp64_reference(name)
        capi.solve_f64(spec, b, w["opts"], values=vals)
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            U, info = capi.solve_f64(spec, b, w["opts"], values=vals)
            ts.append((time.perf_counter() - t0) * 1000)
        ms = float(np.mean(ts))
        out["ring256" if name == "ring2d" else "dense64"] = {
            "value": 1000.0 / ms, "unit": "reconstructions/s", "ms_per_call": ms, "iterations": info["total_iters"],
            "fp64_oracle_iterations": int(ref["iters"][1]) if ref is not None else None,
            "relerr_vs_fp64": rel_l2(U, ref["U"]) if ref is not None else None,
            "what": "tval3g_solve_f64 with host buffers (operator preparation included), double storage"}
    return out


def timed_plan(cx, capi, spec, opts, b, Ut=None, target=0.0, reps=3):
    """Mean CUDA-event time of `reps` solves of a one-instance graph plan
    (after one untimed solve), with the last solve's info."""
    torch, dev, s = cx.torch, cx.dev, cx.stream.cuda_stream
    d_b = torch.tensor(np.ascontiguousarray(b, np.float32), device=dev)
    d_U = torch.empty(spec.n, device=dev)
    uts = [torch.tensor(np.ascontiguousarray(Ut, np.float32).ravel(), device=dev)] if Ut is not None else None
    plan = capi.Plan([spec], [opts], graph=True, trace=Ut is not None)
    plan.set_target(target)
    run = lambda: plan.solve([d_b], [d_U], d_Ut=uts, stream=s)  # noqa: E731
    cx.event_time(run, 1)
    ts, infos = cx.event_time(run, reps)
    plan.close()
    return float(np.mean(ts)), infos[0], d_U.cpu().numpy()


def ring_variants(a, cx, capi, ref):
    """Sub-records of the ring workload: the anisotropic problem (the one the
    reference solves: it has no isotropic TV) and the literal unit-weight
    configuration for a fixed 20 iterations."""
    from tval3g import workloads as W
    out = {}
    if ref is None:
        return out
    w = W.ring2d(seed=1, side=256, T=512, tv_norm=0, maxit=500, tol=1e-5, normalize=True)
    spec = capi.problem_from_workload(w)
    t_ms, t_info, _ = timed_plan(cx, capi, spec, w["opts"], w["b"], Ut=ref["U_aniso"], target=1e-3)
    f_ms, f_info, U = timed_plan(cx, capi, spec, w["opts"], w["b"])
    out["aniso"] = {"time_to_solution_ms": t_ms, "iterations_to_target": t_info["total_iters"],
                    "relerr_at_target": float(t_info["rel_error"]),
                    "reached_target": bool(t_info["rel_error"] <= 1e-3),
                    "full_solve_ms": f_ms, "full_solve_iterations": f_info["total_iters"],
                    "full_solve_relerr_vs_fp64": rel_l2(U, ref["U_aniso"]),
                    "fp64_iterations": int(ref["iters_aniso"][1]),
                    "fp64_noise_floor": float(ref["noise_floor_aniso"][0]) if "noise_floor_aniso" in ref else None,
                    "value": 1000.0 / t_ms, "unit": "reconstructions/s",
                    "what": "the same ring workload with anisotropic TV (the reference arm's problem), "
                            "time to relerr <= 1e-3 vs the FP64 anisotropic solution and the full solve"}
    wu = W.ring2d(seed=1, side=256, T=512, tv_norm=1, maxit=20, tol=1e-5, normalize=False)
    spec = capi.problem_from_workload(wu)
    u_ms, u_info, U = timed_plan(cx, capi, spec, wu["opts"], wu["b"])
    out["unit_weight"] = {"ms_20_iterations": u_ms, "iterations": u_info["total_iters"],
                          "relerr_vs_fp64_20_iterations": rel_l2(U, ref["U_unit20"]),
                          "what": "the literal configuration (weight 1 per hit), a fixed 20 iterations, against "
                                  "the FP64 oracle's first 20 iterations"}
    return out


def run_mrhs(a, cx, capi, world, dist, clocks):
    """Joint multi-RHS solve: the tensor-core product against the
    FP64-accumulating gemv kernels, both as CUDA graphs."""
    from tval3g import workloads as W
    torch, dev, stream = cx.torch, cx.dev, cx.stream
    w = W.mrhs()
    N, (m, n) = w["layers"], w["A"].shape
    d_A = torch.tensor(w["A"], device=dev)
    spec = capi.dense_problem(w["shape"], w["A"], layers=N, device_ptr=d_A.data_ptr())
    opts = dict(w["opts"])
    d_b = torch.tensor(w["b"], device=dev)
    d_U = torch.empty(spec.n, device=dev)
    if a.maxit is not None:
        opts["maxit"] = a.maxit
    if a.profile:
        plan = capi.Plan([spec], [opts], graph=not a.plain, device_inputs=True)
        cx.event_time(lambda: plan.solve([d_b], [d_U], stream=stream.cuda_stream), a.warmup + a.steps)
        plan.close()
        return None
    ref = fp64_reference("mrhs")
    d_ref = torch.tensor(ref["U"].ravel(), device=dev) if ref is not None else None
    target = 1e-3 if ref is not None else 0.0
    res = {}
    for tensor in (True, False):
        plan = capi.Plan([spec], [opts], graph=True, device_inputs=True, tensor=tensor)
        plan.set_target(target)
        run = lambda: plan.solve([d_b], [d_U], d_Ut=[d_ref] if d_ref is not None else None,  # noqa: E731
                                 stream=stream.cuda_stream)
        cx.event_time(run, max(a.warmup, 3) if tensor else 1)
        if tensor:
            if dist:
                dist.barrier()
            clocks.start()
        ts, infos = cx.event_time(run, a.steps if tensor else 2)
        if tensor:
            clk = clocks.stop()
            launches = plan.stats()["kernel_launches"] * a.steps
            U = d_U.cpu().numpy().reshape(N, -1)
        res[tensor] = (float(np.mean(ts)), infos[0])
        plan.close()
    ms, info = res[True]
    ms = max_over_ranks(dist, [ms], dev)[0]
    per_rhs = None
    if ref is not None:
        R = ref["U"].reshape(N, -1)
        per_rhs = [float(np.linalg.norm(U[k] - R[k]) / np.linalg.norm(R[k])) for k in range(N)]
    indep = mrhs_independent(a, cx, capi, w, d_A, d_b)
    # the product alone: forward (split + tcgen05 kernel + reduce), L2 flushed
    op = capi.Operator(spec, tensor=True, device_inputs=True)
    x = torch.rand(op.cols, device=dev)
    y = torch.empty(op.rows, device=dev)
    op.apply_n(x, y, 3, stream=stream.cuda_stream)
    kt, _ = cx.event_time(lambda: op.apply_n(x, y, 1, stream=stream.cuda_stream), 10)
    zt, _ = cx.event_time(lambda: op.apply_n(y, x, 1, trans=True, stream=stream.cuda_stream), 10)
    op.close()
    k_ms = float(np.mean(kt))
    bytes_ = 4 * m * n + 4 * N * (m + n)
    peak, src = peak_hbm()
    achieved = bytes_ / (k_ms * 1e-3) / 1e9
    return {"metric": METRIC, "value": world * N * 1000.0 / ms, "unit": "reconstructions/s (right-hand sides)",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 data, 3xTF32 products",
            "data": "synthetic (seeded A, phantoms, noise)",
            "config": dict(CONFIGS["mrhs"], rhs=N, l2="256 MB write between timed solves"),
            "iterations": info["total_iters"], "relerr_vs_fp64": float(info["rel_error"]) if ref is not None else None,
            "relerr_per_rhs_max": max(per_rhs) if per_rhs else None,
            "relerr_per_rhs": [round(e, 6) for e in per_rhs] if per_rhs else None,
            "reached_target": bool(ref is not None and info["rel_error"] <= target), "target": target,
            "gemv_path": {"ms_per_step": res[False][0], "iterations": res[False][1]["total_iters"],
                          "relerr_vs_fp64": float(res[False][1]["rel_error"]) if ref is not None else None,
                          "form": "same graph, FP64-accumulating gemv kernels, A read once per layer"},
            "tensor_over_gemv": res[False][0] / ms, "independent": indep,
            "roofline": {"bound": "hbm", "kernel": "k_mrhs_split + k_mrhs<32> + k_mrhs_red (A X^T)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": profile_traffic("mrhs_tcgen05_4096x16384.md"), "algorithmic_bytes": bytes_,
                         "ms_per_launch": k_ms, "adjoint_ms_per_launch": float(np.mean(zt)),
                         "tensor_tflops": 3 * 2 * m * n * N / (k_ms * 1e-3) / 1e12, "peak_source": src,
                         "timing": "one launch per CUDA-event pair, 256 MB L2 flush before each"},
            "clocks": clk, "gpu_launches": launches}


def run_unrolled(a, cx, capi, world, dist, clocks):
    """A step is one forward (K = 50 iterations, 8 instances) and one
    backward (the gradients of the loss w.r.t. b, mu_k and beta_k) through
    tval3g_unrolled_*; reported as differentiated reconstructions per second."""
    from tval3g import workloads as W
    torch, dev, s = cx.torch, cx.dev, cx.stream.cuda_stream
    side, T, count, K, ckpt = 128, 256, 8, 50, 10
    ws = [W.ring2d(seed=11 + i, side=side, T=T, tv_norm=1, normalize=True) for i in range(count)]
    spec = capi.ray2d_problem((side, side), ws[0]["geom"])
    opts = W.options(2 ** 8, 2 ** 5, 1e-4, K, tv_norm=1)
    h = capi.Unrolled(spec, count, opts, K, ckpt=ckpt)
    mu, beta = 2.0 ** 8 * np.ones(K), 2.0 ** 5 * np.ones(K)
    d_b = [torch.tensor(w["b"].astype(np.float32), device=dev) for w in ws]
    d_ut = [torch.tensor(w["u_true"].ravel().astype(np.float32), device=dev) for w in ws]
    d_U = [torch.empty(spec.n, device=dev) for _ in range(count)]
    d_gU = [torch.empty(spec.n, device=dev) for _ in range(count)]
    d_gb = [torch.empty(len(w["b"]), device=dev) for w in ws]

    def fwd():
        h.forward(d_b, mu, beta, d_U, stream=s)

    def bwd():
        for u, t, gu in zip(d_U, d_ut, d_gU):
            torch.sub(u, t, out=gu)   # d loss / d U for 0.5 |U - u_true|^2
        return h.backward(d_gU, d_gb, stream=s)

    for _ in range(max(a.warmup, 3)):
        fwd()
        bwd()
    if dist:
        dist.barrier()
    clocks.start()
    tf, tb = [], []
    for _ in range(a.steps):
        t1, _ = cx.event_time(fwd, 1)
        t2, g = cx.event_time(bwd, 1)
        tf += t1
        tb += t2
    clk = clocks.stop()
    ms_f, ms_b = max_over_ranks(dist, [float(np.mean(tf)), float(np.mean(tb))], dev)
    loss = float(sum(0.5 * float(torch.sum((u - t) ** 2)) for u, t in zip(d_U, d_ut)))
    h.close()
    ms = ms_f + ms_b
    return {"metric": METRIC, "value": world * count * 1000.0 / ms, "unit": "differentiated reconstructions/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 scalar reductions)",
            "data": "synthetic (seeded phantoms, noise)",
            "config": dict(CONFIGS["unrolled"], instances=count, K=K, checkpoint=ckpt,
                           l2="256 MB write before each timed call"),
            "forward_ms": ms_f, "backward_ms": ms_b, "loss": loss,
            "grad_mu_norm": float(np.linalg.norm(g[0])), "grad_beta_norm": float(np.linalg.norm(g[1])),
            "clocks": clk}


def mrhs_independent(a, cx, capi, w, d_A, d_b):
    """The 32 right-hand sides solved independently: 32 one-layer instances
    of one plan sharing the device matrix, so that every product of the
    group is one tensor-core contraction while each instance keeps its own
    scaling, step lengths, line search and stopping; against the same plan
    on the FP64-accumulating gemv kernels and against each right-hand side's
    FP64 solution (tests/golden/mrhs32_indep_fp64.npz)."""
    torch, dev, s = cx.torch, cx.dev, cx.stream.cuda_stream
    N, (m, n) = w["layers"], w["A"].shape
    side = int(round(np.sqrt(n)))
    specs = [capi.dense_problem((side, side), w["A"], device_ptr=d_A.data_ptr()) for _ in range(N)]
    bs = [d_b[k * m:(k + 1) * m] for k in range(N)]
    us = [torch.empty(n, device=dev) for _ in range(N)]
    fx = os.path.join(GOLDEN, "mrhs32_indep_fp64.npz")
    fx = dict(np.load(fx)) if os.path.exists(fx) else None
    uts = [torch.tensor(fx["U"][k], device=dev) for k in range(N)] if fx is not None else None
    out = {}
    for tensor in (True, False):
        plan = capi.Plan(specs, [w["opts"]] * N, graph=True, device_inputs=True, tensor=tensor)
        run = lambda: plan.solve(bs, us, d_Ut=uts, stream=s)  # noqa: E731
        cx.event_time(run, 1)
        ts, infos = cx.event_time(run, max(1, min(a.steps, 3)))
        plan.close()
        rel = [float(i["rel_error"]) for i in infos] if uts is not None else None
        its = [i["total_iters"] for i in infos]
        out["tensor" if tensor else "gemv"] = {
            "ms_per_step": float(np.mean(ts)), "value": N * 1000.0 / float(np.mean(ts)),
            "unit": "reconstructions/s (right-hand sides)", "iterations_min_max": [min(its), max(its)],
            "relerr_vs_fp64_max": max(rel) if rel else None,
            "relerr_vs_fp64_per_rhs": [round(e, 6) for e in rel] if rel else None,
            "iterations_vs_fp64": [[i, int(fx["iters"][k][1])] for k, i in enumerate(its)] if fx is not None else None}
    out["form"] = ("32 one-layer instances of one plan sharing the device matrix (per-instance control); 'tensor': "
                   "each product of the group one tcgen05 3xTF32 contraction; 'gemv': FP64-accumulating gemv "
                   "kernels per instance")
    return out


def batch_problems(capi, torch, dev):
    """Materialise the mixed batch: each dense A drawn on the device from its
    instance seed (tval3g_gaussian; the oracle regenerates the same stream on
    the host), b from the library's dense forward; ring geometries and data
    on the host."""
    from tval3g import workloads as W
    specs, opts, bs, keep = [], [], [], []
    for k, d in enumerate(W.batch_specs()):
        if d["kind"] == "dense":
            p = W.batch_dense_parts(d)
            A = torch.empty(p["m"], p["n"], device=dev)
            capi.gaussian(A, d["seed"], p["scale"])
            spec = capi.dense_problem(p["shape"], A, device_ptr=A.data_ptr())
            op = capi.Operator(spec, device_inputs=True)
            y = torch.empty(p["m"], device=dev)
            op.apply(torch.tensor(p["u_true"].ravel().astype(np.float32), device=dev), y)
            op.close()
            b = W.add_noise(y.cpu().numpy().astype(np.float64), 0.01, p["rng"]).astype(np.float32)
            keep.append(A)
            o = p["opts"]
        else:
            w = W.batch_ray(d)
            spec, b, o = capi.ray2d_problem(w["shape"], w["geom"]), w["b"], w["opts"]
        specs.append(spec)
        bs.append(torch.tensor(np.ascontiguousarray(b, np.float32), device=dev))
        opts.append(o)
    return specs, opts, bs, keep


def batch_measure(a, cx, capi, dist, clocks=None, ray_subset=True):
    """The mixed batch of 64 independent 2D problems: the batched graph (one
    plan, one launch per kernel over all instances) against the plain form
    (one plan per instance, host-driven loop, instances in sequence), with
    each instance of the FP64 subset (tests/golden/batch_fp64.npz) checked
    against its FP64 solution."""
    torch, dev, stream = cx.torch, cx.dev, cx.stream
    specs, opts, bs, keep = batch_problems(capi, torch, dev)
    us = [torch.empty(s.n, device=dev) for s in specs]
    nb = len(specs)
    fx = os.path.join(GOLDEN, "batch_fp64.npz")
    fx = dict(np.load(fx)) if os.path.exists(fx) else {}
    uts = [None] * nb
    for k in range(nb):
        if f"U{k}" in fx:
            uts[k] = torch.tensor(fx[f"U{k}"].ravel().astype(np.float32), device=dev)
    have_ut = [k for k in range(nb) if uts[k] is not None]
    plan = capi.Plan(specs, opts, graph=True, device_inputs=True)
    solve = lambda: plan.solve(bs, us, d_Ut=uts, stream=stream.cuda_stream)  # noqa: E731
    cx.event_time(solve, max(1, min(a.warmup, 2)))
    if dist:
        dist.barrier()
    if clocks:
        clocks.start()
    tb, infos = cx.event_time(solve, max(1, min(a.steps, 3)))
    launches = plan.stats()["kernel_launches"]
    clk = clocks.stop() if clocks else None
    ms_b = float(np.mean(tb))
    device_bytes = plan.stats()["device_bytes"]
    plan.close()
    rel = {k: float(infos[k]["rel_error"]) for k in have_ut}
    fp64_iters = {k: int(fx[f"iters{k}"][1]) for k in have_ut}
    floors = {k: float(fx[f"floor{k}"][0]) for k in have_ut if f"floor{k}" in fx}
    # plain: one instance per plan, host-driven loop, instances one after another
    singles = [capi.Plan([s], [o], graph=False, device_inputs=True) for s, o in zip(specs, opts)]

    def plain():
        for p, b, u in zip(singles, bs, us):
            p.solve([b], [u], stream=stream.cuda_stream)
    cx.event_time(plain, 1)
    tp, _ = cx.event_time(plain, 1)
    for p in singles:
        p.close()
    ms_b, ms_p = max_over_ranks(dist, [ms_b, float(np.mean(tp))], dev)
    iters = [i["total_iters"] for i in infos]
    dense = sum(1 for s in specs if s.p.op_kind == capi.OP_DENSE)
    dense_bytes = sum(4 * s.p.m * s.p.n_cols for s in specs if s.p.op_kind == capi.OP_DENSE)
    # HBM floor of the dense instances: A read once per iteration (the
    # one-pass normal product) plus the initial A^T b, at the measured copy rate
    peak, _ = peak_hbm()
    floor_ms = sum(4.0 * s.p.m * s.p.n_cols * (it + 1) for s, it in zip(specs, iters)
                   if s.p.op_kind == capi.OP_DENSE) / (peak * 1e9) * 1e3
    # the ray instances alone: where batching removes launch and latency cost
    rays = [k for k, s in enumerate(specs) if s.p.op_kind != capi.OP_DENSE]
    sub = {}
    if rays and ray_subset:
        rplan = capi.Plan([specs[k] for k in rays], [opts[k] for k in rays], graph=True, device_inputs=True)
        rsolve = lambda: rplan.solve([bs[k] for k in rays], [us[k] for k in rays], stream=stream.cuda_stream)  # noqa: E731
        cx.event_time(rsolve, 1)
        trb, _ = cx.event_time(rsolve, 2)
        rplan.close()
        rsingles = [capi.Plan([specs[k]], [opts[k]], graph=False, device_inputs=True) for k in rays]

        def rplain():
            for p, k in zip(rsingles, rays):
                p.solve([bs[k]], [us[k]], stream=stream.cuda_stream)
        cx.event_time(rplain, 1)
        trp, _ = cx.event_time(rplain, 1)
        for p in rsingles:
            p.close()
        sub = {"instances": len(rays), "batched_ms": float(np.mean(trb)), "plain_ms": float(np.mean(trp)),
               "batched_over_plain": float(np.mean(trp)) / float(np.mean(trb))}
    # the one-pass dense normal product A^T (A u) on the batch's largest matrix
    big = max((k for k, s_ in enumerate(specs) if s_.p.op_kind == capi.OP_DENSE),
              key=lambda k: specs[k].p.m * specs[k].p.n_cols, default=None)
    normal = None
    if big is not None:
        sp = specs[big]
        op = capi.Operator(sp, device_inputs=True)
        xv, yv = torch.rand(op.cols, device=dev), torch.empty(op.cols, device=dev)
        op.apply_n(xv, yv, 2, trans=2, stream=stream.cuda_stream)
        tn, _ = cx.event_time(lambda: op.apply_n(xv, yv, 1, trans=2, stream=stream.cuda_stream), 5)
        op.close()
        a_bytes = 4.0 * sp.p.m * sp.p.n_cols + 4.0 * (2 * sp.p.n_cols + 2 * sp.p.m)
        t_ms = float(np.mean(tn))
        normal = {"m": sp.p.m, "n": sp.p.n_cols, "ms_per_launch": t_ms,
                  "achieved_gbs": a_bytes / (t_ms * 1e-3) / 1e9, "frac": a_bytes / (t_ms * 1e-3) / 1e9 / peak,
                  "kernel": "k_dense_normal (A read once: Au and A^T Au)"}
    del keep
    return {"instances": nb, "dense_instances": dense, "dense_bytes": int(dense_bytes),
            "dense_normal_largest": normal,
            "plan_device_bytes": int(device_bytes), "batched_ms": ms_b, "plain_ms": ms_p,
            "batched_over_plain": ms_p / ms_b, "value": nb * 1000.0 / ms_b, "unit": "reconstructions/s",
            "plain_value": nb * 1000.0 / ms_p, "iterations_min_max": [min(iters), max(iters)],
            "dense_hbm_floor_ms": floor_ms, "batched_over_floor": ms_b / floor_ms,
            "relerr_vs_fp64": {"instances_checked": len(rel), "max": max(rel.values()) if rel else None,
                               "within_1e-3": sum(1 for v in rel.values() if v <= 1e-3),
                               "within_noise_bar": sum(1 for k, v in rel.items() if k in floors and
                                                       v <= max(1e-3, 2 * floors[k])),
                               "noise_bar": "max(1e-3, 2 x the instance's FP32 noise floor: how far its FP64 "
                                            "solve moves under a few FP32 roundings per stored element and "
                                            "iteration)",
                               "fp32_noise_floor": {str(k): round(v, 6) for k, v in floors.items()},
                               "per_instance": {str(k): round(v, 6) for k, v in rel.items()},
                               "iterations_gpu_vs_fp64": {str(k): [iters[k], fp64_iters[k]] for k in rel},
                               "subset": "the ring instances of side <= 192 and the dense ones of side <= 96 "
                                         "(tests/golden/batch_fp64.npz)"},
            "ray_instances_only": sub, "clocks": clk, "gpu_launches": launches}


def run_batch(a, cx, capi, world, dist, clocks):
    r = batch_measure(a, cx, capi, dist, clocks)
    return {"metric": METRIC, "value": world * r["value"], "unit": "reconstructions/s", "n_gpus": world,
            "steps": max(1, min(a.steps, 3)), "warmup": max(1, min(a.warmup, 2)), "ms_per_step": r["batched_ms"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded phantoms and operators)",
            "config": dict(CONFIGS["batch"], instances=r["instances"], dense_instances=r["dense_instances"],
                           dense_bytes=r["dense_bytes"], plan_device_bytes=r["plan_device_bytes"]),
            "plain": {"value": world * r["plain_value"], "unit": "reconstructions/s", "ms_per_step": r["plain_ms"],
                      "form": "one plan per instance, host-driven loop, instances in sequence"},
            "batched_over_plain": r["batched_over_plain"], "iterations_min_max": r["iterations_min_max"],
            "dense_hbm_floor_ms": r["dense_hbm_floor_ms"], "batched_over_floor": r["batched_over_floor"],
            "dense_normal_largest": r["dense_normal_largest"],
            "relerr_vs_fp64": r["relerr_vs_fp64"], "ray_instances_only": r["ray_instances_only"],
            "clocks": r["clocks"], "gpu_launches": r["gpu_launches"]}


def main():
    a = args_()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl" if a.impl == "tval3g" else "gloo", timeout=timedelta(seconds=600))
    if a.impl == "reference":
        run_reference(a, rank)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    import torch
    from tval3g import capi
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # a non-default stream: every kernel is launched on it and the CUDA
    # events are recorded on it
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    cx = Ctx(torch, dev, stream, torch.empty(64 * 1024 * 1024, device=dev))
    clocks = Clocks(local)
    if a.workload == "batch":
        line = run_batch(a, cx, capi, world, dist, clocks)
    elif a.workload == "mrhs":
        line = run_mrhs(a, cx, capi, world, dist, clocks)
    elif a.workload == "unrolled":
        line = run_unrolled(a, cx, capi, world, dist, clocks)
    else:
        line = run_single(a, cx, capi, a.workload, world, rank, dist, clocks)
    if rank == 0 and line is not None:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
