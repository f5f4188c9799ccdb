#!/usr/bin/env python
"""TVAL3 time-to-solution benchmark on B200 (one JSON line on rank 0).

Workload (default): the 2D ultrasound-tomography ring - 256x256 image, 512
transducers on the inscribed circle, each emitter firing at the 256 receivers
on the opposite half (131072 rays, 2.72e7 Bresenham hits), isotropic TV,
mu=2^10, beta=2^6, tol=1e-5, maxit=500 - on the on-the-fly Bresenham
projector.  A step is one full reconstruction (scaleb, A^T b, the whole
continuation / inner loop, final scaling) through a device-resident plan whose
iteration loop is one CUDA graph.

  value   reconstructions/s with inputs resident in HBM (CUDA events around
          each solve on the launching stream; 256 MB L2 flush between solves)
  e2e     the same through the host-buffer C ABI tval3g_solve (geometry and b
          from host memory, U back to host; includes the per-call operator
          preparation), host clock around the blocking call
  roofline  the dominant kernel (ray adjoint gather) timed with CUDA events
  cpu_baseline  the reference solver itself (oracle/_ref, compiled from its
          own sources) on the CSR twin, on a bounded sample of iterations

--impl reference runs only the reference CPU solver on the same workload.
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
FIXTURE = os.path.join(ROOT, "tests", "golden", "ring256_fp64.npz")


def args_():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="tval3g", choices=["tval3g", "reference"])
    p.add_argument("--cpu-sample-iters", type=int, default=20)
    p.add_argument("--profile", action="store_true",
                   help="for ncu: build the plan, run --warmup + --steps solves, print nothing else")
    p.add_argument("--maxit", type=int, default=None, help="override maxit (profiling a short solve)")
    p.add_argument("--plain", action="store_true",
                   help="with --profile: run the host-driven loop (same kernels, same order) instead of the "
                        "CUDA graph, whose conditional nodes ncu cannot profile kernel by kernel")
    return p.parse_args()


def workload():
    from tval3g import workloads as W
    return W.ring2d(seed=1, side=256, T=512, tv_norm=1, maxit=500, tol=1e-5, normalize=True)


def config_dict():
    return {"workload": "2D ring 256x256, 512 transducers x 256 receivers (131072 rays, 2.72e7 hits), iso TV, "
                        "mu 2^10, beta 2^6, tol 1e-5, maxit 500 (configs[1]); hit weight scale_factor = "
                        "1/sigma_max(A) so that mu and beta act as in TVAL3",
            "operator": "on-the-fly Bresenham projector (gather adjoint)", "instances": 1,
            "l2": "256 MB write between timed solves"}


def fp64_reference():
    if os.path.exists(FIXTURE):
        return dict(np.load(FIXTURE))
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
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
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
def reference_rate(w, sample_iters, full_iters):
    """Seconds per reconstruction of the reference's own solver (float data,
    CSR twin, all host threads), from a bounded sample of iterations scaled to
    the iteration count of a full solve."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.ref_available(2):
        return None
    A = w["csr"]
    o = dict(w["opts"])
    o["maxit"] = sample_iters
    o["tv_norm"] = 0
    cwd = os.getcwd()
    t0 = time.perf_counter()
    r = O.ref_solve("csr", w["shape"], w["b"], o, dtype=0, csr=(A["m"], A["n"], A["rowptr"], A["colind"], A["val"]),
                    vppc=1)
    os.chdir(cwd)
    secs = time.perf_counter() - t0
    per_iter = secs / max(r.total_iters, 1)
    return {"secs_per_iter": per_iter, "secs_per_solve": per_iter * full_iters, "sample_iters": r.total_iters,
            "cores": os.cpu_count()}


def run_reference(a, rank):
    if rank != 0:
        return
    w = workload()
    ref = fp64_reference()
    full_iters = int(ref["iters"][1]) if ref is not None else int(w["opts"]["maxit"])
    for _ in range(a.warmup):
        reference_rate(w, a.cpu_sample_iters, full_iters)
    rates = []
    for _ in range(a.steps):
        r = reference_rate(w, a.cpu_sample_iters, full_iters)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (reference sources "
                                                                  "absent when building)"}))
            return
        rates.append(r["secs_per_solve"])
    ms = float(np.mean(rates)) * 1000
    val = 1000.0 / ms
    line = {"metric": METRIC, "value": val, "unit": "reconstructions/s", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "config": config_dict(), "impl": "reference",
            "cpu_baseline": {"value": val, "unit": "reconstructions/s", "cores": r["cores"], "kind": "reference",
                             "sample": f"{r['sample_iters']} iterations of the reference solver (anisotropic TV: it "
                                       f"has no isotropic TV) on the CSR twin, scaled to {full_iters} iterations"},
            "e2e": {"value": val, "unit": "reconstructions/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# --------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------
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
    w = workload()
    spec = capi.ray2d_problem(w["shape"], w["geom"])
    opts = dict(w["opts"])
    if a.maxit is not None:
        opts["maxit"] = a.maxit
    b_host = np.ascontiguousarray(w["b"], np.float32)
    # a non-default stream: every kernel of the solve is launched on it and
    # the CUDA events below are recorded on it
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    d_b = torch.tensor(b_host, device=dev)
    d_U = torch.empty(spec.n, device=dev)
    flush = torch.empty(64 * 1024 * 1024, device=dev)
    ref = fp64_reference()
    # time-to-solution: stop at the first iteration within 1e-3 of the FP64
    # solution (given as Ut), else by the reference's own stopping rules
    d_ref = torch.tensor(ref["U"].ravel().astype(np.float32), device=dev) if ref is not None else None
    target = 1e-3 if ref is not None else 0.0

    plan = capi.Plan([spec], [opts], graph=not (a.profile and a.plain), trace=True)
    plan.set_target(target)

    def solve_timed(p, reps):
        out, inf = [], None
        for _ in range(reps):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            inf = p.solve([d_b], [d_U], d_Ut=[d_ref] if d_ref is not None else None, stream=stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            out.append(e0.elapsed_time(e1))
        return out, inf

    if a.profile:
        solve_timed(plan, a.warmup + a.steps)
        plan.close()
        return
    solve_timed(plan, max(a.warmup, 3))

    clocks = Clocks(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    times, launches, infos = [], 0, None
    for _ in range(a.steps):
        t1, infos = solve_timed(plan, 1)
        times += t1
        launches += plan.stats()["kernel_launches"]
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms = float(np.mean(times))
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * 1000.0 / ms
    iters = infos[0]["total_iters"]
    relerr = float(infos[0]["rel_error"]) if ref is not None else None
    curve = plan.trace(0)[:, 5]

    # the full solve under the reference's stopping rules alone
    plan.set_target(0.0)
    full_t, full_info = solve_timed(plan, 2)
    full_relerr = float(full_info[0]["rel_error"]) if ref is not None else None

    # the plain (host-driven, no graph) form of the same time-to-solution
    plan_plain = capi.Plan([spec], [opts], graph=False)
    plan_plain.set_target(target)
    solve_timed(plan_plain, 1)
    pt, _ = solve_timed(plan_plain, 2)
    plan_plain.close()

    # end to end through the host-buffer C ABI
    et = []
    for k in range(max(1, min(a.steps, 3)) + 1):
        t0 = time.perf_counter()
        Uh, info_h = capi.solve(spec, b_host, opts)
        if k > 0:
            et.append((time.perf_counter() - t0) * 1000)
    geom_bytes = sum(np.asarray(w["geom"][k]).astype(np.int32).nbytes for k in ("use_path", "xe", "ye", "xr", "yr"))
    e2e_ms = float(np.mean(et))

    # dominant kernels, timed alone with CUDA events on their stream
    op = capi.Operator(spec)
    x = torch.rand(op.cols, device=dev)
    y = torch.rand(op.rows, device=dev)
    out_m = torch.empty(op.rows, device=dev)
    out_n = torch.empty(op.cols, device=dev)
    # each launch timed alone after an L2 flush, so its index comes from HBM
    kt = {}
    for name, (src, dst, tr) in {"ray_forward": (x, out_m, False), "ray_adjoint": (y, out_n, True)}.items():
        op.apply_n(src, dst, 3, trans=tr, stream=stream.cuda_stream)
        ts = []
        for _ in range(10):
            flush.fill_(1.0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            op.apply_n(src, dst, 1, trans=tr, stream=stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        kt[name] = float(np.mean(ts))
    nnz, n, m = op.nnz, op.cols, op.rows
    nrays = int(np.count_nonzero(w["geom"]["use_path"]))
    nchunks = -(-nrays // 32768)
    # algorithmic bytes of the staged adjoint (compaction + gather): the
    # measurement vector read once, the traced-ray vector written and read
    # once, the 16-bit pixel->ray index, the per-pixel chunk offsets, the image
    # written once
    adj_bytes = 4 * m + 8 * nrays + 2 * nnz + 4 * n * (nchunks + 1) + 4 * n
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = adj_bytes / (kt["ray_adjoint"] * 1e-3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "ray_adjoint_staged_ring256.md")
    if os.path.exists(prof):
        for line in open(prof):
            if line.startswith("traffic_bytes_per_launch:"):
                traffic = float(line.split(":")[1].split()[0])

    line = {"metric": METRIC, "value": value, "unit": "reconstructions/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded ring phantom, 0.5% noise)", "config": config_dict(),
            "iterations": iters, "time_to_solution_ms": ms, "relerr_vs_fp64": relerr,
            "reached_target": bool(relerr is not None and relerr <= target), "target": target,
            "relerr_curve_every_5": [round(float(x), 6) for x in curve[::5]],
            "full_solve": {"ms": float(np.mean(full_t)), "iterations": full_info[0]["total_iters"],
                           "relerr_vs_fp64": full_relerr, "rule": "reference stopping rules (tol, tol_inn, maxit)"},
            "plain": {"value": world * 1000.0 / float(np.mean(pt)), "unit": "reconstructions/s",
                      "ms_per_step": float(np.mean(pt)), "form": "host-driven loop, one launch per kernel"},
            "e2e": {"value": world * 1000.0 / e2e_ms, "unit": "reconstructions/s",
                    "h2d_bytes_per_step": int(b_host.nbytes + geom_bytes), "d2h_bytes_per_step": int(spec.n * 4)},
            "roofline": {"bound": "hbm", "kernel": "k_ray_compact + k_ray_adj_staged (ray adjoint)",
                         "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes": adj_bytes, "ms_per_launch": kt["ray_adjoint"],
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)",
                         "forward_ms_per_launch": kt["ray_forward"], "hits": nnz},
            "clocks": clk, "gpu_launches": launches}
    if rank == 0 and world == 1:
        full = ref["iters"][1] if ref is not None else iters
        cb = reference_rate(w, a.cpu_sample_iters, iters)
        if cb:
            line["cpu_baseline"] = {"value": 1.0 / cb["secs_per_solve"], "unit": "reconstructions/s",
                                    "cores": cb["cores"], "kind": "reference",
                                    "sample": f"{cb['sample_iters']} iterations of the reference solver "
                                              f"(anisotropic TV, CSR twin, float) scaled to {iters} iterations "
                                              f"(FP64 oracle solve: {int(full)})"}
    plan.close()
    op.close()
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
