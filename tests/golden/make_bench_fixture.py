"""FP64 solutions of the benchmark workloads (bench.py), for their relerr checks.

    python tests/golden/make_bench_fixture.py [ring] [dense64] [mrhs] [batch]

Solves the 256x256 ring workload (tval3g.workloads.ring2d with normalize=True,
isotropic TV, maxit 500) with the FP64 oracle restatement and stores U and the
iteration counts in tests/golden/ring256_fp64.npz (with its FP32 noise
floor: how far the FP64 solve moves under a few FP32 roundings per stored
element and iteration), together with the
anisotropic FP64 solution of the same problem (U_aniso: what the reference,
which has no isotropic TV, solves) and the first 20 iterations of the literal
unit-weight ring (normalize=False, U_unit20).  Also records the reference's
own float solver on the CSR twin of the same operator with anisotropic TV for
the drift statement.
The dense 64x64 workload goes to dense64_fp64.npz and the joint 32-layer
multi-RHS workload to mrhs32_fp64.npz, its 32 right-hand sides solved
independently to mrhs32_indep_fp64.npz.  The mixed batch's FP64 subset (its
ring instances of side <= 192 and its dense instances of side <= 96, dense A
regenerated from the counter-based Gaussian stream the bench draws on the
device) goes to batch_fp64.npz as U<k>, iters<k> and the FP32 noise floor
floor<k> (three seeds) per batch index k.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tval3-cpu_b200", "python"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from tval3g import workloads as W  # noqa: E402


def fp32_noise_floor(op, w, seeds=(1, 2, 3, 4, 5, 6)):
    """How far the FP64 solve moves when a few FP32 roundings per stored
    element and iteration are added (the oracle's noise model, four unit
    roundoffs; tests/helpers.py)."""
    b = w["b"].astype(np.float64)
    r = O.solve(op, b, w["shape"], w["opts"])
    return max(float(np.linalg.norm(O.solve(op, b, w["shape"], dict(w["opts"], noise=4 * 2.0 ** -24,
                                                                        noise_seed=s)).U - r.U)
                     / np.linalg.norm(r.U)) for s in seeds)


def main():
    w = W.ring2d(seed=1, side=256, T=512, tv_norm=1, maxit=500, tol=1e-5, normalize=True)
    op = O.Op.ray2d(w["geom"], 256 * 256)
    t = time.time()
    r = O.solve(op, w["b"].astype(np.float64), w["shape"], w["opts"], Ut=w["u_true"])
    print(f"FP64 oracle: {r.total_iters} iterations, {r.outer_iters} outer, relerr to phantom {r.rel_error:.4f}, "
          f"{time.time() - t:.1f} s")
    out = {"U": r.U.astype(np.float32), "iters": np.array([r.outer_iters, r.total_iters]),
           "noise_floor": np.array([fp32_noise_floor(op, w)]),
           "scale": np.array([w["geom"]["scale"]]), "b_sum": np.array([float(np.sum(w["b"], dtype=np.float64))])}
    o = dict(w["opts"])
    o["tv_norm"] = 0
    r64 = O.solve(op, w["b"].astype(np.float64), w["shape"], o)
    print(f"FP64 oracle, anisotropic: {r64.total_iters} iterations")
    out["U_aniso"] = r64.U.astype(np.float32)
    out["noise_floor_aniso"] = np.array([fp32_noise_floor(op, dict(w, opts=o))])
    out["iters_aniso"] = np.array([r64.outer_iters, r64.total_iters])
    if O.ref_available(2):
        A = w["csr"]
        cwd = os.getcwd()
        rr = O.ref_solve("csr", w["shape"], w["b"], o, dtype=0, csr=(A["m"], A["n"], A["rowptr"], A["colind"], A["val"]))
        os.chdir(cwd)
        d = float(np.linalg.norm(rr.U.ravel() - r64.U.ravel()) / np.linalg.norm(r64.U))
        print(f"aniso: reference float {rr.total_iters} it vs FP64 oracle {r64.total_iters} it, relerr {d:.2e}")
        out["aniso_ref_f32_vs_fp64"] = np.array([d, rr.total_iters, r64.total_iters])
    # the literal configuration: unit weight per hit, 20 iterations
    wu = W.ring2d(seed=1, side=256, T=512, tv_norm=1, maxit=20, tol=1e-5, normalize=False)
    ru = O.solve(O.Op.ray2d(wu["geom"], 256 * 256), wu["b"].astype(np.float64), wu["shape"], wu["opts"])
    out["U_unit20"] = ru.U.astype(np.float32)
    out["iters_unit20"] = np.array([ru.outer_iters, ru.total_iters])
    np.savez_compressed(os.path.join(HERE, "ring256_fp64.npz"), **out)


def dense64():
    """The plain dense 2D workload (64x64, 30 % sampling, isotropic TV)."""
    w = W.dense2d(seed=0, side=64, sampling=0.3, tv_norm=1, maxit=300, tol=1e-4)
    r = O.solve(O.Op.dense(w["A"].astype(np.float64)), w["b"].astype(np.float64), w["shape"], w["opts"],
                Ut=w["u_true"])
    print(f"dense 64x64 FP64 oracle: {r.total_iters} iterations, relerr to phantom {r.rel_error:.4f}")
    np.savez_compressed(os.path.join(HERE, "dense64_fp64.npz"), U=r.U.astype(np.float32),
                        iters=np.array([r.outer_iters, r.total_iters]),
                        noise_floor=np.array([fp32_noise_floor(O.Op.dense(w["A"].astype(np.float64)), w)]))


def mrhs():
    """The multi-right-hand-side workload (A 4096 x 16384, 32 phantoms of
    128x128, solved jointly as 32 layers, isotropic TV)."""
    w = W.mrhs()
    t = time.time()
    r = O.solve(O.Op.dense(w["A"].astype(np.float64), layers=w["layers"]), w["b"].astype(np.float64), w["shape"],
                w["opts"], Ut=w["u_true"])
    print(f"multi-RHS FP64 oracle: {r.total_iters} iterations, relerr to phantoms {r.rel_error:.4f}, "
          f"{time.time() - t:.0f} s")
    np.savez_compressed(os.path.join(HERE, "mrhs32_fp64.npz"), U=r.U.astype(np.float32),
                        iters=np.array([r.outer_iters, r.total_iters]))


def mrhs_indep():
    """The same 32 right-hand sides solved independently (one layer each,
    each with its own scaling, step lengths and stopping), as 32 calls of the
    reference with one layer would: U (32 x 16384) and iteration counts."""
    w = W.mrhs()
    N, (m, n) = w["layers"], w["A"].shape
    op = O.Op.dense(w["A"].astype(np.float64))
    Us, its = [], []
    t = time.time()
    for k in range(N):
        r = O.solve(op, w["b"][k * m:(k + 1) * m].astype(np.float64), (128, 128), w["opts"])
        Us.append(r.U.ravel().astype(np.float32))
        its.append([r.outer_iters, r.total_iters])
        print(f"independent right-hand side {k}: {r.total_iters} iterations ({time.time() - t:.0f} s)")
    np.savez_compressed(os.path.join(HERE, "mrhs32_indep_fp64.npz"), U=np.stack(Us), iters=np.array(its))


def batch():
    out = {}
    t0 = time.time()
    for k, d in enumerate(W.batch_specs()):
        if d["kind"] == "dense" and d["side"] <= 96:
            w = W.batch_dense_host(d)
            op = O.Op.dense(w["A"].astype(np.float64))
        elif d["kind"] == "ray2d" and d["side"] <= 192:
            w = W.batch_ray(d)
            op = O.Op.ray2d(w["geom"], d["side"] ** 2)
        else:
            continue
        r = O.solve(op, w["b"].astype(np.float64), w["shape"], w["opts"])
        out[f"U{k}"] = r.U.astype(np.float32)
        out[f"iters{k}"] = np.array([r.outer_iters, r.total_iters])
        out[f"floor{k}"] = np.array([fp32_noise_floor(op, w, seeds=(1, 2, 3))])
        print(f"batch {k}: {d['kind']} side {d['side']}: {r.total_iters} iterations ({time.time() - t0:.0f} s)")
    np.savez_compressed(os.path.join(HERE, "batch_fp64.npz"), **out)


if __name__ == "__main__":
    parts = sys.argv[1:] or ["ring", "dense64", "mrhs", "mrhs_indep", "batch"]
    if "ring" in parts:
        main()
    if "dense64" in parts:
        dense64()
    if "mrhs" in parts:
        mrhs()
    if "mrhs_indep" in parts:
        mrhs_indep()
    if "batch" in parts:
        batch()
