"""Solve parity at the benchmark configurations, at equal iteration counts.

An FP32 TVAL3 trajectory and the FP64 one take discrete decisions - the
number of Armijo backtracking steps, the A^T-skip heuristic, where the inner
loop ends (RelChg < tol_inn) and where the solve stops - by comparing
floating-point values with thresholds (2d/tval3_cpu_2d.cpp:540-574,790-853).
When one such comparison lands on the other side, the two solves take
different paths from there on and their final images differ by the effect of
that one decision, not by rounding.  So parity is checked twice:

* replayed (the bar): the FP64 oracle replays the GPU's recorded decisions
  (oracle.replay_from_trace), so both solves run the same iteration count and
  path; the GPU's FP32 image must then lie within 1e-3 relative L2 of the
  FP64 image.
* free-running (reported): the GPU's image against the FP64 oracle's own
  solve, with both iteration counts; asserted against a stated bar only where
  the decisions agree.

Configurations (full size): dense 64x64 (A 1229 x 4096, isotropic TV); the
256x256 ring (131072 rays) with isotropic and anisotropic TV; the literal
unit-weight ring for 20 iterations; the 128^3 hemisphere (2048 x 1024 rays)
for 20 iterations and to convergence; multi-RHS dense 4096 x 16384 with 32
right-hand sides for 10 iterations.  Inputs are the seeded synthetic
workloads of tval3g.workloads; every measured error is printed.
"""
import numpy as np
import pytest

import oracle as O
from helpers import golden, relerr
from tval3g import capi, workloads as W

pytestmark = pytest.mark.gpu

BAR = 1e-3


def _gpu(torch, spec, b, opts, device_inputs=False):
    plan = capi.Plan([spec], [opts], graph=True, trace=True, device_inputs=device_inputs)
    db = [torch.tensor(np.ascontiguousarray(b, np.float32), device="cuda")]
    du = [torch.empty(spec.n, device="cuda")]
    info = plan.solve(db, du)[0]
    tr = plan.trace(0)
    plan.close()
    return du[0].cpu().numpy(), info, tr


def _replayed(name, U, info, tr, op, b, shape, opts):
    rp = O.replay_from_trace(tr)
    r = O.solve(op, np.asarray(b, np.float64), shape, opts, replay=rp)
    e = relerr(U, r.U)
    print(f"{name}: GPU {info['total_iters']} iterations ({info['outer_iters']} outer), replayed FP64 "
          f"{r.total_iters}; relerr vs replayed FP64 {e:.3e}")
    assert info["status"] == 0
    assert r.total_iters == info["total_iters"]
    assert e <= BAR, (name, e)
    return r


def _free(name, U, info, fp64_U, fp64_iters):
    e = relerr(U, fp64_U)
    print(f"{name}: free-running FP64 oracle {fp64_iters} iterations, GPU {info['total_iters']}; "
          f"relerr vs FP64 {e:.3e}")
    return e


def test_dense64_full_solve(torch_cuda):
    """Dense 64x64 (A 1229 x 4096, 30 % sampling), isotropic TV, maxit 300."""
    w = W.dense2d(seed=0, side=64, sampling=0.3, tv_norm=1, maxit=300, tol=1e-4)
    spec = capi.problem_from_workload(w)
    U, info, tr = _gpu(torch_cuda, spec, w["b"], w["opts"])
    _replayed("dense 64^2", U, info, tr, O.Op.dense(w["A"].astype(np.float64)), w["b"], w["shape"], w["opts"])
    g = golden("dense64_fp64.npz")
    _free("dense 64^2", U, info, g["U"], int(g["iters"][1]))


@pytest.mark.parametrize("tv", ["iso", "aniso"])
def test_ring256_full_solve(tv, torch_cuda):
    """Ring 256x256, 512 transducers x 256 receivers, hit weight 1/sigma_max."""
    w = W.ring2d(seed=1, side=256, T=512, tv_norm=1 if tv == "iso" else 0, maxit=500, tol=1e-5, normalize=True)
    spec = capi.problem_from_workload(w)
    U, info, tr = _gpu(torch_cuda, spec, w["b"], w["opts"])
    _replayed(f"ring 256^2 {tv}", U, info, tr, O.Op.ray2d(w["geom"], 256 * 256), w["b"], w["shape"], w["opts"])
    g = golden("ring256_fp64.npz")
    key, it = ("U", g["iters"][1]) if tv == "iso" else ("U_aniso", g["iters_aniso"][1])
    e = _free(f"ring 256^2 {tv}", U, info, g[key], int(it))
    if info["total_iters"] == int(it):
        assert e <= BAR


def test_ring256_unit_weight_20_iterations(torch_cuda):
    """The literal unit-weight ring (weight 1 per hit) for 20 iterations."""
    w = W.ring2d(seed=1, side=256, T=512, tv_norm=1, maxit=20, tol=1e-5, normalize=False)
    spec = capi.problem_from_workload(w)
    U, info, tr = _gpu(torch_cuda, spec, w["b"], w["opts"])
    _replayed("ring 256^2 unit weight", U, info, tr, O.Op.ray2d(w["geom"], 256 * 256), w["b"], w["shape"],
              w["opts"])
    g = golden("ring256_fp64.npz")
    _free("ring 256^2 unit weight", U, info, g["U_unit20"], int(g["iters_unit20"][1]))


def _hemi128(torch, maxit):
    """The 128^3 hemisphere; hit weight 1/sigma_max(A) (power iteration on the
    GPU operator, as the benchmark does), data from the FP64 oracle's
    projector."""
    holder = {}

    def fwd(g, u):
        op = capi.Operator(capi.ray3d_problem(u.shape, dict(g, scale=1.0)))
        x = torch.rand(op.cols, device="cuda", generator=torch.Generator(device="cuda").manual_seed(7))
        y = torch.empty(op.rows, device="cuda")
        lam = 1.0
        for _ in range(30):
            x /= torch.linalg.vector_norm(x)
            op.apply(x, y)
            op.apply(y, x, trans=True)
            lam = float(torch.linalg.vector_norm(x))
        op.close()
        g["scale"] = float(np.float32(1.0 / np.sqrt(lam)))
        holder["op"] = O.Op.ray3d(g)
        return holder["op"].apply(u.ravel())

    w = W.hemi3d(seed=2, side=128, T=2048, receivers=1024, tv_norm=0, maxit=maxit, tol=1e-5, forward=fwd)
    return w, holder["op"]


@pytest.mark.parametrize("maxit", [20, 400])
def test_hemi128(maxit, torch_cuda):
    """3D 128^3 hemisphere, 2048 transducers x 1024 receivers (2.1M rays),
    anisotropic TV: 20 iterations, and the full solve (maxit 400)."""
    w, op = _hemi128(torch_cuda, maxit)
    spec = capi.problem_from_workload(w)
    U, info, tr = _gpu(torch_cuda, spec, w["b"], w["opts"])
    _replayed(f"hemisphere 128^3 maxit {maxit}", U, info, tr, op, w["b"], w["shape"], w["opts"])
    r = O.solve(op, w["b"].astype(np.float64), w["shape"], w["opts"])
    e = _free(f"hemisphere 128^3 maxit {maxit}", U, info, r.U, r.total_iters)
    if maxit == 20:
        assert info["total_iters"] == 20 == r.total_iters
        assert e <= BAR


def test_mrhs_10_iterations(torch_cuda):
    """Dense A 4096 x 16384, 32 right-hand sides solved jointly (the
    reference's layers), 3xTF32 tensor-core products, 10 iterations."""
    torch = torch_cuda
    w = W.mrhs()
    opts = dict(w["opts"], maxit=10)
    d_A = torch.tensor(w["A"], device="cuda")
    spec = capi.dense_problem(w["shape"], w["A"], layers=w["layers"], device_ptr=d_A.data_ptr())
    U, info, tr = _gpu(torch, spec, w["b"], opts, device_inputs=True)
    r = _replayed("multi-RHS 32 x 128^2", U, info, tr, O.Op.dense(w["A"].astype(np.float64), layers=w["layers"]),
                  w["b"], w["shape"], opts)
    N = w["layers"]
    per = [relerr(U.reshape(N, -1)[k], r.U.reshape(N, -1)[k]) for k in range(N)]
    print(f"multi-RHS: worst right-hand side {max(per):.3e}")
    assert max(per) <= BAR
