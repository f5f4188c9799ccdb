"""Solve parity at the benchmark configurations, at full size.

The GPU's FP32 solution against the FP64 oracle's solve of the same problem
(free-running: its own decisions), within 1e-3 relative L2 - or, for a solve
run to convergence, within twice the problem's FP32 noise floor where that is
larger: how far FP64 solves of the same problem move when one FP32 rounding
per stored element and iteration is added (helpers.noise_floor; the
threshold decisions and the nonmonotone line search of TVAL3 amplify such
perturbations, 2d/tval3_cpu_2d.cpp:540-574,790-853).  Fixed short solves are
held to 1e-3.  The distance to the oracle replaying the GPU's own recorded
decisions (oracle.replay_from_trace: the same iteration count and path) is
printed beside it.

Configurations: dense 64x64 (A 1229 x 4096, isotropic TV); the 256x256 ring
(131072 rays) with isotropic and anisotropic TV; the literal unit-weight ring
for 20 iterations; the 128^3 hemisphere (2048 x 1024 rays) for 20 iterations
and to convergence; multi-RHS dense 4096 x 16384 with 32 right-hand sides
for 10 iterations.  Inputs are the seeded synthetic workloads of
tval3g.workloads; every measured error is printed.
"""
import numpy as np
import pytest

import oracle as O
from helpers import BAR, NOISE_SEEDS, golden, noise_floor, relerr, solve_bar
from tval3g import capi, workloads as W

pytestmark = pytest.mark.gpu


def _gpu(torch, spec, b, opts, device_inputs=False):
    plan = capi.Plan([spec], [opts], graph=True, trace=True, device_inputs=device_inputs)
    db = [torch.tensor(np.ascontiguousarray(b, np.float32), device="cuda")]
    du = [torch.empty(spec.n, device="cuda")]
    info = plan.solve(db, du)[0]
    tr = plan.trace(0)
    plan.close()
    return du[0].cpu().numpy(), info, tr


def _check(name, U, info, tr, op, b, shape, opts, converged):
    """FP64 free-running (and noise floor when converged) and replayed."""
    b64 = np.asarray(b, np.float64)
    solve = lambda extra: O.solve(op, b64, shape, dict(opts, **extra))  # noqa: E731
    r = solve({})
    floor = noise_floor(solve, r.U, seeds=(1, 2, 3) if b64.size > 1e6 else NOISE_SEEDS) if converged else 0.0
    bar = solve_bar(floor)
    e = relerr(U, r.U)
    rr = O.solve(op, b64, shape, opts, replay=O.replay_from_trace(tr))
    print(f"{name}: GPU {info['total_iters']} iterations, FP64 {r.total_iters}; relerr vs FP64 {e:.3e}, bar "
          f"{bar:.2e} (FP32 noise floor {floor:.2e}); vs FP64 replaying the GPU's decisions {relerr(U, rr.U):.3e}")
    assert info["status"] == 0
    assert e <= bar, (name, e, bar)
    return r


def test_dense64_full_solve(torch_cuda):
    """Dense 64x64 (A 1229 x 4096, 30 % sampling), isotropic TV, maxit 300."""
    w = W.dense2d(seed=0, side=64, sampling=0.3, tv_norm=1, maxit=300, tol=1e-4)
    U, info, tr = _gpu(torch_cuda, capi.problem_from_workload(w), w["b"], w["opts"])
    _check("dense 64^2", U, info, tr, O.Op.dense(w["A"].astype(np.float64)), w["b"], w["shape"], w["opts"], True)
    g = golden("dense64_fp64.npz")
    print(f"dense 64^2: vs the committed FP64 solution {relerr(U, g['U']):.3e}")


@pytest.mark.parametrize("tv", ["iso", "aniso"])
def test_ring256_full_solve(tv, torch_cuda):
    """Ring 256x256, 512 transducers x 256 receivers, hit weight 1/sigma_max."""
    w = W.ring2d(seed=1, side=256, T=512, tv_norm=1 if tv == "iso" else 0, maxit=500, tol=1e-5, normalize=True)
    U, info, tr = _gpu(torch_cuda, capi.problem_from_workload(w), w["b"], w["opts"])
    _check(f"ring 256^2 {tv}", U, info, tr, O.Op.ray2d(w["geom"], 256 * 256), w["b"], w["shape"], w["opts"], True)


def test_ring256_unit_weight_20_iterations(torch_cuda):
    """The literal unit-weight ring (weight 1 per hit) for 20 iterations."""
    w = W.ring2d(seed=1, side=256, T=512, tv_norm=1, maxit=20, tol=1e-5, normalize=False)
    U, info, tr = _gpu(torch_cuda, capi.problem_from_workload(w), w["b"], w["opts"])
    _check("ring 256^2 unit weight", U, info, tr, O.Op.ray2d(w["geom"], 256 * 256), w["b"], w["shape"], w["opts"],
           False)
    g = golden("ring256_fp64.npz")
    assert relerr(U, g["U_unit20"]) <= BAR


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
    U, info, tr = _gpu(torch_cuda, capi.problem_from_workload(w), w["b"], w["opts"])
    r = _check(f"hemisphere 128^3 maxit {maxit}", U, info, tr, op, w["b"], w["shape"], w["opts"], maxit > 20)
    if maxit == 20:
        assert info["total_iters"] == 20 == r.total_iters


def test_mrhs_10_iterations(torch_cuda):
    """Dense A 4096 x 16384, 32 right-hand sides solved jointly (the
    reference's layers), 3xTF32 tensor-core products, 10 iterations; every
    right-hand side within 1e-3."""
    torch = torch_cuda
    w = W.mrhs()
    opts = dict(w["opts"], maxit=10)
    d_A = torch.tensor(w["A"], device="cuda")
    spec = capi.dense_problem(w["shape"], w["A"], layers=w["layers"], device_ptr=d_A.data_ptr())
    U, info, tr = _gpu(torch, spec, w["b"], opts, device_inputs=True)
    r = _check("multi-RHS 32 x 128^2", U, info, tr, O.Op.dense(w["A"].astype(np.float64), layers=w["layers"]),
               w["b"], w["shape"], opts, False)
    N = w["layers"]
    per = [relerr(U.reshape(N, -1)[k], r.U.reshape(N, -1)[k]) for k in range(N)]
    print(f"multi-RHS: worst right-hand side {max(per):.3e}")
    assert max(per) <= BAR


def test_dense128_wide_rows_20_iterations(torch_cuda):
    """Dense 128x128 (A 4915 x 16384, 322 MB: the one-pass normal product
    with many bands), 20 iterations, within 1e-3 of the FP64 oracle."""
    w = W.dense2d(seed=5, side=128, sampling=0.3, tv_norm=1, maxit=20, tol=1e-4)
    U, info, tr = _gpu(torch_cuda, capi.problem_from_workload(w), w["b"], w["opts"])
    _check("dense 128^2", U, info, tr, O.Op.dense(w["A"].astype(np.float64)), w["b"], w["shape"], w["opts"], False)
    assert info["total_iters"] == 20
