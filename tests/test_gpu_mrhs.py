"""The multi-right-hand-side dense operator on the tcgen05 tensor cores
(3xTF32, `layers` in {16, 32, 48, 64}): products against FP64 and against the
FP64-accumulating gemv kernels, determinism, and a layered solve against the
FP64 oracle (the reference's joint multi-layer solve, 2d/mat_mult.h:15-36)."""
import numpy as np
import pytest

import oracle as O
from helpers import relerr
from tval3g import capi
from tval3g import workloads as W

pytestmark = pytest.mark.gpu

# (m, n, layers): ragged tile edges (300, 1000), long K (16384), wide N (64), and
# the multi-RHS bench shape (4096 x 16384, 32 right-hand sides)
SHAPES = [(256, 512, 16), (300, 1000, 32), (1024, 4096, 48), (4096, 2048, 64), (512, 16384, 32), (4096, 16384, 32)]
PRODUCT_TOL = 1e-5   # per layer, relative L2 against the FP64 product


def _layer_err(got, ref):
    return max(relerr(g, r) for g, r in zip(got, ref))


@pytest.mark.parametrize("m,n,N", SHAPES)
def test_products_match_fp64(m, n, N, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(m * 7 + n * 3 + N)
    A = (rng.standard_normal((m, n)) / np.sqrt(m)).astype(np.float32)
    X = rng.standard_normal((N, n)).astype(np.float32)
    R = rng.standard_normal((N, m)).astype(np.float32)
    Y64 = X.astype(np.float64) @ A.T.astype(np.float64)
    Z64 = R.astype(np.float64) @ A.astype(np.float64)
    spec = capi.dense_problem((N, n), A, layers=N)
    dx, dr = torch.tensor(X.ravel(), device="cuda"), torch.tensor(R.ravel(), device="cuda")
    res = {}
    for tensor in (True, False):
        op = capi.Operator(spec, tensor=tensor)
        y = torch.empty(N * m, device="cuda")
        z = torch.empty(N * n, device="cuda")
        op.apply(dx, y)
        op.apply(dr, z, trans=True)
        res[tensor] = (y.cpu().numpy().reshape(N, m), z.cpu().numpy().reshape(N, n))
        if tensor:   # same inputs, same bits
            y2 = torch.empty_like(y)
            op.apply(dx, y2)
            assert torch.equal(y, y2)
        op.close()
    ey, ez = _layer_err(res[True][0], Y64), _layer_err(res[True][1], Z64)
    assert ey <= PRODUCT_TOL and ez <= PRODUCT_TOL, (ey, ez)
    # the gemv path (FP64 accumulation) is the closer of the two
    assert _layer_err(res[False][0], Y64) <= 1e-6 and _layer_err(res[False][1], Z64) <= 1e-6


def _layered_case(side=16, layers=16, m=128, seed=5):
    rng = np.random.default_rng(seed)
    n = side * side
    A = (rng.standard_normal((m, n)) / np.sqrt(m)).astype(np.float32)
    us = [W.ellipse_phantom(side, side, rng, 3, 0.0, lambda r: r.uniform(0.2, 1.0), (2, 6)) for _ in range(layers)]
    b = np.concatenate([A.astype(np.float64) @ u.ravel() for u in us])
    b = W.add_noise(b, 0.01, rng).astype(np.float32)
    opts = W.options(2 ** 8, 2 ** 5, 1e-12, 40, tv_norm=1)
    return A, b, opts, (side * layers, side)


def test_layered_solve_matches_oracle(torch_cuda):
    A, b, opts, shape = _layered_case()
    layers = shape[0] // shape[1]
    ref = O.solve(O.Op.dense(A.astype(np.float64), layers=layers), b.astype(np.float64), shape, opts)
    spec = capi.dense_problem(shape, A, layers=layers)
    out = {}
    for tensor in (True, False):
        plan = capi.Plan([spec], [opts], graph=True, tensor=tensor)
        d_b = torch_cuda.tensor(b, device="cuda")
        d_U = torch_cuda.empty(spec.n, device="cuda")
        info = plan.solve([d_b], [d_U])[0]
        plan.close()
        out[tensor] = (d_U.cpu().numpy(), info["total_iters"])
    assert out[True][1] == out[False][1] == ref.total_iters
    e_t, e_g = relerr(out[True][0], ref.U.ravel()), relerr(out[False][0], ref.U.ravel())
    assert e_t <= 1e-3 and e_g <= 1e-3, (e_t, e_g)


@pytest.mark.parametrize("count", [16, 35])
def test_independent_right_hand_sides(count, torch_cuda):
    """Independent right-hand sides: one-layer instances of one plan sharing
    a device matrix are grouped (16 or 32 of them; the 3 left over of 35 keep
    their gemv products) and every product of a group is one tensor-core
    contraction, while each instance keeps its own scaling, step lengths,
    line search and stopping.  A fixed 20 iterations (short enough that the
    FP64 solves' FP32 noise floor is ~1e-6): each instance against its own
    FP64 oracle solve, and against the same plan on the gemv kernels, within
    1e-3; the distance to the oracle replaying that instance's decisions is
    printed beside it."""
    torch = torch_cuda
    side, m = 16, 128
    rng = np.random.default_rng(count)
    n = side * side
    A = (rng.standard_normal((m, n)) / np.sqrt(m)).astype(np.float32)
    us = [W.ellipse_phantom(side, side, rng, 3, 0.0, lambda r: r.uniform(0.2, 1.0), (2, 6)) for _ in range(count)]
    bs = [W.add_noise(A.astype(np.float64) @ u.ravel(), 0.01, rng).astype(np.float32) for u in us]
    opts = W.options(2 ** 8, 2 ** 5, 1e-4, 20, tv_norm=1)
    d_A = torch.tensor(A, device="cuda")
    specs = [capi.dense_problem((side, side), A, device_ptr=d_A.data_ptr()) for _ in range(count)]
    db = [torch.tensor(b, device="cuda") for b in bs]
    out = {}
    for tensor in (True, False):
        plan = capi.Plan(specs, [opts] * count, graph=True, device_inputs=True, trace=True, tensor=tensor)
        du = [torch.empty(n, device="cuda") for _ in range(count)]
        infos = plan.solve(db, du)
        out[tensor] = ([u.cpu().numpy() for u in du], infos, [plan.trace(k) for k in range(count)],
                       plan.stats()["device_bytes"])
        plan.close()
    op64 = O.Op.dense(A.astype(np.float64))
    worst, worst_r, worst_g = 0.0, 0.0, 0.0
    for k in range(count):
        U, info, tr = out[True][0][k], out[True][1][k], out[True][2][k]
        b64 = bs[k].astype(np.float64)
        r = O.solve(op64, b64, (side, side), opts)
        rr = O.solve(op64, b64, (side, side), opts, replay=O.replay_from_trace(tr))
        assert r.total_iters == info["total_iters"] == 20
        worst = max(worst, relerr(U, r.U.ravel()))
        worst_r = max(worst_r, relerr(U, rr.U.ravel()))
        worst_g = max(worst_g, relerr(U, out[False][0][k]))
    print(f"{count} independent right-hand sides: worst relerr vs FP64 {worst:.2e}, vs FP64 replaying the GPU's "
          f"decisions {worst_r:.2e}, vs the gemv plan {worst_g:.2e}")
    assert worst <= 1e-3 and worst_g <= 1e-3
    assert worst_g > 0   # the group's products ran on the tensor cores (other rounding than the gemv plan)
