"""Degenerate and ragged problems through the C ABI against the FP64 oracle:
a one-pixel image, images whose sides are not multiples of any tile, CSR
rows without entries, rays of length zero and unused paths, a 2x2x2 volume."""
import numpy as np
import pytest

import oracle as O
from helpers import relerr
from tval3g import capi, workloads as W

pytestmark = pytest.mark.gpu


def _opts(maxit=10):
    return W.options(2 ** 8, 2 ** 5, 1e-4, maxit, tv_norm=0)


def _check(spec, op, b, shape, opts, bar=1e-3):
    U, info = capi.solve(spec, b, opts)
    r = O.solve(op, np.asarray(b, np.float64), shape, opts)
    assert info["status"] == 0
    assert info["total_iters"] == r.total_iters, (info, r.total_iters)
    scale = max(np.linalg.norm(r.U), 1e-30)
    assert np.linalg.norm(U.astype(np.float64) - r.U) <= bar * scale, relerr(U, r.U)
    return U


def test_one_pixel_is_reported_not_returned_as_nan(torch_cuda):
    """On a 1x1 image the first step length is 0/0: the reference (and the
    oracle) return NaN; the C ABI stops with TVAL3G_ERR_NONFINITE instead."""
    A = np.array([[0.7]], np.float32)
    b = np.array([0.35], np.float32)
    r = O.solve(O.Op.dense(A.astype(np.float64)), b.astype(np.float64), (1, 1), _opts())
    assert np.isnan(r.U).all()
    with pytest.raises(capi.TVAL3Error) as e:
        capi.solve(capi.dense_problem((1, 1), A), b, _opts())
    assert e.value.code == capi.ERR_NONFINITE


@pytest.mark.parametrize("shape,m", [((2, 3), 4), ((3, 5), 7), ((17, 9), 40)])
def test_dense_tiny_and_ragged(shape, m, torch_cuda):
    rng = np.random.default_rng(sum(shape) + m)
    n = shape[0] * shape[1]
    A = (rng.standard_normal((m, n)) / np.sqrt(m)).astype(np.float32)
    b = (A.astype(np.float64) @ rng.uniform(0, 1, n)).astype(np.float32)
    _check(capi.dense_problem(shape, A), O.Op.dense(A.astype(np.float64)), b, shape, _opts())


def test_csr_with_empty_rows(torch_cuda):
    rng = np.random.default_rng(3)
    shape, m = (6, 7), 20
    n = shape[0] * shape[1]
    lens = rng.integers(0, 5, m)
    lens[[0, 5, 19]] = 0                       # rows without entries
    rowptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    colind = np.concatenate([np.sort(rng.choice(n, k, replace=False)) for k in lens]).astype(np.int32)
    val = rng.standard_normal(len(colind)).astype(np.float32)
    x = rng.uniform(0, 1, n)
    y = np.zeros(m)
    rows = np.repeat(np.arange(m), lens)
    np.add.at(y, rows, val * x[colind])
    b = y.astype(np.float32)
    b[[0, 5, 19]] = 0.1                        # data no operator row explains
    _check(capi.csr_problem(shape, m, n, rowptr, colind, val),
           O.Op.csr(m, n, rowptr, colind, val.astype(np.float64)), b, shape, _opts())


def test_rays_of_length_zero_and_unused_paths(torch_cuda):
    side = 5
    xs = np.array([0, 4, 2, 0, 4], np.int32)
    ys = np.array([0, 0, 4, 2, 4], np.int32)
    T = len(xs)
    use = np.ones((T, T), np.int32)
    use[1, 3] = use[3, 1] = 0                  # unused paths
    # emitter == receiver on the diagonal: one-pixel rays
    g = dict(use_path=use.ravel(), xe=xs, ye=ys, xr=xs, yr=ys, ld=side, scale=0.25)
    rng = np.random.default_rng(4)
    b = rng.uniform(0.5, 1.5, T * T).astype(np.float32) * use.ravel()
    _check(capi.ray2d_problem((side, side), g), O.Op.ray2d(g, side * side), b, (side, side), _opts())


def test_two_by_two_by_two_volume(torch_cuda):
    N = 4
    pts = np.array([[0, 0, 0], [1, 1, 1], [1, 0, 1], [0, 1, 0]], np.int32)
    use = np.zeros((N, N), np.int32)
    k = 1
    for e in range(N):
        for r in range(N):
            if e != r:
                use[e, r] = k
                k += 1
    g = dict(numMPs=1, numPaths=k - 1, E=N, R=N, use_path=use.ravel(), xe=pts[:, 0], ye=pts[:, 1], ze=pts[:, 2],
             xr=pts[:, 0], yr=pts[:, 1], zr=pts[:, 2], rv_x=2, rv_y=2, rv_z=2, scale=0.5)
    b = np.random.default_rng(5).uniform(0.5, 1.5, k - 1).astype(np.float32)
    _check(capi.ray3d_problem((2, 2, 2), g), O.Op.ray3d(g), b, (2, 2, 2), _opts())


def test_bounded_wait_timeout_reports_and_recovers(torch_cuda, monkeypatch):
    """The failure path of the bounded device waits, without a fault: with
    the test hook TVAL3G_TEST_FIRST_WAIT_POLLS=0 the tiled ray adjoint's first
    wait (its ray list) gives up at once; the kernel drains its bulk copies in
    flight, raises the operator's error word and returns, and the solve
    reports TVAL3G_ERR_CUDA.  A plan built afterwards, without the hook,
    solves normally in the same process: bit for bit the solve made before
    the failure."""
    from golden.cases import api_problem, build_case
    torch = torch_cuda
    c = build_case("ring2d_s64_it20")
    spec = api_problem(c, capi)
    U0, info0 = capi.solve(spec, c["b"], c["opts"])
    monkeypatch.setenv("TVAL3G_TEST_FIRST_WAIT_POLLS", "0")
    plan = capi.Plan([spec], [dict(c["opts"], maxit=5)], graph=True)
    monkeypatch.delenv("TVAL3G_TEST_FIRST_WAIT_POLLS")
    db = [torch.tensor(c["b"], device="cuda")]
    du = [torch.empty(spec.n, device="cuda")]
    with pytest.raises(capi.TVAL3Error) as e:
        plan.solve(db, du)
    assert e.value.code == capi.ERR_CUDA and "bounded wait" in str(e.value)
    plan.close()
    U1, info1 = capi.solve(spec, c["b"], c["opts"])
    assert info1["status"] == 0 and info1["total_iters"] == info0["total_iters"] == 20
    np.testing.assert_array_equal(U1, U0)


def _ray_error(spec):
    with pytest.raises(capi.TVAL3Error) as e:
        capi.Operator(spec)
    assert e.value.code == capi.ERR_ARGUMENT
    return str(e.value)


def test_ray_geometry_argument_errors(torch_cuda):
    """The rays are packed on the device; an endpoint outside the image or
    volume and a 3D use_path index beyond numPaths are still reported with
    the reference's messages (2d/tval3_cpu_2d.cpp:696-750,
    3d/tval3_cpu_3d.cpp:1028-1165), the first offending ray in the
    reference's loop order (plane, emitter, receiver) deciding which."""
    g2 = dict(use_path=np.ones(6, np.int32), xe=[0, 1], ye=[0, 2], xr=[3, 4, 9], yr=[1, 1, 1], ld=5, scale=1.0)
    assert "lies outside the image" in _ray_error(capi.ray2d_problem((4, 5), g2))
    g3 = W.hemisphere_geometry(8, 8, 4, 3.0, np.random.default_rng(1))
    bad = dict(g3, use_path=np.array(g3["use_path"]))
    k = int(np.nonzero(bad["use_path"])[0][-1])      # the last used path: beyond numPaths
    bad["use_path"][k] = g3["numPaths"] + 1
    assert "use_path index exceeds numPaths" in _ray_error(capi.ray3d_problem((8, 8, 8), bad))
    both = dict(bad, xe=np.array(g3["xe"]))          # and an endpoint error on a later emitter
    e_last = len(both["xe"]) - 1
    both["xe"][e_last] = 99
    first_bad_emitter = k // g3["R"]
    msg = _ray_error(capi.ray3d_problem((8, 8, 8), both))
    if first_bad_emitter < e_last:
        assert "use_path index exceeds numPaths" in msg
    else:
        assert "lies outside the volume" in msg
    ok = capi.Operator(capi.ray3d_problem((8, 8, 8), g3))   # the unaltered geometry still builds
    ok.close()


def test_time_stencils_after_a_solve(torch_cuda):
    """tval3g_plan_time_stencils times the three vector kernels after a solve;
    the next solve starts afresh and gives the same result as the first."""
    torch = torch_cuda
    w = W.ring2d(seed=1, side=64, T=64, tv_norm=1, maxit=20, tol=1e-5, normalize=True)
    spec = capi.problem_from_workload(w)
    plan = capi.Plan([spec], [w["opts"]])
    db = [torch.tensor(np.asarray(w["b"], np.float32), device="cuda")]
    u1, u2 = [torch.empty(spec.n, device="cuda")], [torch.empty(spec.n, device="cuda")]
    i1 = plan.solve(db, u1)[0]
    ms = plan.time_stencils(5)
    i2 = plan.solve(db, u2)[0]
    plan.close()
    print("stencil ms per launch:", ms)
    assert all(v > 0 for v in ms.values())
    assert i1["total_iters"] == i2["total_iters"] and torch.equal(u1[0], u2[0])
