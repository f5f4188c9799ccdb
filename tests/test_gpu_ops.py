"""GPU parity of the measurement operators and stencils, through the C ABI.

Bresenham pixel lists are compared bit-exactly with the oracle's sequential
recurrence; operator applications within 1e-5 relative of the FP64 oracle.
"""
import numpy as np
import pytest

import oracle as O
from golden.cases import api_problem, build_case
from helpers import BAR, relerr
from tval3g import capi, workloads as W

pytestmark = pytest.mark.gpu

OP_CASES = ["dense2d_s32_it20", "dense2d_layers", "ring2d_s64_it20", "ring2d_s64_skip", "hemi3d_s16_it20",
            "csr3d_s16", "dense3d_s8", "hemi3d_mp2_s16", "csr2d_layers"]


def _dev(torch, a):
    return torch.tensor(np.ascontiguousarray(a, np.float32), device="cuda")


@pytest.mark.parametrize("name", OP_CASES)
def test_operator_forward_adjoint(name, torch_cuda):
    torch = torch_cuda
    c = build_case(name)
    op = capi.Operator(api_problem(c, capi))
    rng = np.random.default_rng(3)
    x = rng.standard_normal(op.cols).astype(np.float32)
    y = rng.standard_normal(op.rows).astype(np.float32)
    dy = torch.empty(op.rows, device="cuda")
    op.apply(_dev(torch, x), dy)
    ref = c["oracle_op"].apply(x.astype(np.float64))
    assert relerr(dy.cpu().numpy(), ref) < 1e-5
    dx = torch.empty(op.cols, device="cuda")
    op.apply(_dev(torch, y), dx, trans=True)
    ref = c["oracle_op"].apply(y.astype(np.float64), trans=True)
    assert relerr(dx.cpu().numpy(), ref) < 1e-5
    # adjoint identity <A x, y> = <x, A^T y>
    lhs = float(np.dot(dy.cpu().numpy().astype(np.float64), y))
    rhs = float(np.dot(x.astype(np.float64), dx.cpu().numpy()))
    assert abs(lhs - rhs) <= 1e-5 * (abs(lhs) + abs(rhs))
    # deterministic: a second application is bit-identical
    dx2 = torch.empty(op.cols, device="cuda")
    op.apply(_dev(torch, y), dx2, trans=True)
    assert torch.equal(dx, dx2)


def _expected_rows(oracle_op, rows):
    ray, off, pix = oracle_op.ray_lists()
    lens = np.zeros(rows, np.int64)
    lens[ray] = np.diff(off)
    rowptr = np.zeros(rows + 1, np.int64)
    np.cumsum(lens, out=rowptr[1:])
    colind = np.zeros(rowptr[-1], np.int32)
    for k, r in enumerate(ray):
        colind[rowptr[r]:rowptr[r + 1]] = pix[off[k]:off[k + 1]]
    return rowptr, colind


@pytest.mark.parametrize("name", ["ring2d_s64_it20", "hemi3d_s16_it20"])
def test_bresenham_lists_bit_exact(name, torch_cuda):
    c = build_case(name)
    op = capi.Operator(api_problem(c, capi))
    rowptr, colind = op.ray_csr()
    erp, eci = _expected_rows(c["oracle_op"], op.rows)
    np.testing.assert_array_equal(rowptr, erp)
    np.testing.assert_array_equal(colind, eci)


def test_bresenham_edge_rays_bit_exact(torch_cuda):
    """Axis-aligned, 45 degree, steep, zero-length and negative rays, 2D and 3D ties."""
    x0 = np.array([0, 0, 7, 0, 7, 2, 1, 6, 1, 3, 0, 5])
    y0 = np.array([0, 0, 7, 0, 0, 3, 1, 3, 6, 0, 7, 2])
    x1 = np.array([7, 0, 0, 7, 0, 2, 6, 1, 3, 1, 7, 0])
    y1 = np.array([0, 7, 0, 7, 7, 3, 3, 1, 0, 6, 6, 4])
    N = len(x0)
    g = dict(use_path=np.eye(N, dtype=np.int32).ravel(), xe=x0, ye=y0, xr=x1, yr=y1, ld=8, scale=1.0)
    op = capi.Operator(capi.ray2d_problem((8, 8), g))
    rowptr, colind = op.ray_csr()
    erp, eci = _expected_rows(O.Op.ray2d(g, 64), N * N)
    np.testing.assert_array_equal(rowptr, erp)
    np.testing.assert_array_equal(colind, eci)
    p0 = np.array([[0, 0, 0], [0, 0, 0], [0, 0, 0], [5, 5, 5], [1, 2, 3], [7, 0, 3], [3, 3, 3], [0, 7, 7]])
    p1 = np.array([[7, 7, 0], [0, 7, 7], [7, 0, 7], [0, 0, 0], [6, 4, 7], [0, 7, 5], [3, 3, 3], [7, 0, 0]])
    N = len(p0)
    g3 = dict(numMPs=1, numPaths=N, E=N, R=N, use_path=(np.eye(N, dtype=np.int32) * np.arange(1, N + 1)).ravel(),
              xe=p0[:, 0], ye=p0[:, 1], ze=p0[:, 2], xr=p1[:, 0], yr=p1[:, 1], zr=p1[:, 2], rv_x=8, rv_y=8, rv_z=8,
              scale=1.0)
    op = capi.Operator(capi.ray3d_problem((8, 8, 8), g3))
    rowptr, colind = op.ray_csr()
    erp, eci = _expected_rows(O.Op.ray3d(g3), N)
    np.testing.assert_array_equal(rowptr, erp)
    np.testing.assert_array_equal(colind, eci)


def test_full_ring_operator_properties(torch_cuda):
    """256x256, 512 transducers, 131072 rays: GPU rasterisation == closed form
    CSR twin bit-exactly; A x and A^T y against the twin; adjoint identity."""
    torch = torch_cuda
    w = W.ring2d(seed=1, side=256, T=512)
    op = capi.Operator(capi.ray2d_problem(w["shape"], w["geom"]))
    rowptr, colind = op.ray_csr()
    A = w["csr"]
    np.testing.assert_array_equal(rowptr, A["rowptr"])
    np.testing.assert_array_equal(colind, A["colind"])
    rng = np.random.default_rng(0)
    x = rng.standard_normal(op.cols).astype(np.float32)
    y = rng.standard_normal(op.rows).astype(np.float32)
    dy = torch.empty(op.rows, device="cuda")
    op.apply(_dev(torch, x), dy)
    assert relerr(dy.cpu().numpy(), W.csr_matvec(A, x)) < 1e-5
    dx = torch.empty(op.cols, device="cuda")
    op.apply(_dev(torch, y), dx, trans=True)
    lhs = float(np.dot(dy.cpu().numpy().astype(np.float64), y))
    rhs = float(np.dot(x.astype(np.float64), dx.cpu().numpy()))
    assert abs(lhs - rhs) <= 1e-5 * (abs(lhs) + abs(rhs))
    # the CSR twin on the GPU gives the same products
    csr = capi.Operator(capi.csr_problem(w["shape"], A["m"], A["n"], A["rowptr"], A["colind"], A["val"]))
    dy2 = torch.empty(op.rows, device="cuda")
    csr.apply(_dev(torch, x), dy2)
    assert relerr(dy2.cpu().numpy(), dy.cpu().numpy()) < 1e-6
    dx2 = torch.empty(op.cols, device="cuda")
    csr.apply(_dev(torch, y), dx2, trans=True)
    assert relerr(dx2.cpu().numpy(), dx.cpu().numpy()) < 1e-6


@pytest.mark.parametrize("m, shape", [
    (1229, (64, 64)),      # one band
    (3000, (200, 200)),    # rows too long for the band form (n = 40000): two-pass gemv, A 480 MB
    (601, (256, 256)),     # n = 65536
    (2000, (100, 100)),    # the band form (n = 10000): bands of rows
    (100, (16, 20)),       # fewer rows than CTAs
    (500, (31, 33)),       # n not a multiple of 4: scalar loads
])
def test_dense_normal_product(m, shape, torch_cuda):
    """y = A^T (A x) in one pass over A (trans = 2) against the FP64 product
    and against the two separate products; deterministic."""
    torch = torch_cuda
    rng = np.random.default_rng(m)
    n = shape[0] * shape[1]
    A = (rng.standard_normal((m, n), dtype=np.float32) / np.float32(np.sqrt(m)))
    op = capi.Operator(capi.dense_problem(shape, A))
    x = rng.standard_normal(n).astype(np.float32)
    dx = _dev(torch, x)
    y = torch.empty(n, device="cuda")
    op.apply(dx, y, trans=2)
    A64 = A.astype(np.float64)
    ref = A64.T @ (A64 @ x.astype(np.float64))
    assert relerr(y.cpu().numpy(), ref) < 1e-5
    au = torch.empty(m, device="cuda")
    y2 = torch.empty(n, device="cuda")
    op.apply(dx, au)
    op.apply(au, y2, trans=True)
    assert relerr(y.cpu().numpy(), y2.cpu().numpy()) < 1e-5
    y3 = torch.empty(n, device="cuda")
    op.apply(dx, y3, trans=2)
    assert torch.equal(y, y3)


def _random_rays(rng, H, ld, E, R, frac):
    return dict(use_path=(rng.uniform(size=E * R) < frac).astype(np.int32),
                xe=rng.integers(0, ld, E), ye=rng.integers(0, H, E),
                xr=rng.integers(0, ld, R), yr=rng.integers(0, H, R), ld=ld, scale=0.75)


@pytest.mark.parametrize("H, ld, E, R, frac", [
    (50, 37, 40, 30, 0.7),      # tiles cut by both image edges
    (17, 300, 25, 40, 0.5),     # one tile row and a partial one
    (40, 40, 640, 480, 0.9),    # 276480 traced rays: beyond the tiled index, pixel-major gather
])
def test_ray2d_adjoint_ragged_and_large(H, ld, E, R, frac, torch_cuda):
    """The 2D ray adjoint on images that the 16x16 pixel tiles do not divide,
    and past the tiled index's ray limit, against the FP64 oracle."""
    torch = torch_cuda
    rng = np.random.default_rng(H * ld + E)
    g = _random_rays(rng, H, ld, E, R, frac)
    op = capi.Operator(capi.ray2d_problem((H, ld), g))
    ref_op = O.Op.ray2d(g, H * ld)
    y = rng.standard_normal(op.rows).astype(np.float32)
    dx = torch.empty(op.cols, device="cuda")
    op.apply(_dev(torch, y), dx, trans=True)
    assert relerr(dx.cpu().numpy(), ref_op.apply(y.astype(np.float64), trans=True)) < 1e-5
    x = rng.standard_normal(op.cols).astype(np.float32)
    dy = torch.empty(op.rows, device="cuda")
    op.apply(_dev(torch, x), dy)
    assert relerr(dy.cpu().numpy(), ref_op.apply(x.astype(np.float64))) < 1e-5
    dx2 = torch.empty(op.cols, device="cuda")
    op.apply(_dev(torch, y), dx2, trans=True)
    assert torch.equal(dx, dx2)
    assert op.adjoint_index_bytes > 0


@pytest.mark.parametrize("shape", [(5, 7), (16, 16), (3, 4, 5), (8, 6, 4)])
def test_stencils_match_oracle(shape, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(sum(shape))
    dims = len(shape)
    n = int(np.prod(shape))
    U = rng.standard_normal(shape).astype(np.float32)
    dU = _dev(torch, U)
    outs = [torch.empty(n, device="cuda") for _ in range(3)]
    capi.D(dims, shape, dU, *outs[:dims])
    ref = O.D(U.astype(np.float64))
    for k in range(dims):
        np.testing.assert_allclose(outs[k].cpu().numpy(), ref[k], rtol=0, atol=1e-6)
    X = [rng.standard_normal(n).astype(np.float32) for _ in range(3)]
    res = torch.empty(n, device="cuda")
    capi.Dt(dims, shape, _dev(torch, X[0]), _dev(torch, X[1]), _dev(torch, X[2]) if dims == 3 else None, res)
    ref = O.Dt(X[0], X[1], X[2] if dims == 3 else None, shape=shape)
    np.testing.assert_allclose(res.cpu().numpy(), ref, rtol=0, atol=1e-5)
    for tv in (0, 1):
        S = [rng.standard_normal(n).astype(np.float32) * 0.1 for _ in range(dims)]
        Wd = [torch.empty(n, device="cuda") for _ in range(dims)]
        lam = capi.shrink(dims, n, tv, 8.0, [_dev(torch, x) for x in X[:dims]], [_dev(torch, s) for s in S], Wd)
        Wr, lamr = O.shrink([x.astype(np.float64) for x in X[:dims]], [s.astype(np.float64) for s in S], 8.0, tv)
        for k in range(dims):
            np.testing.assert_allclose(Wd[k].cpu().numpy(), Wr[k], rtol=0, atol=1e-6)
        assert abs(lam - lamr) < 1e-5 * abs(lamr)


def test_bresenham_3d_gpu_matches_the_reference_projector(torch_cuda):
    """The GPU's 3D rasterisation equals the reference's live projector
    (3d/mat_mult.h:148-363, oracle/_ref) hit for hit on the tie cases and a
    12^3 hemisphere (one-hot columns of the reference)."""
    from test_oracle import _ref_matrix_3d, _tie_geometry
    for g in (_tie_geometry(), W.hemisphere_geometry(12, 24, 8, 5.0, np.random.default_rng(4))):
        n = int(g["rv_x"]) * int(g["rv_y"]) * int(g["rv_z"])
        op = capi.Operator(capi.ray3d_problem((int(g["rv_z"]), int(g["rv_y"]), int(g["rv_x"])), g))
        rowptr, colind = op.ray_csr()
        op.close()
        M = np.zeros((len(rowptr) - 1, n))
        for r in range(len(rowptr) - 1):
            np.add.at(M[r], colind[rowptr[r]:rowptr[r + 1]], 1.0)
        np.testing.assert_array_equal(M, _ref_matrix_3d(g))


def test_hemi128_products_match_the_reference_projector(torch_cuda):
    """The 128^3 hemisphere (2048 transducers x 1024 receivers, 2.1M rays,
    1.3e8 hits): the GPU operator's forward and adjoint products of integer
    probes (weight 1 per hit) equal the reference projector's exactly - every
    sum is an integer below 2^24 - so each ray's voxel moments (count, index
    residues, a hash) and each voxel's ray moments agree."""
    from test_oracle import moment_probes_3d
    torch = torch_cuda
    g = W.hemisphere_geometry(128, 2048, 1024, (128 - 1) / 2.0 - 0.5, np.random.default_rng(2))
    n = 128 ** 3
    op = capi.Operator(capi.ray3d_problem((128, 128, 128), g))
    dy = torch.empty(op.rows, device="cuda")
    for p in moment_probes_3d(n):
        op.apply(_dev(torch, p), dy)
        np.testing.assert_array_equal(dy.cpu().numpy().astype(np.float64), O.ref_project3d(g, p))
    q = ((np.arange(op.rows, dtype=np.int64) * 40503) % 211).astype(np.float64)
    dx = torch.empty(op.cols, device="cuda")
    op.apply(_dev(torch, q), dx, trans=True)
    np.testing.assert_array_equal(dx.cpu().numpy().astype(np.float64), O.ref_project3d(g, q, trans=True))
    op.close()


def test_gaussian_device_equals_host(torch_cuda):
    """tval3g_gaussian on the device gives the host stream: the integer
    streams are identical and every element agrees to one FP32 unit in the
    last place (the FP64 log / sin / cos of the two math libraries), almost
    all of them bit for bit."""
    torch = torch_cuda
    for seed, off, cnt, sc in [(5, 0, 1 << 20, 1.0), ((1 << 35) + 11, 3, 100003, 1 / 64.0)]:
        d = torch.empty(cnt, device="cuda")
        capi.gaussian(d, seed, sc, off)
        got = d.cpu().numpy()
        want = capi.gaussian_host(cnt, seed, sc, off)
        ulp = np.abs(got.view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64))
        print(f"seed {seed}: {np.count_nonzero(ulp)} of {cnt} elements differ (max {ulp.max()} ulp)")
        assert ulp.max() <= 1 and np.count_nonzero(ulp) <= cnt * 1e-4


@pytest.mark.parametrize("name", ["ring2d_s64_it20", "hemi3d_s16_it20", "hemi3d_mp2_s16"])
def test_ray_adjoint_atomics_variant(name, torch_cuda):
    """The adjoint by on-the-fly tracing with atomic adds
    (TVAL3G_RAY_ADJ_ATOMICS) against the FP64 oracle (1e-5) and against the
    default gather form; a solve built with it stays within the solve bar of
    the default form."""
    torch = torch_cuda
    c = build_case(name)
    spec = api_problem(c, capi)
    op = capi.Operator(spec, adj_atomics=True)
    y = np.random.default_rng(4).standard_normal(op.rows).astype(np.float32)
    dx = torch.empty(op.cols, device="cuda")
    op.apply(_dev(torch, y), dx, trans=True)
    op.close()
    e = relerr(dx.cpu().numpy(), c["oracle_op"].apply(y.astype(np.float64), trans=True))
    print(f"{name}: atomics adjoint vs FP64 {e:.2e}")
    assert e < 1e-5


def test_solve_with_atomics_adjoint(torch_cuda):
    """A well-conditioned 64x64 ring (hit weight 1/sigma_max), 20 iterations:
    the solve with the atomics adjoint equals the default one within the
    suite's bar for short solves, 1e-3 (the atomic adds' order varies from
    run to run, so the distance does too: about 1e-4 measured)."""
    torch = torch_cuda
    w = W.ring2d(seed=1, side=64, T=64, tv_norm=1, maxit=20, tol=1e-5, normalize=True)
    spec = capi.problem_from_workload(w)
    plan = capi.Plan([spec], [w["opts"]], adj_atomics=True)
    du = [torch.empty(spec.n, device="cuda")]
    info = plan.solve([_dev(torch, w["b"])], du)[0]
    plan.close()
    U0, info0 = capi.solve(spec, w["b"], w["opts"])
    e = relerr(du[0].cpu().numpy(), U0)
    print(f"solve with the atomics adjoint vs the gather form: {e:.2e}")
    assert info["total_iters"] == info0["total_iters"] == 20
    assert e < BAR


@pytest.mark.parametrize("which", ["ring2d_s64_it20", "hemi3d_s16_it20", "hemi3d_mp2_s16", "ragged3d"])
def test_tiled_adjoint_equals_plain_gather(which, torch_cuda):
    """The tiled adjoint (2D tiles; 3D bricks of 8 x 8 x 4 voxels with their
    rays' measurements staged in shared memory and 16-bit positions) against
    the plain pixel-major gather (TVAL3G_RAY_ADJ_PLAIN) and the FP64 oracle,
    on a volume whose sides are not multiples of the brick."""
    torch = torch_cuda
    if which == "ragged3d":
        g = W.hemisphere_geometry(20, 96, 24, 8.5, np.random.default_rng(8))
        g = dict(g, rv_x=20, rv_y=20, rv_z=20)
        shape = (20, 20, 20)
        spec, ref = capi.ray3d_problem(shape, g), O.Op.ray3d(g)
    else:
        c = build_case(which)
        spec, ref = api_problem(c, capi), c["oracle_op"]
    tiled, plain = capi.Operator(spec), capi.Operator(spec, adj_plain=True)
    y = np.random.default_rng(2).standard_normal(tiled.rows).astype(np.float32)
    a, b = torch.empty(tiled.cols, device="cuda"), torch.empty(tiled.cols, device="cuda")
    tiled.apply(_dev(torch, y), a, trans=True)
    plain.apply(_dev(torch, y), b, trans=True)
    e64 = relerr(a.cpu().numpy(), ref.apply(y.astype(np.float64), trans=True))
    ep = relerr(a.cpu().numpy(), b.cpu().numpy())
    print(f"{which}: tiled adjoint vs FP64 {e64:.2e}, vs the plain gather {ep:.2e}; index bytes "
          f"{tiled.adjoint_index_bytes} (tiled) vs {plain.adjoint_index_bytes} (plain)")
    assert e64 < 1e-5 and ep < 1e-6
    tiled.close()
    plain.close()
