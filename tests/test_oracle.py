"""The oracle pinned against the reference (no GPU).

The reference ships no tests or golden vectors, so the FP64 restatement is
pinned against the reference itself: its own sources compiled unchanged
(oracle/_ref), whose outputs on seeded problems are the golden fixtures in
tests/golden (written by tests/golden/make_golden.py).
"""
import os

import numpy as np
import pytest

import oracle as O
from helpers import golden, relerr
from tval3g import workloads as W

from golden.cases import CASES, COMPLEX_CASES, build_case  # noqa: E402


def _checksum(a):
    a = np.asarray(a, np.float64).ravel()
    return np.array([a.size, a.sum(), np.abs(a).sum(), (a * np.arange(a.size) % 7.0).sum()])


@pytest.mark.parametrize("name", CASES)
def test_inputs_regenerate_bit_identically(name):
    c = build_case(name)
    g = golden(f"{name}.npz")
    np.testing.assert_array_equal(_checksum(c["b"]), g["b_sum"])
    if "A" in c:
        np.testing.assert_array_equal(_checksum(c["A"]), g["A_sum"])


@pytest.mark.parametrize("name", [n for n in CASES if n != "ring2d_s64_iso"])
def test_restatement_matches_reference_fp64(name):
    """FP64 oracle == the reference's double build (same iteration counts)."""
    c = build_case(name)
    g = golden(f"{name}.npz")
    r = O.solve(c["oracle_op"], c["b"].astype(np.float64), c["shape"], c["opts"])
    assert tuple(g["ref2_iters"]) == (r.outer_iters, r.total_iters)
    assert relerr(r.U, g["ref2_U"]) < 1e-6
    np.testing.assert_allclose(r.U, g["oracle_U"], rtol=0, atol=1e-12 * np.abs(g["oracle_U"]).max())


def test_reference_float_build_drift_documented():
    """The reference's own float build drifts from its double build: this is
    why solver parity tolerances are stated per iteration count."""
    g = golden("dense2d_s32_it20.npz")
    assert relerr(g["ref0_U"], g["ref2_U"]) < 1e-3
    g = golden("dense2d_s32_conv.npz")
    assert relerr(g["ref0_U"], g["ref2_U"]) < 2e-2


@pytest.mark.parametrize("name", COMPLEX_CASES)
def test_complex_inputs_regenerate_bit_identically(name):
    c = build_case(name)
    g = golden(f"{name}.npz")
    np.testing.assert_array_equal(_checksum(np.concatenate([c["b"].real, c["b"].imag])), g["b_sum"])
    if "A" in c:
        np.testing.assert_array_equal(_checksum(np.concatenate([c["A"].real.ravel(), c["A"].imag.ravel()])),
                                      g["A_sum"])


def test_complex_reference_float_drift_documented():
    """The reference's complex<float> build against its complex<double>
    build (the FP64 anchor of the complex cases): the GPU bar is twice this."""
    drift = {n: relerr(golden(f"{n}.npz")["ref3_U"], golden(f"{n}.npz")["ref4_U"]) for n in COMPLEX_CASES}
    assert drift["cdense2d_s32"] < 2e-2 and drift["ccsr2d_s32"] < 1e-3 and drift["cring2d_s64"] < 5e-2, drift
    for n in COMPLEX_CASES:   # the anchor is the complex<double> solution, complex-valued
        g = golden(f"{n}.npz")
        assert np.iscomplexobj(g["oracle_U"]) and np.abs(g["oracle_U"].imag).max() > 0.05


@pytest.mark.skipif(not O.ref_available(2), reason="reference not built here")
def test_complex_reference_live_matches_fixture(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    c = build_case("ccsr2d_s32")
    g = golden("ccsr2d_s32.npz")
    r = O.ref_solve("csr", c["shape"], c["b"], c["opts"], dtype=4, csr=c["csr_tuple"], Ut=c["u_true"])
    np.testing.assert_array_equal(r.U, g["ref4_U"])


@pytest.mark.skipif(not O.ref_available(2), reason="reference not built here")
def test_reference_live_matches_fixture(tmp_path, monkeypatch):
    c = build_case("dense2d_s32_it20")
    g = golden("dense2d_s32_it20.npz")
    r = O.ref_solve("dense", c["shape"], c["b"], c["opts"], dtype=2, A=c["A"])
    np.testing.assert_array_equal(r.U, g["ref2_U"])


# --------------------------------------------------------------------------
# Bresenham: closed form (product generator / kernels) == recurrence (oracle)
# --------------------------------------------------------------------------
EDGE_RAYS_2D = [  # (x0, y0, x1, y1)
    (0, 0, 7, 0), (0, 0, 0, 7), (7, 7, 0, 0), (0, 0, 7, 7), (7, 0, 0, 7), (2, 3, 2, 3), (1, 1, 6, 3),
    (6, 3, 1, 1), (1, 6, 3, 0), (3, 0, 1, 6), (0, 7, 7, 6), (5, 2, 0, 4),
]


def test_bresenham_2d_edge_cases():
    ld = 8
    x0, y0, x1, y1 = (np.array(v) for v in zip(*EDGE_RAYS_2D))
    g = dict(use_path=np.ones(len(x0) * len(x0), np.int32), xe=x0, ye=y0, xr=x1, yr=y1, ld=ld, scale=1.0)
    # one emitter per ray, paired with its own receiver
    use = np.eye(len(x0), dtype=np.int32).ravel()
    g["use_path"] = use
    op = O.Op.ray2d(g, 64)
    ray, off, pix = op.ray_lists()
    coff, cpix = W.bresenham_csr_2d(x0, y0, x1, y1, ld)
    np.testing.assert_array_equal(off, coff)
    np.testing.assert_array_equal(pix, cpix)
    # both endpoints included; zero-length ray has one pixel
    assert off[6] - off[5] == 1


def test_bresenham_3d_ties_and_edges():
    p0 = np.array([[0, 0, 0], [0, 0, 0], [0, 0, 0], [5, 5, 5], [1, 2, 3], [7, 0, 3], [3, 3, 3], [0, 7, 7]])
    p1 = np.array([[7, 7, 0], [0, 7, 7], [7, 0, 7], [0, 0, 0], [6, 4, 7], [0, 7, 5], [3, 3, 3], [7, 0, 0]])
    N = len(p0)
    g = dict(numMPs=1, numPaths=N, E=N, R=N, use_path=(np.eye(N, dtype=np.int32) * np.arange(1, N + 1)).ravel(),
             xe=p0[:, 0], ye=p0[:, 1], ze=p0[:, 2], xr=p1[:, 0], yr=p1[:, 1], zr=p1[:, 2], rv_x=8, rv_y=8, rv_z=8,
             scale=1.0)
    ray, off, pix = O.Op.ray3d(g).ray_lists()
    coff, cpix = W.bresenham_csr_3d(p0, p1, 8, 8)
    np.testing.assert_array_equal(off, coff)
    np.testing.assert_array_equal(pix, cpix)


def test_bresenham_ring_and_hemisphere_geometries():
    w = W.ring2d(seed=1, side=64, T=64)
    ray, off, pix = O.Op.ray2d(w["geom"], 64 * 64).ray_lists()
    A = w["csr"]
    np.testing.assert_array_equal(pix, A["colind"])
    np.testing.assert_array_equal(ray, np.nonzero(np.diff(A["rowptr"]))[0])
    w = W.hemi3d(seed=2, side=16, T=64, receivers=16, csr=True)
    ray, off, pix = O.Op.ray3d(w["geom"]).ray_lists()
    A = w["csr"]
    order = np.argsort(ray, kind="stable")
    np.testing.assert_array_equal(np.concatenate([pix[off[k]:off[k + 1]] for k in order]), A["colind"])


def test_bresenham_full_ring_geometry_lengths():
    """256x256, 512 transducers: max(|dx|,|dy|)+1 hits per ray (size-independent property)."""
    g = W.ring_geometry(256, 512)
    use = g["use_path"].reshape(512, 512)
    e, r = np.nonzero(use)
    off, pix = W.bresenham_csr_2d(g["xe"][e], g["ye"][e], g["xr"][r], g["yr"][r], 256)
    L = np.maximum(np.abs(g["xr"][r] - g["xe"][e]), np.abs(g["yr"][r] - g["ye"][e])) + 1
    np.testing.assert_array_equal(np.diff(off), L)
    assert pix.min() >= 0 and pix.max() < 65536
    assert len(e) == 131072


# --------------------------------------------------------------------------
# stencils
# --------------------------------------------------------------------------
def test_D_Dt_adjoint_2d():
    rng = np.random.default_rng(0)
    U = rng.standard_normal((5, 7))
    X, Y = rng.standard_normal(35), rng.standard_normal(35)
    Ux, Uy = O.D(U)
    lhs = Ux @ X + Uy @ Y
    rhs = U.ravel() @ O.Dt(X, Y, shape=(5, 7))
    assert abs(lhs - rhs) < 1e-12 * (abs(lhs) + 1)


def test_Dt_3d_is_the_reference_not_the_adjoint():
    """The reference's 3D Dt adds X[last row of slice z-1] - X[first row of slice z]
    on every first row of slices z >= 1 (3d/tval3_cpu_3d.cpp:402-413)."""
    rng = np.random.default_rng(1)
    shape = (3, 4, 5)
    U = rng.standard_normal(shape)
    X, Y, Z = (rng.standard_normal(60) for _ in range(3))
    Ux, Uy, Uz = O.D(U)
    lhs = Ux @ X + Uy @ Y + Uz @ Z
    res = O.Dt(X, Y, Z, shape=shape)
    # exact adjoint + the reference's extra term
    Y3 = Y.reshape(shape)
    extra = np.zeros(shape)
    extra[1:, 0, :] = Y3[:-1, -1, :] - Y3[1:, 0, :]
    assert abs(lhs - U.ravel() @ (res - extra.ravel())) < 1e-12 * (abs(lhs) + 1)
    assert np.abs(extra).max() > 0


def test_shrink_edges():
    beta = 4.0
    ux = np.array([0.25, -0.25, 0.0, 1.0, -1.0, 0.3])
    uy = np.array([0.0, 0.0, 0.0, 0.0, 0.5, -0.1])
    z = np.zeros(6)
    (wx, wy), lam = O.shrink([ux, uy], [z, z], beta, 0)
    # |Ubar| == 1/beta -> 0; 0 -> 0; sign kept
    assert wx[0] == 0 and wx[1] == 0 and wx[2] == 0
    assert wx[3] == 0.75 and wx[4] == -0.75 and wy[4] == 0.25
    (ix, iy), lam_iso = O.shrink([ux, uy], [z, z], beta, 1)
    n4 = np.hypot(ux[4], uy[4])
    assert abs(ix[4] - (n4 - 0.25) * ux[4] / n4) < 1e-15
    assert ix[2] == 0 and iy[2] == 0


@pytest.mark.parametrize("name", ["dense2d_s32_conv", "ring2d_s64_skip", "hemi3d_s16_conv", "dense2d_layers"])
def test_replay_of_own_decisions_is_identical(name):
    """The replay mode (the checker for equal-iteration-count parity) follows
    recorded decisions exactly: replaying the oracle's own decisions gives
    the same iterations, backtracking steps, skips and bits."""
    c = build_case(name)
    b = c["b"].astype(np.float64)
    r = O.solve(c["oracle_op"], b, c["shape"], c["opts"], record=True)
    rp = {"count": r.total_iters, "backtracks": [x[3] for x in r.iters], "skipped": [x[4] for x in r.iters],
          "inner_end": r.inner_end}
    r2 = O.solve(c["oracle_op"], b, c["shape"], c["opts"], record=True, replay=rp)
    assert r2.total_iters == r.total_iters and r2.outer_iters == r.outer_iters
    assert r2.iters == r.iters
    np.testing.assert_array_equal(r2.U, r.U)


def test_replay_takes_the_given_path():
    """Replayed decisions that differ from the oracle's own (one extra
    backtracking step, the inner loop ended one iteration early) are taken:
    the iteration records show them, and the image moves away from the
    unforced solve."""
    c = build_case("dense2d_s32_it20")
    b = c["b"].astype(np.float64)
    r = O.solve(c["oracle_op"], b, c["shape"], c["opts"], record=True)
    bt = [x[3] for x in r.iters]
    end = list(r.inner_end)
    k = next(i for i in range(2, len(bt)) if bt[i] == 0)
    bt[k] = 1
    end[3] = 1
    r2 = O.solve(c["oracle_op"], b, c["shape"], c["opts"], record=True,
                 replay={"count": r.total_iters, "backtracks": bt, "skipped": [0] * len(bt), "inner_end": end})
    assert [x[3] for x in r2.iters] == bt
    assert r2.inner_end[3] == 1 and r2.total_iters == r.total_iters
    assert r2.outer_iters > r.outer_iters
    assert relerr(r2.U, r.U) > 1e-6


def test_replay_from_gpu_trace_rows():
    """replay_from_trace reads the plan trace's columns (backtracks, skipped,
    outer update flag): the inner loop ends where the multipliers were
    updated, and at the last iteration."""
    tr = np.zeros((5, 8))
    tr[:, 3] = [0, 2, 0, 6, 1]
    tr[:, 4] = [0, 0, 1, 0, 0]
    tr[1, 7] = 1
    rp = O.replay_from_trace(tr)
    assert rp["count"] == 5
    assert list(rp["backtracks"]) == [0, 2, 0, 6, 1] and list(rp["skipped"]) == [0, 0, 1, 0, 0]
    assert list(rp["inner_end"]) == [0, 1, 0, 0, 0]


def _ref_matrix_3d(g):
    """The reference's own 3D projector as a dense count matrix (rays x
    voxels), read column by column from its forward applied to one-hot voxel
    vectors (weight 1 per hit)."""
    g = dict(g, scale=1.0)
    nvox = int(g["rv_x"]) * int(g["rv_y"]) * int(g["rv_z"])
    M = np.zeros((int(g["numMPs"]) * int(g["numPaths"]), nvox))
    e = np.zeros(nvox)
    for j in range(nvox):
        e[j] = 1.0
        M[:, j] = O.ref_project3d(g, e)
        e[j] = 0.0
    return M


def _list_matrix(op_lists, rows, nvox):
    ray, off, pix = op_lists
    M = np.zeros((rows, nvox))
    for k in range(len(ray)):
        np.add.at(M[ray[k]], pix[off[k]:off[k + 1]], 1.0)
    return M


def _tie_geometry():
    p0 = np.array([[0, 0, 0], [0, 0, 0], [0, 0, 0], [5, 5, 5], [1, 2, 3], [7, 0, 3], [3, 3, 3], [0, 7, 7],
                   [2, 2, 0], [7, 7, 7]])
    p1 = np.array([[7, 7, 0], [0, 7, 7], [7, 0, 7], [0, 0, 0], [6, 4, 7], [0, 7, 5], [3, 3, 3], [7, 0, 0],
                   [2, 5, 7], [0, 1, 2]])
    N = len(p0)
    return dict(numMPs=1, numPaths=N, E=N, R=N, use_path=(np.eye(N, dtype=np.int32) * np.arange(1, N + 1)).ravel(),
                xe=p0[:, 0], ye=p0[:, 1], ze=p0[:, 2], xr=p1[:, 0], yr=p1[:, 1], zr=p1[:, 2], rv_x=8, rv_y=8,
                rv_z=8, scale=1.0)


def moment_probes_3d(nvox):
    """Integer-valued voxel probes whose projections identify each ray's voxel
    set: the hit count, residues of the voxel index and a multiplicative hash
    (every projection is an integer well below 2^24, exact in FP32 too)."""
    j = np.arange(nvox, dtype=np.int64)
    return [np.ones(nvox), (j % 7).astype(np.float64), (j % 61).astype(np.float64),
            ((j * 2654435761) % 251).astype(np.float64), ((j // 97) % 13).astype(np.float64)]


@pytest.mark.skipif(not O.ref_available_proj3d(), reason="reference not built here")
def test_bresenham_3d_lists_match_the_reference_projector():
    """The restated 3D Bresenham lists equal the reference's live projector
    (3d/mat_mult.h:148-363) hit for hit: on the tie cases and a 12^3
    hemisphere (one-hot columns), and with two measurement positions."""
    cases = [_tie_geometry(), W.hemisphere_geometry(12, 24, 8, 5.0, np.random.default_rng(4))]
    g2 = dict(cases[1])
    for a, b_ in (("xe", "ye"), ("xr", "yr")):
        x, y = np.asarray(g2[a]), np.asarray(g2[b_])
        g2[a] = np.concatenate([x, 11 - y]).astype(np.int32)
        g2[b_] = np.concatenate([y, x]).astype(np.int32)
    for a in ("ze", "zr"):
        g2[a] = np.concatenate([g2[a], g2[a]]).astype(np.int32)
    g2["numMPs"] = 2
    cases.append(g2)
    for g in cases:
        nvox = int(g["rv_x"]) * int(g["rv_y"]) * int(g["rv_z"])
        rows = int(g["numMPs"]) * int(g["numPaths"])
        Mref = _ref_matrix_3d(g)
        Mor = _list_matrix(O.Op.ray3d(g).ray_lists(), rows, nvox)
        np.testing.assert_array_equal(Mor, Mref)


@pytest.mark.skipif(not O.ref_available_proj3d(), reason="reference not built here")
def test_bresenham_3d_moments_match_the_reference_projector():
    """A 48^3 hemisphere of 256 transducers x 128 receivers (32768 rays):
    per-ray integer moments of the restated lists equal the reference
    projector's products of the same probes (forward), and per-voxel ray
    moments its adjoint."""
    g = W.hemisphere_geometry(48, 256, 128, 23.0, np.random.default_rng(9))
    nvox = 48 ** 3
    rows = int(g["numPaths"])
    ray, off, pix = O.Op.ray3d(g).ray_lists()
    row_of = np.repeat(ray, np.diff(off))
    for p in moment_probes_3d(nvox):
        want = np.zeros(rows)
        np.add.at(want, row_of, p[pix])
        np.testing.assert_array_equal(O.ref_project3d(g, p), want)
    q = ((np.arange(rows, dtype=np.int64) * 40503) % 211).astype(np.float64)
    want = np.zeros(nvox)
    np.add.at(want, pix, q[row_of])
    np.testing.assert_array_equal(O.ref_project3d(g, q, trans=True), want)


@pytest.mark.parametrize("name", COMPLEX_CASES)
def test_complex_restatement_matches_reference(name):
    """The oracle's complex mode (planar vectors, the real form of the
    operator, complex shrinkage, scaleb and Barzilai-Borwein step) against
    the reference's own complex<double> build (the golden fixture): the same
    iteration counts, 1e-12 after 20 iterations, 1e-6 at the end."""
    from golden.cases import complex_oracle_op
    c = build_case(name)
    g = golden(f"{name}.npz")
    op = complex_oracle_op(c)
    r = O.solve_complex(op, c["b"], c["shape"], c["opts"])
    r20 = O.solve_complex(op, c["b"], c["shape"], dict(c["opts"], maxit=20))
    assert r.total_iters == int(g["ref4_iters"][1])
    assert relerr(r20.U, g["ref4_U_it20"]) < 1e-12
    assert relerr(r.U, g["ref4_U"]) < 1e-6


def test_fp32_noise_model():
    """The noise model behind the parity bars' FP32 noise floor: off it
    changes nothing; a few FP32 unit roundoffs per stored element and
    iteration move a fixed 20-iteration solve by about 1e-6 and different
    seeds give different perturbations."""
    from helpers import NOISE_EPS
    c = build_case("dense2d_s32_it20")
    b = c["b"].astype(np.float64)
    r = O.solve(c["oracle_op"], b, c["shape"], c["opts"])
    r0 = O.solve(c["oracle_op"], b, c["shape"], dict(c["opts"], noise=0.0, noise_seed=5))
    np.testing.assert_array_equal(r0.U, r.U)
    r1 = O.solve(c["oracle_op"], b, c["shape"], dict(c["opts"], noise=NOISE_EPS, noise_seed=1))
    r2 = O.solve(c["oracle_op"], b, c["shape"], dict(c["opts"], noise=NOISE_EPS, noise_seed=2))
    assert 1e-9 < relerr(r1.U, r.U) < 1e-4 and relerr(r1.U, r2.U) > 0
