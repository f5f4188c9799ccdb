"""Complex data on the GPU (the reference's complex<float> overloads,
2d/tval3_cpu_2d.cpp:913-929 and the sparse and geometry ones).

The FP64 anchors are the reference's own complex<double> build and the FP64
oracle's complex mode (oracle.solve_complex: the real form of the operator
on planar vectors), which equals that build to 1e-12 after 20 iterations and
to 1e-7 at convergence (tests/test_oracle.py).  After 20 iterations the GPU
solution is compared with the reference's complex<double> build; the full
solve with the complex oracle's own solve, within 1e-3 relative L2 or twice
the problem's FP32 noise floor where that is larger (helpers.noise_floor:
how far FP64 solves move under one FP32 rounding per stored element and
iteration); the distance to the oracle replaying the GPU's recorded
decisions is printed beside it.  The engine solves the real form of the problem on planar vectors
(real plane, imaginary plane) with the complex shrinkage coupling the planes;
the operator tests check that real form against numpy's complex products.
"""
import numpy as np
import pytest

import oracle as O
from golden.cases import COMPLEX_CASES, api_problem, build_case, complex_oracle_op
from helpers import golden, noise_floor, relerr, solve_bar
from tval3g import capi

pytestmark = pytest.mark.gpu

BAR = 1e-3


@pytest.mark.parametrize("name", COMPLEX_CASES)
def test_complex_fixed_iterations_match_reference(name, torch_cuda):
    """20 iterations: against the reference's complex<double> build."""
    c = build_case(name)
    g = golden(f"{name}.npz")
    U, info = capi.solve(api_problem(c, capi), c["b"], dict(c["opts"], maxit=20))
    assert U.dtype == np.complex64 and info["status"] == 0 and info["total_iters"] == 20
    e = relerr(U, g["ref4_U_it20"])
    print(f"{name}: 20 iterations, relerr vs the reference's complex<double> build {e:.3e} (its complex<float> "
          f"build {relerr(g['ref3_U_it20'], g['ref4_U_it20']):.3e})")
    assert e < BAR, (name, e)


def _interleaved(x):
    x = np.asarray(x).ravel()
    out = np.empty(2 * x.size, np.float32)
    out[0::2], out[1::2] = x.real, x.imag
    return out


@pytest.mark.parametrize("name", COMPLEX_CASES)
def test_complex_solve_matches_reference(name, torch_cuda):
    """The full solve under the reference's stopping rules against the FP64
    complex oracle (which equals the reference's complex<double> build to
    1e-6 here), under the noise-floor bar; the replayed comparison and the
    reference's build are printed."""
    torch = torch_cuda
    c = build_case(name)
    g = golden(f"{name}.npz")
    spec = api_problem(c, capi)
    plan = capi.Plan([spec], [c["opts"]], graph=True, trace=True)
    db = [torch.tensor(_interleaved(c["b"]), device="cuda")]
    du = [torch.empty(2 * spec.n, device="cuda")]
    info = plan.solve(db, du)[0]
    tr = plan.trace(0)
    plan.close()
    assert info["status"] == 0
    Ui = du[0].cpu().numpy()
    U = (Ui[0::2] + 1j * Ui[1::2]).reshape(c["shape"])
    op = complex_oracle_op(c)
    solve = lambda extra: O.solve_complex(op, c["b"], c["shape"], dict(c["opts"], **extra))  # noqa: E731
    r = solve({})
    floor = noise_floor(solve, r.U)
    bar = solve_bar(floor)
    e = relerr(U, r.U)
    rr = O.solve_complex(op, c["b"], c["shape"], c["opts"], replay=O.replay_from_trace(tr))
    print(f"{name}: {info['total_iters']} iterations (FP64 {r.total_iters}); relerr vs FP64 {e:.3e}, bar {bar:.2e} "
          f"(FP32 noise floor {floor:.2e}); vs FP64 replaying the GPU's decisions {relerr(U, rr.U):.3e}; vs the "
          f"reference's complex<double> build {relerr(U, g['ref4_U']):.3e}")
    assert e < bar, (name, e, bar)
    U2, info2 = capi.solve(spec, c["b"], c["opts"], Ut=c["u_true"])
    assert abs(info2["rel_error"] - relerr(U2, c["u_true"])) < 1e-5


def _planar(x):
    return np.concatenate([x.real, x.imag]).astype(np.float32)


@pytest.mark.parametrize("name", COMPLEX_CASES)
def test_complex_operator_is_the_real_form(name, torch_cuda):
    """Operator on planar vectors: [Re A x; Im A x] and [Re A^H y; Im A^H y]."""
    torch = torch_cuda
    c = build_case(name)
    op = capi.Operator(api_problem(c, capi))
    rng = np.random.default_rng(3)
    n, m = op.cols // 2, op.rows // 2       # complex lengths, all layers
    L = c.get("layers", 1)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y = rng.standard_normal(m) + 1j * rng.standard_normal(m)
    if "A" in c:
        A = c["A"].astype(np.complex128)
        fwd = lambda v: A @ v            # noqa: E731
        adj = lambda v: A.conj().T @ v   # noqa: E731
    else:
        csr = c["csr"]
        rows = np.repeat(np.arange(csr["m"]), np.diff(csr["rowptr"]))
        val = csr["val"].astype(np.complex128)

        def fwd(v):
            out = np.zeros(csr["m"], complex)
            np.add.at(out, rows, val * v[csr["colind"]])
            return out

        def adj(v):
            out = np.zeros(csr["n"], complex)
            np.add.at(out, csr["colind"], val.conj() * v[rows])
            return out
    Ax = np.concatenate([fwd(xl) for xl in x.reshape(L, -1)])      # layer by layer
    Ahy = np.concatenate([adj(yl) for yl in y.reshape(L, -1)])
    dx = torch.tensor(_planar(x), device="cuda")
    dy = torch.tensor(_planar(y), device="cuda")
    out_m = torch.empty(2 * m, device="cuda")
    out_n = torch.empty(2 * n, device="cuda")
    op.apply(dx, out_m)
    op.apply(dy, out_n, trans=True)
    torch.cuda.synchronize()
    got_m, got_n = out_m.cpu().numpy(), out_n.cpu().numpy()
    op.close()
    assert relerr(got_m[:m] + 1j * got_m[m:], Ax) < 1e-6
    assert relerr(got_n[:n] + 1j * got_n[n:], Ahy) < 1e-6


def test_complex_data_with_real_values_is_the_real_solve(torch_cuda):
    """Complex data whose imaginary parts are 0 stay real: the solution's
    imaginary part is exactly 0 and its real part is the real solve's."""
    c = build_case("dense2d_s32_it20")
    Ur, ir = capi.solve(capi.dense_problem(c["shape"], c["A"]), c["b"], c["opts"])
    Uc, ic = capi.solve(capi.dense_problem(c["shape"], c["A"].astype(np.complex64)), c["b"].astype(np.complex64),
                        c["opts"])
    assert np.all(Uc.imag == 0)
    assert ic["total_iters"] == ir["total_iters"]
    assert relerr(Uc.real, Ur) < 1e-4


def test_complex_batch_equals_single_bitwise(torch_cuda):
    names = ["cdense2d_s32", "ccsr2d_s32", "dense2d_s32_it20", "cring2d_s64"]
    cases = [build_case(n) for n in names]
    specs = [api_problem(c, capi) for c in cases]
    ub, ib = capi.solve_batch(specs, [c["b"] for c in cases], [c["opts"] for c in cases])
    for k, c in enumerate(cases):
        us, is_ = capi.solve_batch([specs[k]], [c["b"]], [c["opts"]])
        np.testing.assert_array_equal(ub[k], us[0])
        assert ib[k]["total_iters"] == is_[0]["total_iters"]


def test_complex_operator_needs_host_arrays(torch_cuda):
    c = build_case("cdense2d_s32")
    with pytest.raises(capi.TVAL3Error) as e:
        capi.Plan([api_problem(c, capi)], [c["opts"]], device_inputs=True)
    assert str(e.value) == "Argument error: complex operators must be given in host memory"


def test_complex_isreal_keeps_the_real_part(torch_cuda):
    """isreal (2d:855-859): the solve is the same, the returned U is the real
    part of the complex solution (then scaled), rel_error measured on it."""
    c = build_case("cdense2d_s32")
    spec = api_problem(c, capi)
    o = dict(c["opts"], maxit=20)
    U, _ = capi.solve(spec, c["b"], o)
    Ur, info = capi.solve(spec, c["b"], dict(o, isreal=1), Ut=c["u_true"])
    assert np.all(Ur.imag == 0)
    np.testing.assert_array_equal(Ur.real, U.real)
    assert abs(info["rel_error"] - relerr(Ur, c["u_true"])) < 1e-5


def test_complex_isotropic_tv_with_real_values_is_the_real_solve(torch_cuda):
    """Isotropic TV (no reference counterpart) on complex data shrinks by the
    modulus over both components and both planes; with imaginary parts 0 it
    is the real isotropic solve."""
    c = build_case("dense2d_s32_it20")
    o = dict(c["opts"], tv_norm=1)
    Ur, ir = capi.solve(capi.dense_problem(c["shape"], c["A"]), c["b"], o)
    Uc, ic = capi.solve(capi.dense_problem(c["shape"], c["A"].astype(np.complex64)), c["b"].astype(np.complex64), o)
    assert np.all(Uc.imag == 0) and ic["total_iters"] == ir["total_iters"]
    assert relerr(Uc.real, Ur) < 1e-4
