"""GPU solver parity through the C ABI.

Tolerances (relative L2 of U):
* at 20 iterations the float reference and the FP64 restatement agree to
  ~5e-5, so the GPU solution must be within 1e-3 of both;
* at convergence (tol-stopped) the reference's own float build is up to ~7e-3
  away from its double build (tests/test_oracle.py), so the GPU solution must
  be within 2e-2 of the FP64 oracle and of the float reference;
* graph and plain execution, and batched and single solves, run the same
  kernels in the same order with deterministic reductions: bit-identical.
"""
import numpy as np
import pytest

from golden.cases import CASES, api_problem, build_case
from helpers import golden, relerr
from tval3g import capi

pytestmark = pytest.mark.gpu

TOL = {"it20": 1e-3, "conv": 2e-2, "layers": 2e-3, "iso": 2e-3, "nonneg": 2e-3, "skip": 2e-3, "s16": 1e-3,
       "s8": 2e-3}


def _tol(name):
    return TOL[name.split("_")[-1]]


@pytest.mark.parametrize("name", CASES)
def test_solve_matches_oracle_and_reference(name, torch_cuda):
    c = build_case(name)
    g = golden(f"{name}.npz")
    U, info = capi.solve(api_problem(c, capi), c["b"], c["opts"], Ut=c["u_true"])
    assert info["status"] == 0
    e_or = relerr(U, g["oracle_U"])
    assert e_or < _tol(name), (name, e_or, info)
    if "ref0_U" in g:
        e_ref = relerr(U, g["ref0_U"])
        assert e_ref < _tol(name), (name, e_ref, info)
    if name.endswith("it20"):
        assert info["total_iters"] == 20
    # rel_error is ||Ut - U|| / ||Ut|| of the returned U
    assert abs(info["rel_error"] - relerr(U, c["u_true"])) < 1e-5


def _plan_run(torch, specs, bs, opts, graph):
    plan = capi.Plan(specs, opts, graph=graph)
    db = [torch.tensor(np.ascontiguousarray(b, np.float32), device="cuda") for b in bs]
    du = [torch.empty(s.n, device="cuda") for s in specs]
    infos = plan.solve(db, du)
    out = [u.cpu().numpy() for u in du]
    stats = plan.stats()
    plan.close()
    return out, infos, stats


@pytest.mark.parametrize("name", ["ring2d_s64_conv", "dense2d_s32_conv", "hemi3d_s16_it20"])
def test_graph_equals_plain_bitwise(name, torch_cuda):
    torch = torch_cuda
    c = build_case(name)
    spec = api_problem(c, capi)
    ug, ig, sg = _plan_run(torch, [spec], [c["b"]], [c["opts"]], graph=True)
    up, ip, sp = _plan_run(torch, [spec], [c["b"]], [c["opts"]], graph=False)
    np.testing.assert_array_equal(ug[0], up[0])
    assert ig[0]["total_iters"] == ip[0]["total_iters"]
    assert sg["kernel_launches"] > 0 and sp["kernel_launches"] > 0


def test_batch_equals_single_bitwise(torch_cuda):
    torch = torch_cuda
    names = ["dense2d_s32_conv", "ring2d_s64_conv", "ring2d_s64_iso", "ring2d_s64_skip", "hemi3d_s16_it20",
             "dense3d_s8", "dense2d_layers"]
    cases = [build_case(n) for n in names]
    specs = [api_problem(c, capi) for c in cases]
    ub, ib, _ = _plan_run(torch, specs, [c["b"] for c in cases], [c["opts"] for c in cases], graph=True)
    for k, c in enumerate(cases):
        us, is_, _ = _plan_run(torch, [specs[k]], [c["b"]], [c["opts"]], graph=True)
        np.testing.assert_array_equal(ub[k], us[0])
        assert ib[k]["total_iters"] == is_[0]["total_iters"]


def test_host_batch_api(torch_cuda):
    names = ["dense2d_s32_it20", "ring2d_s64_it20"]
    cases = [build_case(n) for n in names]
    Us, infos = capi.solve_batch([api_problem(c, capi) for c in cases], [c["b"] for c in cases],
                                 [c["opts"] for c in cases])
    for c, U in zip(cases, Us):
        U1, _ = capi.solve(api_problem(c, capi), c["b"], c["opts"])
        np.testing.assert_array_equal(U, U1)


def test_nonfinite_data_stops_with_status(torch_cuda):
    c = build_case("dense2d_s32_it20")
    b = c["b"].copy()
    b[3] = np.nan
    with pytest.raises(capi.TVAL3Error) as e:
        capi.solve(api_problem(c, capi), b, c["opts"])
    assert e.value.code == capi.ERR_NONFINITE


def test_plan_reuse_is_deterministic(torch_cuda):
    torch = torch_cuda
    c = build_case("ring2d_s64_conv")
    spec = api_problem(c, capi)
    plan = capi.Plan([spec], [c["opts"]], graph=True)
    db = [torch.tensor(c["b"], device="cuda")]
    outs = []
    for _ in range(3):
        du = [torch.empty(spec.n, device="cuda")]
        plan.solve(db, du)
        outs.append(du[0].cpu().numpy())
    plan.close()
    np.testing.assert_array_equal(outs[0], outs[1])
    np.testing.assert_array_equal(outs[0], outs[2])
