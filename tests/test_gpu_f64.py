"""The FP64 engine behind tval3g_solve_f64 and the drop-in's double and
complex<double> overloads (2d/tval3_cpu_2d.cpp:905-1016,
3d/tval3_cpu_3d.cpp:1408-1581), whose reference instantiations compute in
double.

Anchor: the reference's own double build (fixtures ref2_U) and
complex<double> build (ref4_U, ref4_U_it20), given the same inputs in double,
at the same iteration count.  How close two FP64 solves that differ only in
summation order can be is measured by the FP64 oracle (an independent
restatement with its own loop order) against the same build: about 1e-14 -
1e-12 after 20 - 40 iterations and 1e-11 - 1e-7 on converged solves.  The GPU
is held to 100 times that distance and never more than 1e-10 on the fixed
short solves; isotropic TV, which the reference lacks, against the FP64
oracle at 1e-10.
"""
import numpy as np
import pytest

import oracle as O
from golden.cases import COMPLEX_CASES, api_problem, build_case, complex_oracle_op
from helpers import golden, relerr
from tval3g import capi

pytestmark = pytest.mark.gpu

REAL_CASES = ["dense2d_s32_it20", "dense2d_s32_conv", "dense2d_layers", "ring2d_s64_it20", "ring2d_s64_conv",
              "ring2d_s64_nonneg", "ring2d_s64_skip", "hemi3d_s16_it20", "hemi3d_s16_conv", "csr3d_s16",
              "dense3d_s8", "hemi3d_mp2_s16", "csr2d_layers"]


def _values(c):
    """The operator's values in double (dense A or CSR values), or None."""
    if c["api"] == "dense":
        return np.asarray(c["A"]).astype(np.complex128 if np.iscomplexobj(c["A"]) else np.float64)
    if c["api"] == "csr":
        v = np.asarray(c["csr"]["val"])
        return v.astype(np.complex128 if np.iscomplexobj(v) else np.float64)
    return None


def _bar(d_oracle):
    return max(1e-10, 100.0 * d_oracle)


@pytest.mark.parametrize("name", REAL_CASES)
def test_f64_solve_matches_reference_double_build(name, torch_cuda):
    c = build_case(name)
    g = golden(f"{name}.npz")
    U, info = capi.solve_f64(api_problem(c, capi), c["b"].astype(np.float64), c["opts"], values=_values(c))
    assert U.dtype == np.float64 and info["status"] == 0
    assert info["total_iters"] == int(g["ref2_iters"][1]) and info["outer_iters"] == int(g["ref2_iters"][0])
    e = relerr(U, g["ref2_U"])
    d = relerr(g["oracle_U"], g["ref2_U"])
    bar = _bar(d)
    print(f"{name}: FP64 engine vs the reference's double build {e:.2e} (bar {bar:.1e}; the FP64 oracle {d:.2e}; "
          f"the FP32 engine's class: the reference's float build {relerr(g['ref0_U'], g['ref2_U']):.2e})")
    assert e <= bar, (name, e, bar)


def test_f64_isotropic_matches_oracle(torch_cuda):
    name = "ring2d_s64_iso"
    c = build_case(name)
    g = golden(f"{name}.npz")
    U, info = capi.solve_f64(api_problem(c, capi), c["b"].astype(np.float64), c["opts"])
    assert info["status"] == 0 and info["total_iters"] == int(g["oracle_iters"][1])
    e = relerr(U, g["oracle_U"])
    print(f"{name}: FP64 engine vs the FP64 oracle {e:.2e}")
    assert e <= 1e-10


@pytest.mark.parametrize("name", COMPLEX_CASES)
def test_f64_complex_matches_reference_complex_double_build(name, torch_cuda):
    c = build_case(name)
    g = golden(f"{name}.npz")
    spec = api_problem(c, capi)
    b = np.asarray(c["b"]).astype(np.complex128)
    U20, info20 = capi.solve_f64(spec, b, dict(c["opts"], maxit=20), values=_values(c))
    assert U20.dtype == np.complex128 and info20["status"] == 0 and info20["total_iters"] == 20
    e20 = relerr(U20, g["ref4_U_it20"])
    U, info = capi.solve_f64(spec, b, c["opts"], values=_values(c))
    assert info["status"] == 0 and info["total_iters"] == int(g["ref4_iters"][1])
    e = relerr(U, g["ref4_U"])
    # the FP64 oracle's own complex solve (the fixture's complex oracle_U is
    # the reference's)
    r = O.solve_complex(complex_oracle_op(c), c["b"], c["shape"], c["opts"])
    assert r.total_iters == info["total_iters"]
    d = relerr(r.U, g["ref4_U"])
    bar = _bar(d)
    print(f"{name}: FP64 engine vs the reference's complex<double> build after 20 iterations {e20:.2e}, full solve "
          f"({info['total_iters']} iterations) {e:.2e} (bar {bar:.1e}; the FP64 oracle {d:.2e})")
    assert e20 <= 1e-10, (name, e20)
    assert e <= bar, (name, e, bar)


def test_f64_argument_errors_match_float_path(torch_cuda):
    """Validation is shared with the float entry point: the reference's
    messages."""
    c = build_case("dense2d_s32_it20")
    spec = api_problem(c, capi)
    with pytest.raises(capi.TVAL3Error) as e:
        capi.solve_f64(spec, np.zeros(c["b"].size + 1), c["opts"], values=_values(c))
    assert "b.len must be equal to A.dim_y" in str(e.value)
    with pytest.raises(capi.TVAL3Error) as e:
        capi.solve_f64(spec, c["b"].astype(np.float64), c["opts"], values=None)
    assert "A is NULL" in str(e.value)
