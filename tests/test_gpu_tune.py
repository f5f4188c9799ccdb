"""The launch-shape autotuner (TVAL3G_TUNE): tuned operators give the same
products within rounding, tuned solves stay within the parity bars of the
untuned ones, and the choices are cached per operator signature in memory
and in the file named by TVAL3G_TUNE_CACHE."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from golden.cases import api_problem, build_case
from helpers import ROOT, golden, relerr, solve_bar
from tval3g import capi

pytestmark = pytest.mark.gpu

CASES = ["ring2d_s64_conv", "csr3d_s16", "hemi3d_s16_it20"]


def _bar(name):
    """1e-3, or twice the case's FP32 noise floor (helpers.noise_floor)."""
    from test_gpu_solve import _fp64
    return solve_bar(_fp64(name)[2])


@pytest.mark.parametrize("name", CASES)
def test_tuned_operator_products_match_untuned(name, torch_cuda):
    torch = torch_cuda
    c = build_case(name)
    spec = api_problem(c, capi)
    plain, tuned = capi.Operator(spec), capi.Operator(spec, tune=True)
    print(name, "launch shape (lanes per ray, forward gather, adjoint gather):", tuned.launch_shape())
    rng = np.random.default_rng(1)
    x = torch.tensor(rng.standard_normal(plain.cols).astype(np.float32), device="cuda")
    y = torch.tensor(rng.standard_normal(plain.rows).astype(np.float32), device="cuda")
    for trans, v, size in ((False, x, plain.rows), (True, y, plain.cols)):
        a = torch.empty(size, device="cuda")
        b = torch.empty(size, device="cuda")
        plain.apply(v, a, trans=trans)
        tuned.apply(v, b, trans=trans)
        torch.cuda.synchronize()
        assert relerr(b.cpu().numpy(), a.cpu().numpy()) < 1e-6
    plain.close()
    tuned.close()


@pytest.mark.parametrize("name", CASES)
def test_tuned_solve_within_parity_bar(name, torch_cuda):
    torch = torch_cuda
    c = build_case(name)
    g = golden(f"{name}.npz")
    spec = api_problem(c, capi)
    plan = capi.Plan([spec], [c["opts"]], graph=True, tune=True)
    d_b = torch.tensor(np.ascontiguousarray(c["b"], np.float32), device="cuda")
    d_U = torch.empty(spec.n, device="cuda")
    info = plan.solve([d_b], [d_U])[0]
    plan.close()
    U = d_U.cpu().numpy().reshape(c["shape"])
    assert info["status"] == 0
    bar = _bar(name)
    print(f"{name}: tuned solve, relerr vs FP64 {relerr(U, g['oracle_U']):.3e}, bar {bar:.2e}")
    assert relerr(U, g["oracle_U"]) < bar, (name, relerr(U, g["oracle_U"]))


_CHILD = r"""
import json, sys
sys.path[:0] = [sys.argv[1], sys.argv[2], sys.argv[3]]
from golden.cases import api_problem, build_case
from tval3g import capi
spec = api_problem(build_case("hemi3d_s16_it20"), capi)
shapes = []
for _ in range(2):
    op = capi.Operator(spec, tune=True)
    shapes.append(op.launch_shape())
    op.close()
print(json.dumps({"stats": capi.tune_stats(), "shapes": shapes}))
"""


def test_tuner_caches_per_signature_in_memory_and_on_disk(tmp_path, torch_cuda):
    cache = tmp_path / "tune.tsv"
    env = dict(os.environ, TVAL3G_TUNE_CACHE=str(cache))
    args = [sys.executable, "-c", _CHILD, os.path.join(ROOT, "tests"), os.path.join(ROOT, "tval3-cpu_b200", "python"),
            os.path.join(ROOT, "oracle")]
    runs = []
    for _ in range(2):   # two fresh processes: the second reads the file
        out = subprocess.run(args, env=env, capture_output=True, text=True, check=True).stdout.strip().splitlines()
        runs.append(json.loads(out[-1]))
    first, second = runs
    assert first["stats"] == [1, 1]     # timed once, then found in memory
    assert second["stats"] == [0, 2]    # found in the file both times
    assert first["shapes"][0] == first["shapes"][1] == second["shapes"][0] == second["shapes"][1]
    assert len(cache.read_text().strip().splitlines()) == 1


_CHILD_SOLVE = r"""
import json, sys
sys.path[:0] = [sys.argv[1], sys.argv[2], sys.argv[3]]
from golden.cases import api_problem, build_case
from tval3g import capi
c = build_case("csr3d_s16")
U, info = capi.solve(api_problem(c, capi), c["b"], c["opts"])
print(json.dumps({"stats": capi.tune_stats(), "status": info["status"]}))
"""


def test_drop_in_path_tunes_when_asked_by_the_environment(torch_cuda):
    """tval3g_solve (the path of the C++ overloads) takes no flags: the
    environment variable TVAL3G_TUNE=1 turns the autotuner on for it."""
    args = [sys.executable, "-c", _CHILD_SOLVE, os.path.join(ROOT, "tests"),
            os.path.join(ROOT, "tval3-cpu_b200", "python"), os.path.join(ROOT, "oracle")]
    for value, measured in (("1", 1), ("0", 0)):
        env = dict(os.environ, TVAL3G_TUNE=value)
        env.pop("TVAL3G_TUNE_CACHE", None)
        out = subprocess.run(args, env=env, capture_output=True, text=True, check=True).stdout.strip().splitlines()
        got = json.loads(out[-1])
        assert got["status"] == 0 and got["stats"][0] == measured, (value, got)
