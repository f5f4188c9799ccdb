"""The C++ drop-in libraries: same exported symbols as the reference, same
argument errors, and (GPU) the same results as the C ABI."""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O
from helpers import ROOT

LIB = os.path.join(ROOT, "tval3-cpu_b200", "lib")


def _exports(path, name):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    # the public overloads (not the driver's template instantiations)
    return {s for s in re.findall(rf"(_Z12{name}R\S+)", out)}


@pytest.mark.parametrize("dims", [2, 3])
def test_exports_the_reference_overloads(dims):
    name = f"tval3_cpu_{dims}d"
    ours = _exports(os.path.join(LIB, f"libtval3_gpu_{dims}d.so"), name)
    assert len(ours) == 15
    if O.ref_available(dims):
        ref = _exports(os.path.join(ROOT, "oracle", "_ref", f"libref_tval3_{dims}d.so"), name)
        assert ours == ref


@pytest.fixture(scope="module")
def demo(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("dropin") / "dropin_demo")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "dropin_demo.cpp"), "-o", exe, "-L", LIB, "-ltval3_gpu_2d",
                    "-ltval3g", f"-Wl,-rpath,{LIB}"], check=True)
    return exe


def test_argument_errors_match_reference(demo):
    out = subprocess.run([demo, "errors"], capture_output=True, text=True, check=True).stdout.strip().splitlines()
    got = dict(line.split(": ", 1) for line in out)
    assert got["format"] == "Argument error: Matrices must be in row major format!"
    assert got["ut"] == "Argument error: U and Ut must have the same size!"
    assert got["ulen"] == "Argument error: the length of U must be equal to A.dim_x * layers!"
    assert got["blen"] == "Argument error: b.len must be equal to A.dim_y * layers!"
    assert got["csc"] == "Argument error: A must be available in CSR and CSC format!"
    assert got["geom_layers_or_blen"] == "Argument error: b.len must be equal to A.num_emitters * A.num_receivers!"
    assert got["double"] == "Argument error: Matrices must be in row major format!"   # checked as for float
    assert got["complex"] == "Argument error: b.len must be equal to A.dim_y * layers!"
    assert got["complex_format"] == "Argument error: Matrices must be in row major format!"
    if O.ref_available(2):   # the reference itself, same arguments
        opts = dict(mu=256.0, beta=32.0, mu0=256.0, beta0=32.0, tol=1e-4, tol_inn=1e-3, c=1e-5, gamma=0.6,
                    gam=0.9995, rate_gam=0.9, rate_cnt=2.0, maxit=30, maxcnt=10)
        A = np.zeros((20, 64), np.float32)
        for fmts, blen, msg in [((0, 0, 1), 20, got["format"]), ((1, 0, 1), 21, got["blen"])]:
            with pytest.raises(O.ReferenceError) as e:
                O.ref_solve("dense", (8, 8), np.zeros(blen, np.float32), opts, A=A, formats=fmts)
            assert str(e.value) == msg


@pytest.mark.gpu
def test_dropin_solves_equal_c_abi(demo, torch_cuda):
    out = subprocess.run([demo, "solve"], capture_output=True, text=True, check=True).stdout.strip().splitlines()
    rows = {line.split()[0]: line.split()[1:] for line in out}
    for case in ("dense", "dense_f64", "csr", "ray2d", "ray2d_f64", "cdense"):
        rc, diff, it1, it2 = rows[case][:4]
        assert rc == "0" and float(diff) == 0.0 and it1 == it2, (case, rows[case])
    # double data is solved in double: not the float solve of the same values
    print("dense: double overload vs the float solve of the same values", rows["dense_f64"][4])
    assert float(rows["dense_f64"][4]) > 0.0
