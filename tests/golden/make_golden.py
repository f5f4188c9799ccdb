"""Generate the golden fixtures of the TVAL3 parity tests.

Runs the reference solver itself (modk/tval3-cpu, compiled unchanged from its
own sources by oracle/Makefile into oracle/_ref) and the FP64 oracle
restatement on small seeded problems from tval3g.workloads, and stores their
outputs with checksums of the inputs (the inputs are regenerated from the same
seeds at test time).  Must run where the reference sources are available:

    python tests/golden/make_golden.py [case ...]

The 3D reference prints to stdout and writes profile.txt into the current
directory (3d/tval3_cpu_3d.cpp:1228,1328-1335), so it runs in a temporary
directory.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tval3-cpu_b200", "python"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from tval3g import workloads as W  # noqa: E402

from cases import CASES, COMPLEX_CASES, build_case  # noqa: E402


def checksum(a):
    a = np.asarray(a, np.float64).ravel()
    return np.array([a.size, a.sum(), np.abs(a).sum(), (a * np.arange(a.size) % 7.0).sum()])


def complex_case(name, tmp):
    """Complex data: the reference's complex<float> (dtype 3) and
    complex<double> (dtype 4) builds; the latter is the FP64 anchor."""
    c = build_case(name)
    out = {"b_sum": checksum(np.concatenate([c["b"].real, c["b"].imag]))}
    if "A" in c:
        out["A_sum"] = checksum(np.concatenate([c["A"].real.ravel(), c["A"].imag.ravel()]))
    cwd = os.getcwd()
    os.chdir(tmp)
    try:
        for dtype in (3, 4):
            rr = O.ref_solve(c["ref_kind"], c["shape"], c["b"], c["opts"], dtype=dtype, A=c.get("A"),
                             csr=c.get("csr_tuple"), geom=c.get("geom"), Ut=c["u_true"])
            out[f"ref{dtype}_U"] = rr.U.astype(np.complex128)
            out[f"ref{dtype}_iters"] = np.array([rr.outer_iters, rr.total_iters])
            out[f"ref{dtype}_relerr"] = np.array([rr.rel_error, rr.rel_chg])
        o20 = dict(c["opts"], maxit=20)   # a fixed count: no stopping decision involved
        for dtype in (3, 4):
            rr = O.ref_solve(c["ref_kind"], c["shape"], c["b"], o20, dtype=dtype, A=c.get("A"),
                             csr=c.get("csr_tuple"), geom=c.get("geom"), Ut=c["u_true"])
            out[f"ref{dtype}_U_it20"] = rr.U.astype(np.complex128)
    finally:
        os.chdir(cwd)
    out["oracle_U"] = out["ref4_U"]
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, {k: v.shape for k, v in out.items()})


def main():
    O.build(reference=True)
    cwd = os.getcwd()
    tmp = tempfile.mkdtemp()
    only = set(sys.argv[1:])
    for name in COMPLEX_CASES:
        if not only or name in only:
            complex_case(name, tmp)
    for name in CASES:
        if only and name not in only:
            continue
        c = build_case(name)
        out = {"b_sum": checksum(c["b"])}
        if "A" in c:
            out["A_sum"] = checksum(c["A"])
        # FP64 oracle restatement
        r = O.solve(c["oracle_op"], c["b"].astype(np.float64), c["shape"], c["opts"], Ut=c["u_true"])
        out["oracle_U"] = r.U.astype(np.float64)
        out["oracle_iters"] = np.array([r.outer_iters, r.total_iters])
        # the reference itself (float data with float / double options, double)
        if c["ref_kind"] is not None:
            os.chdir(tmp)
            try:
                for dtype in (0, 1, 2):
                    rr = O.ref_solve(c["ref_kind"], c["shape"], c["b"], c["opts"], dtype=dtype, A=c.get("A"),
                                     csr=c.get("csr_tuple"), geom=c.get("geom"), Ut=c["u_true"])
                    out[f"ref{dtype}_U"] = rr.U.astype(np.float64)
                    out[f"ref{dtype}_iters"] = np.array([rr.outer_iters, rr.total_iters])
                    out[f"ref{dtype}_relerr"] = np.array([rr.rel_error, rr.rel_chg])
            finally:
                os.chdir(cwd)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
