"""Small seeded parity cases shared by make_golden.py and the tests.

Each case gives the problem inputs (regenerated from seeds), the oracle
operator, how the reference runs it (ref_kind: 'dense', 'csr', 'ray3d' or None
when the reference cannot run it: isotropic TV) and how the C ABI sees it.
2D ray cases run the reference on the CSR twin of the rays, because the
reference's 2D ray projector is commented out (2d/mat_mult.h:111-193).
"""
import math

import numpy as np

import oracle as O
from tval3g import workloads as W

CASES = [
    "dense2d_s32_it20", "dense2d_s32_conv", "dense2d_layers", "ring2d_s64_it20", "ring2d_s64_conv",
    "ring2d_s64_iso", "ring2d_s64_nonneg", "ring2d_s64_skip", "hemi3d_s16_it20", "hemi3d_s16_conv",
    "csr3d_s16", "dense3d_s8",
]


def _csr_tuple(A):
    return (A["m"], A["n"], A["rowptr"], A["colind"], A["val"])


def build_case(name):
    c = {"name": name}
    if name.startswith("dense2d_s32"):
        it = name.endswith("it20")
        w = W.dense2d(seed=0, side=32, sampling=0.3, tv_norm=0, maxit=20 if it else 300, tol=1e-4)
        c.update(shape=w["shape"], A=w["A"], b=w["b"], u_true=w["u_true"], opts=w["opts"], ref_kind="dense",
                 api="dense", layers=1)
        c["oracle_op"] = O.Op.dense(w["A"].astype(np.float64))
    elif name == "dense2d_layers":
        rng = np.random.default_rng(5)
        side, layers = 16, 3
        n = side * side
        m = int(0.3 * n)
        A = (rng.standard_normal((m, n)) / math.sqrt(m)).astype(np.float32)
        us = [W.ellipse_phantom(side, side, rng, 3, 0.0, lambda r: r.uniform(0.2, 1.0), (2, 6)) for _ in range(layers)]
        b = np.concatenate([W.add_noise(A.astype(np.float64) @ u.ravel(), 0.01, rng) for u in us]).astype(np.float32)
        u_true = np.concatenate([u.ravel() for u in us]).reshape(side * layers, side)
        c.update(shape=(side * layers, side), A=A, b=b, u_true=u_true, ref_kind="dense", api="dense", layers=layers,
                 opts=W.options(2 ** 8, 2 ** 5, 1e-4, 30, tv_norm=0))
        c["oracle_op"] = O.Op.dense(A.astype(np.float64), layers=layers)
    elif name.startswith("ring2d_s64"):
        kind = name.split("_")[-1]
        maxit = {"it20": 20, "conv": 300}.get(kind, 40)
        extra = {}
        if kind == "skip":
            extra = dict(skipMulRatio=0.5, numInitIterations=3, maxRelativeChange=0.05)
        w = W.ring2d(seed=1, side=64, T=64, tv_norm=1 if kind == "iso" else 0, maxit=maxit, tol=1e-5)
        w["opts"].update(extra)
        # nonnegativity keeps this problem in its stable regime (FP32 and FP64
        # trajectories agree), which the iso and skip cases need to be compared
        # by their final U; without it the first iterations are chaotic
        if kind in ("nonneg", "iso", "skip"):
            w["opts"]["nonneg"] = 1
        c.update(shape=w["shape"], b=w["b"], u_true=w["u_true"], opts=w["opts"], geom=w["geom"], csr=w["csr"],
                 csr_tuple=_csr_tuple(w["csr"]), ref_kind=None if kind == "iso" else "csr",
                 api="csr" if kind == "skip" else "ray2d", layers=1)
        c["oracle_op"] = O.Op.ray2d(w["geom"], 64 * 64)
    elif name.startswith("hemi3d_s16") or name == "csr3d_s16":
        it = name.endswith("it20") or name == "csr3d_s16"
        w = W.hemi3d(seed=2, side=16, T=64, receivers=16, maxit=20 if it else 200, tol=1e-5, csr=True)
        c.update(shape=w["shape"], b=w["b"], u_true=w["u_true"], opts=w["opts"], geom=w["geom"], csr=w["csr"],
                 csr_tuple=_csr_tuple(w["csr"]), layers=1)
        if name == "csr3d_s16":
            c.update(ref_kind="csr", api="csr")
            A = w["csr"]
            c["oracle_op"] = O.Op.csr(A["m"], A["n"], A["rowptr"], A["colind"], A["val"])
        else:
            c.update(ref_kind="ray3d", api="ray3d")
            c["oracle_op"] = O.Op.ray3d(w["geom"])
    elif name == "dense3d_s8":
        rng = np.random.default_rng(7)
        s = 8
        n = s ** 3
        m = int(0.3 * n)
        u = W.ellipsoid_phantom(s, rng, 3, 0.0, lambda r: r.uniform(0.2, 1.0), (1.5, 3.5))
        A = (rng.standard_normal((m, n)) / math.sqrt(m)).astype(np.float32)
        b = W.add_noise(A.astype(np.float64) @ u.ravel(), 0.01, rng).astype(np.float32)
        c.update(shape=(s, s, s), A=A, b=b, u_true=u, ref_kind="dense", api="dense", layers=1,
                 opts=W.options(2 ** 8, 2 ** 5, 1e-4, 40, tv_norm=0))
        c["oracle_op"] = O.Op.dense(A.astype(np.float64))
    else:
        raise KeyError(name)
    return c


def api_problem(c, capi):
    """The C-ABI ProblemSpec of a case."""
    if c["api"] == "dense":
        return capi.dense_problem(c["shape"], c["A"], c.get("layers", 1))
    if c["api"] == "csr":
        A = c["csr"]
        return capi.csr_problem(c["shape"], A["m"], A["n"], A["rowptr"], A["colind"], A["val"], c.get("layers", 1))
    if c["api"] == "ray2d":
        return capi.ray2d_problem(c["shape"], c["geom"])
    return capi.ray3d_problem(c["shape"], c["geom"])
