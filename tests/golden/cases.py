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
    "csr3d_s16", "dense3d_s8", "hemi3d_mp2_s16", "csr2d_layers",
]
# complex data (the reference's complex<float> / complex<double> overloads):
# the FP64 anchor is the reference's own complex<double> build
COMPLEX_CASES = ["cdense2d_s32", "ccsr2d_s32", "cring2d_s64", "cdense3d_s8", "chemi3d_s16", "cdense2d_layers",
                 "ccsr2d_layers"]


def _complex_phantom(side, rng):
    ur = W.ellipse_phantom(side, side, rng, 4, 0.0, lambda r: r.uniform(0.2, 1.0), (side / 10, side / 3))
    ui = W.ellipse_phantom(side, side, rng, 3, 0.0, lambda r: r.uniform(-0.6, 0.6), (side / 10, side / 3))
    return ur + 1j * ui


def _complex_noise(y, rel, rng):
    e = rng.standard_normal(y.shape) + 1j * rng.standard_normal(y.shape)
    return y + e * (rel * np.linalg.norm(y) / np.linalg.norm(e))


def _csr_apply(csr, x):
    m, rowptr, colind, val = csr["m"], csr["rowptr"], csr["colind"], csr["val"]
    rows = np.repeat(np.arange(m), np.diff(rowptr))
    y = np.zeros(m, np.complex128)
    np.add.at(y, rows, val.astype(np.complex128) * x[colind])
    return y


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
        w = W.ring2d(seed=1, side=64, T=64, tv_norm=1 if kind == "iso" else 0, maxit=maxit, tol=1e-5,
                     normalize=True)
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
        w = W.hemi3d(seed=2, side=16, T=64, receivers=16, maxit=20 if it else 200, tol=1e-5, csr=True,
                     normalize=True)
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
    elif name == "hemi3d_mp2_s16":
        # two measurement positions (numMPs = 2, 3d/mat_mult.h:183): the same
        # hemisphere, and the hemisphere turned a quarter about z
        w = W.hemi3d(seed=2, side=16, T=64, receivers=16, maxit=20, tol=1e-5, csr=True, normalize=True)
        g = dict(w["geom"])
        s_ = 15
        for a, b_ in (("xe", "ye"), ("xr", "yr")):
            x, y = g[a], g[b_]
            g[a] = np.concatenate([x, s_ - y]).astype(np.int32)
            g[b_] = np.concatenate([y, x]).astype(np.int32)
        for a in ("ze", "zr"):
            g[a] = np.concatenate([g[a], g[a]]).astype(np.int32)
        g["numMPs"] = 2
        rng = np.random.default_rng(21)
        A = W.ray3d_csr(g)
        b = W.add_noise(W.csr_matvec(A, w["u_true"].ravel()), 0.005, rng).astype(np.float32)
        c.update(shape=w["shape"], b=b, u_true=w["u_true"], opts=w["opts"], geom=g, csr=A, csr_tuple=_csr_tuple(A),
                 layers=1, ref_kind="ray3d", api="ray3d")
        c["oracle_op"] = O.Op.ray3d(g)
    elif name == "csr2d_layers":
        # 2D sparse operator with three layers (the reference's cscmm path,
        # 2d/mat_mult.h:68-90)
        rng = np.random.default_rng(6)
        side, layers, k = 16, 3, 24
        n = side * side
        m = int(0.4 * n)
        colind = np.concatenate([np.sort(rng.choice(n, k, replace=False)) for _ in range(m)]).astype(np.int32)
        rowptr = (np.arange(m + 1) * k).astype(np.int32)
        val = (rng.standard_normal(m * k) / math.sqrt(k)).astype(np.float32)
        csr = {"m": m, "n": n, "rowptr": rowptr, "colind": colind, "val": val}
        us = [W.ellipse_phantom(side, side, rng, 3, 0.0, lambda r: r.uniform(0.2, 1.0), (2, 6)) for _ in range(layers)]
        b = np.concatenate([W.add_noise(W.csr_matvec(csr, u.ravel()), 0.01, rng) for u in us]).astype(np.float32)
        u_true = np.concatenate([u.ravel() for u in us]).reshape(side * layers, side)
        c.update(shape=(side * layers, side), b=b, u_true=u_true, csr=csr, csr_tuple=_csr_tuple(csr),
                 ref_kind="csr", api="csr", layers=layers, opts=W.options(2 ** 8, 2 ** 5, 1e-4, 30, tv_norm=0))
        c["oracle_op"] = O.Op.csr(m, n, rowptr, colind, val, layers=layers)
    elif name == "cdense2d_s32":
        rng = np.random.default_rng(11)
        side = 32
        n = side * side
        m = int(0.4 * n)
        u = _complex_phantom(side, rng)
        A = ((rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))) / math.sqrt(2 * m)).astype(np.complex64)
        b = _complex_noise(A.astype(np.complex128) @ u.ravel(), 0.01, rng).astype(np.complex64)
        c.update(shape=(side, side), A=A, b=b, u_true=u.astype(np.complex64), ref_kind="dense", api="dense",
                 layers=1, opts=W.options(2 ** 8, 2 ** 5, 1e-4, 300, tv_norm=0))
    elif name == "ccsr2d_s32":
        rng = np.random.default_rng(12)
        side = 32
        n = side * side
        m = int(0.5 * n)
        k = 40   # entries per row
        colind = np.concatenate([np.sort(rng.choice(n, k, replace=False)) for _ in range(m)]).astype(np.int32)
        rowptr = (np.arange(m + 1) * k).astype(np.int32)
        val = ((rng.standard_normal(m * k) + 1j * rng.standard_normal(m * k)) / math.sqrt(2 * k)).astype(np.complex64)
        csr = {"m": m, "n": n, "rowptr": rowptr, "colind": colind, "val": val}
        u = _complex_phantom(side, rng)
        b = _complex_noise(_csr_apply(csr, u.ravel()), 0.01, rng).astype(np.complex64)
        c.update(shape=(side, side), b=b, u_true=u.astype(np.complex64), csr=csr, csr_tuple=_csr_tuple(csr),
                 ref_kind="csr", api="csr", layers=1, opts=W.options(2 ** 8, 2 ** 5, 1e-4, 300, tv_norm=0))
    elif name in ("cdense2d_layers", "ccsr2d_layers"):
        # complex data with three stacked layers (2d/tval3_cpu_2d.cpp:894)
        rng = np.random.default_rng(16)
        side, layers = 16, 3
        n = side * side
        m = int(0.4 * n)
        us = [_complex_phantom(side, rng) for _ in range(layers)]
        u_true = np.concatenate([u.ravel() for u in us]).reshape(side * layers, side).astype(np.complex64)
        if name == "cdense2d_layers":
            A = ((rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))) / math.sqrt(2 * m)).astype(np.complex64)
            ys = [A.astype(np.complex128) @ u.ravel() for u in us]
            c.update(A=A, ref_kind="dense", api="dense")
        else:
            k = 32
            colind = np.concatenate([np.sort(rng.choice(n, k, replace=False)) for _ in range(m)]).astype(np.int32)
            rowptr = (np.arange(m + 1) * k).astype(np.int32)
            val = ((rng.standard_normal(m * k) + 1j * rng.standard_normal(m * k)) / math.sqrt(2 * k)).astype(np.complex64)
            csr = {"m": m, "n": n, "rowptr": rowptr, "colind": colind, "val": val}
            ys = [_csr_apply(csr, u.ravel()) for u in us]
            c.update(csr=csr, csr_tuple=_csr_tuple(csr), ref_kind="csr", api="csr")
        b = np.concatenate([_complex_noise(y, 0.01, rng) for y in ys]).astype(np.complex64)
        c.update(shape=(side * layers, side), b=b, u_true=u_true, layers=layers,
                 opts=W.options(2 ** 8, 2 ** 5, 1e-4, 300, tv_norm=0))
    elif name == "cdense3d_s8":
        rng = np.random.default_rng(14)
        sd = 8
        n = sd ** 3
        m = int(0.4 * n)
        ur = W.ellipsoid_phantom(sd, rng, 3, 0.0, lambda r: r.uniform(0.2, 1.0), (1.5, 3.5))
        ui = W.ellipsoid_phantom(sd, rng, 2, 0.0, lambda r: r.uniform(-0.6, 0.6), (1.5, 3.5))
        u = ur + 1j * ui
        A = ((rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))) / math.sqrt(2 * m)).astype(np.complex64)
        b = _complex_noise(A.astype(np.complex128) @ u.ravel(), 0.01, rng).astype(np.complex64)
        # 100 iterations: beyond them the problem is chaotic (two FP64 solves
        # with different summation orders part by 1e-2 at 150)
        c.update(shape=(sd, sd, sd), A=A, b=b, u_true=u.astype(np.complex64), ref_kind="dense", api="dense",
                 layers=1, opts=W.options(2 ** 8, 2 ** 5, 1e-4, 100, tv_norm=0))
    elif name == "chemi3d_s16":
        # complex data on the 3D hemisphere geometry (the reference runs its
        # own 3D projector on complex vectors)
        # 40 iterations: the problem is chaotic beyond them (two FP64 solves
        # with different summation orders part by 1e-4 at 60)
        w = W.hemi3d(seed=15, side=16, T=64, receivers=16, maxit=40, tol=1e-5, csr=True, normalize=True)
        rng = np.random.default_rng(15)
        u = w["u_true"] * np.exp(1j * np.linspace(0, 1.5, w["u_true"].size)).reshape(w["u_true"].shape)
        csr = dict(w["csr"])
        csr["val"] = csr["val"].astype(np.complex64)
        b = _complex_noise(_csr_apply(csr, u.ravel()), 0.005, rng).astype(np.complex64)
        c.update(shape=w["shape"], b=b, u_true=u.astype(np.complex64), opts=w["opts"], geom=w["geom"], csr=csr,
                 ref_kind="ray3d", api="ray3d_complex", layers=1)
    elif name == "cring2d_s64":
        w = W.ring2d(seed=13, side=64, T=64, tv_norm=0, maxit=300, tol=1e-5, normalize=True)
        rng = np.random.default_rng(13)
        u = _complex_phantom(64, rng)
        csr = dict(w["csr"])
        csr["val"] = csr["val"].astype(np.complex64)
        b = _complex_noise(_csr_apply(csr, u.ravel()), 0.005, rng).astype(np.complex64)
        c.update(shape=w["shape"], b=b, u_true=u.astype(np.complex64), opts=w["opts"], geom=w["geom"], csr=csr,
                 csr_tuple=_csr_tuple(csr), ref_kind="csr", api="ray2d_complex", layers=1)
    else:
        raise KeyError(name)
    return c


def complex_oracle_op(c):
    """The oracle operator of a complex case: the real form of its complex
    operator over all layers (layer-major, block diagonal)."""
    import scipy.sparse as sp
    L = c.get("layers", 1)
    if "A" in c:
        M = sp.csr_matrix(c["A"].astype(np.complex128))
    else:
        A = c["csr"]
        M = sp.csr_matrix((np.asarray(A["val"]).astype(np.complex128), A["colind"], A["rowptr"]),
                          shape=(A["m"], A["n"]))
    if L > 1:
        M = sp.kron(sp.identity(L), M, format="csr")
    return O.complex_real_form(M)


def api_problem(c, capi):
    """The C-ABI ProblemSpec of a case."""
    if c["api"] == "dense":
        return capi.dense_problem(c["shape"], c["A"], c.get("layers", 1))
    if c["api"] == "csr":
        A = c["csr"]
        return capi.csr_problem(c["shape"], A["m"], A["n"], A["rowptr"], A["colind"], A["val"], c.get("layers", 1))
    if c["api"] == "ray2d":
        return capi.ray2d_problem(c["shape"], c["geom"])
    if c["api"] == "ray2d_complex":
        return capi.ray2d_problem(c["shape"], c["geom"], complex_data=True)
    if c["api"] == "ray3d_complex":
        return capi.ray3d_problem(c["shape"], c["geom"], complex_data=True)
    return capi.ray3d_problem(c["shape"], c["geom"])
