"""TVAL3 oracle bindings — test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product path never does.  It wraps

* ``_build/liboracle.so`` — the FP64 C restatement (tval3_oracle.c) of the
  reference solver (modk/tval3-cpu 2d/tval3_cpu_2d.cpp, 3d/tval3_cpu_3d.cpp),
  including the 2D Bresenham projector that is commented out in the reference
  (2d/mat_mult.h:109-194) and isotropic TV, which the reference lacks;
* ``_ref/libref_tval3_{2d,3d}.so`` — the reference's own sources compiled
  unchanged against shim headers (oracle/Makefile), called through their C++
  overloads ``tval3_cpu_2d`` / ``tval3_cpu_3d``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = {}


def build(reference: bool = False) -> None:
    """Compile the restatement (and, when asked and the reference sources are
    present, the reference itself) with oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", HERE, "restate"], check=True)
    if reference:   # the Makefile builds nothing when the sources are absent
        subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def ref_available(dims: int = 2) -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", f"libref_tval3_{dims}d.so"))


class OrcOpts(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("mu", "beta", "mu0", "beta0", "tol", "tol_inn", "c", "gamma",
                                          "gam", "rate_gam", "rate_cnt", "skipMulRatio",
                                          "maxRelativeChange")] + \
               [(k, C.c_int) for k in ("maxit", "maxcnt", "nonneg", "isreal", "numInitIterations",
                                       "tv_norm", "cplx")] + [("noise", C.c_double), ("noise_seed", C.c_ulonglong)]


class RefOpts(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("mu", "beta", "mu0", "beta0", "tol", "tol_inn", "c", "gamma",
                                          "gam", "rate_gam", "rate_cnt", "skipMulRatio",
                                          "maxRelativeChange")] + \
               [(k, C.c_int) for k in ("maxit", "maxcnt", "nonneg", "isreal", "numInitIterations")]


class Info(C.Structure):
    _fields_ = [("secs", C.c_double), ("rel_chg", C.c_double), ("rel_error", C.c_double),
                ("outer_iters", C.c_int), ("total_iters", C.c_int)]


class Replay(C.Structure):
    _fields_ = [("count", C.c_int), ("backtracks", C.POINTER(C.c_int)), ("skipped", C.POINTER(C.c_int)),
                ("inner_end", C.POINTER(C.c_int))]


class Iter(C.Structure):
    _fields_ = [("tau", C.c_double), ("f", C.c_double), ("relchg", C.c_double), ("backtracks", C.c_int),
                ("skipped", C.c_int), ("inner_end", C.c_int), ("pad", C.c_int)]


def _fill(struct, opts: dict):
    s = struct()
    for name, _ in struct._fields_:
        if name in opts:
            setattr(s, name, opts[name])
    return s


def _p(a, ct=C.c_double):
    return a.ctypes.data_as(C.POINTER(ct)) if a is not None else None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "_build", "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp, ip, dp, i, d = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int, C.c_double
        L.orc_op_dense.restype = vp
        L.orc_op_dense.argtypes = [i, i, i, dp]
        L.orc_op_csr.restype = vp
        L.orc_op_csr.argtypes = [i, i, i, i, ip, ip, dp]
        L.orc_op_ray2d.restype = vp
        L.orc_op_ray2d.argtypes = [i, i, ip, ip, ip, ip, ip, i, d, i]
        L.orc_op_ray3d.restype = vp
        L.orc_op_ray3d.argtypes = [i, i, i, i, ip, ip, ip, ip, ip, ip, ip, i, i, i, d]
        L.orc_op_free.argtypes = [vp]
        L.orc_op_rows.argtypes = [vp]
        L.orc_op_cols.argtypes = [vp]
        L.orc_apply.argtypes = [vp, i, dp, dp]
        L.orc_ray_lists.argtypes = [vp, ip, C.POINTER(C.c_long), ip, C.POINTER(C.c_long)]
        L.orc_D.argtypes = [i, i, i, i, dp, dp, dp, dp]
        L.orc_Dt.argtypes = [i, i, i, i, dp, dp, dp, dp]
        L.orc_shrink.restype = d
        L.orc_shrink.argtypes = [i, i, i, d] + [dp] * 9
        L.orc_solve.argtypes = [i, i, i, i, vp, dp, i, C.POINTER(OrcOpts), dp, dp, C.POINTER(Info),
                                C.POINTER(Iter)]
        L.orc_solve_replay.argtypes = [i, i, i, i, vp, dp, i, C.POINTER(OrcOpts), dp, dp, C.POINTER(Info),
                                       C.POINTER(Iter), C.POINTER(Replay)]
        _LIB = L
    return _LIB


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Op:
    """An oracle operator (dense, CSR, 2D rays or 3D rays)."""

    def __init__(self, handle, rows, cols):
        self.h, self.rows, self.cols = handle, rows, cols

    def __del__(self):
        if getattr(self, "h", None) and _LIB is not None:
            _LIB.orc_op_free(self.h)
            self.h = None

    @staticmethod
    def dense(A, layers=1):
        A = _f64(A)
        h = lib().orc_op_dense(A.shape[0], A.shape[1], layers, _p(A))
        return Op(h, A.shape[0] * layers, A.shape[1] * layers)

    @staticmethod
    def csr(m, n, rowptr, colind, val, layers=1):
        rowptr, colind, val = _i32(rowptr), _i32(colind), _f64(val)
        h = lib().orc_op_csr(m, n, layers, len(colind), _p(rowptr, C.c_int), _p(colind, C.c_int), _p(val))
        return Op(h, m * layers, n * layers)

    @staticmethod
    def ray2d(g, n_pixels):
        a = [_i32(g[k]) for k in ("use_path", "xe", "ye", "xr", "yr")]
        E, R = len(a[1]), len(a[3])
        h = lib().orc_op_ray2d(E, R, *[_p(x, C.c_int) for x in a], int(g["ld"]), float(g["scale"]),
                               int(n_pixels))
        return Op(h, E * R, n_pixels)

    @staticmethod
    def ray3d(g):
        a = [_i32(g[k]) for k in ("use_path", "xe", "ye", "ze", "xr", "yr", "zr")]
        h = lib().orc_op_ray3d(int(g["numMPs"]), int(g["numPaths"]), int(g["E"]), int(g["R"]),
                               *[_p(x, C.c_int) for x in a], int(g["rv_x"]), int(g["rv_y"]),
                               int(g["rv_z"]), float(g["scale"]))
        return Op(h, int(g["numPaths"]) * int(g["numMPs"]), int(g["rv_x"]) * int(g["rv_y"]) * int(g["rv_z"]))

    def apply(self, x, trans=False):
        x = _f64(x)
        y = np.zeros(self.cols if trans else self.rows)
        lib().orc_apply(self.h, int(trans), _p(x), _p(y))
        return y

    def ray_lists(self):
        """(ray_index[k], offsets[k..k+1], pixels) of every traced ray."""
        L = lib()
        tot = C.c_long(0)
        cnt = L.orc_ray_lists(self.h, None, None, None, C.byref(tot))
        ray = np.zeros(cnt, np.int32)
        off = np.zeros(cnt + 1, np.int64)
        pix = np.zeros(max(tot.value, 1), np.int32)
        L.orc_ray_lists(self.h, _p(ray, C.c_int), off.ctypes.data_as(C.POINTER(C.c_long)), _p(pix, C.c_int),
                        C.byref(tot))
        return ray, off, pix[:tot.value]


def D(U):
    """Periodic forward differences of a (dim_y, dim_x) or (dim_z, dim_y, dim_x) array."""
    U = _f64(U)
    dims = U.ndim
    shp = U.shape if dims == 3 else (1,) + U.shape
    r, p, q = shp
    out = [np.zeros(U.size) for _ in range(3)]
    lib().orc_D(dims, p, q, r, _p(U), *[_p(o) for o in out])
    return out[:dims]


def Dt(X, Y, Z=None, shape=None):
    dims = 3 if Z is not None else 2
    shp = shape if dims == 3 else (1,) + tuple(shape)
    r, p, q = shp
    X, Y = _f64(X), _f64(Y)
    Z = _f64(Z) if Z is not None else np.zeros(X.size)
    res = np.zeros(X.size)
    lib().orc_Dt(dims, p, q, r, _p(X), _p(Y), _p(Z), _p(res))
    return res


def shrink(comps, sigmas, beta, tv_norm):
    dims = len(comps)
    n = comps[0].size
    comps = [_f64(c) for c in comps] + [np.zeros(n)] * (3 - dims)
    sigmas = [_f64(s) for s in sigmas] + [np.zeros(n)] * (3 - dims)
    W = [np.zeros(n) for _ in range(3)]
    lam1 = lib().orc_shrink(dims, n, tv_norm, beta, *[_p(c) for c in comps], *[_p(s) for s in sigmas],
                            *[_p(w) for w in W])
    return W[:dims], lam1


@dataclass
class Result:
    U: np.ndarray
    secs: float
    outer_iters: int
    total_iters: int
    rel_chg: float
    rel_error: float
    iters: list | None = None


def replay_from_trace(trace):
    """Decisions of a recorded solve, from its per-iteration trace rows
    (tau, f, relchg, backtracks, skipped, relerr_ut, step, outer), as the
    tval3g plan trace gives them: backtracks, skipped and whether the inner
    loop ended after the iteration (the multipliers were updated, or it was
    the last iteration)."""
    tr = np.asarray(trace, np.float64)
    k = len(tr)
    inner_end = (tr[:, 7] != 0).astype(np.int32)
    inner_end[k - 1] = 1 if tr[k - 1, 7] != 0 else 0
    return {"count": k, "backtracks": tr[:, 3].astype(np.int32), "skipped": tr[:, 4].astype(np.int32),
            "inner_end": inner_end}


def complex_real_form(M):
    """The real form [[Re M, -Im M], [Im M, Re M]] of a complex matrix (dense
    array or scipy sparse) as an oracle CSR operator on planar vectors (real
    plane, imaginary plane); its transpose is the real form of M^H."""
    import scipy.sparse as sp
    M = sp.csr_matrix(M)
    R = sp.bmat([[M.real, -M.imag], [M.imag, M.real]], format="csr")
    R.sort_indices()
    return Op.csr(R.shape[0], R.shape[1], R.indptr, R.indices, R.data)


def solve_complex(op: Op, b, shape, opts: dict, Ut=None, record=False, replay=None) -> Result:
    """FP64 oracle solve of complex data (the reference's complex<T>
    overloads): op is the real form of the operator (complex_real_form), b
    and Ut complex; the solve runs on planar vectors and U comes back
    complex."""
    b = np.asarray(b).ravel()
    bp = np.concatenate([b.real, b.imag])
    Utp = None
    if Ut is not None:
        Ut = np.asarray(Ut).ravel()
        Utp = np.concatenate([Ut.real, Ut.imag])
    r = solve(op, bp, shape, dict(opts, cplx=1), Ut=Utp, record=record, replay=replay)
    n = int(np.prod(shape))
    U = r.U.ravel()
    r.U = (U[:n] + 1j * U[n:]).reshape(shape)
    return r


def solve(op: Op, b, shape, opts: dict, Ut=None, record=False, replay=None) -> Result:
    """FP64 oracle solve; shape = (dim_y, dim_x) or (dim_z, dim_y, dim_x).

    replay: decisions of another solve (replay_from_trace) to follow instead
    of taking its own Armijo, skip and stopping decisions: the FP64 solution
    at the same iteration count and discrete path."""
    b = _f64(b)
    dims = len(shape)
    if dims == 2:
        dz, dy, dx = 1, shape[0], shape[1]
    else:
        dz, dy, dx = shape
    U = np.zeros(dz * dy * dx * (2 if opts.get("cplx") else 1))
    o = _fill(OrcOpts, opts)
    info = Info()
    its = (Iter * max(int(opts["maxit"]), 1))() if record else None
    Utp = _f64(Ut).ravel() if Ut is not None else None
    if replay is None:
        rc = lib().orc_solve(dims, dy, dx, dz, op.h, _p(b), len(b), C.byref(o), _p(Utp), _p(U), C.byref(info),
                             its)
    else:
        arrs = [np.ascontiguousarray(replay[k], np.int32) for k in ("backtracks", "skipped", "inner_end")]
        rp = Replay(int(replay["count"]), *[_p(a, C.c_int) for a in arrs])
        rc = lib().orc_solve_replay(dims, dy, dx, dz, op.h, _p(b), len(b), C.byref(o), _p(Utp), _p(U),
                                    C.byref(info), its, C.byref(rp))
    if rc != 0:
        raise ValueError(f"oracle solve rejected its arguments ({rc})")
    rec = None
    if record:
        rec = [(its[k].tau, its[k].f, its[k].relchg, its[k].backtracks, its[k].skipped)
               for k in range(info.total_iters)]
        rec_end = [its[k].inner_end for k in range(info.total_iters)]
    res = Result(U if opts.get("cplx") else U.reshape(shape), info.secs, info.outer_iters, info.total_iters,
                 info.rel_chg, info.rel_error, rec)
    if record:
        res.inner_end = rec_end
    return res


# --------------------------------------------------------------------------
# the reference itself (oracle/_ref)
# --------------------------------------------------------------------------
class ReferenceError(Exception):
    """The reference threw tval3_exception; the message is its what()."""


def ref_lib(dims):
    if dims not in _REF:
        path = os.path.join(HERE, "_ref", f"libref_tval3_{dims}d.so")
        if not os.path.exists(path):
            build(reference=True)
        L = C.CDLL(path)
        vp, ip, i, f = C.c_void_p, C.POINTER(C.c_int), C.c_int, C.c_float
        common_tail = [vp, i, C.POINTER(RefOpts), vp, i, i, i, i, C.POINTER(Info), C.c_char_p, i]
        if dims == 2:
            L.ref2d_dense.argtypes = [i, vp, i, i, i, vp, i, i, i] + common_tail
            L.ref2d_csr.argtypes = [i, vp, i, i, i, i, i, i, i, ip, ip, vp, ip, ip, vp] + common_tail
        else:
            L.ref3d_dense.argtypes = [i, vp, i, i, i, i, vp, i, i, i] + common_tail
            L.ref3d_csr.argtypes = [i, vp, i, i, i, i, i, i, i, i, ip, ip, vp, ip, ip, vp] + common_tail
            L.ref3d_ray.argtypes = [i, vp, i, i, i, i, i, i, i, i, ip, ip, ip, ip, ip, ip, ip, i, i, i, f] + \
                common_tail
        _REF[dims] = L
    return _REF[dims]


_DT = {0: np.float32, 1: np.float32, 2: np.float64, 3: np.complex64, 4: np.complex128}
_PROJ = None


def ref_project3d(g, x, trans=False):
    """The reference's own 3D Bresenham projector (3d/mat_mult.h:148-595,
    compiled from its sources into oracle/_ref/libref_proj_3d.so) applied in
    double precision: y = A x (x over voxels) or y = A^T x (x over rays)."""
    global _PROJ
    if _PROJ is None:
        path = os.path.join(HERE, "_ref", "libref_proj_3d.so")
        if not os.path.exists(path):
            build(reference=True)
        L = C.CDLL(path)
        ip, i = C.POINTER(C.c_int), C.c_int
        L.ref3d_project.argtypes = [i, i, i, i, i, ip, ip, ip, ip, ip, ip, ip, i, i, i, C.c_float,
                                    C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _PROJ = L
    a = [_i32(g[k]) for k in ("use_path", "xe", "ye", "ze", "xr", "yr", "zr")]
    nvox = int(g["rv_x"]) * int(g["rv_y"]) * int(g["rv_z"])
    nray = int(g["numMPs"]) * int(g["numPaths"])
    x = _f64(x)
    assert x.size == (nray if trans else nvox)
    y = np.zeros(nvox if trans else nray)
    _PROJ.ref3d_project(int(trans), int(g["numMPs"]), int(g["numPaths"]), int(g["E"]), int(g["R"]),
                        *[_p(v, C.c_int) for v in a], int(g["rv_x"]), int(g["rv_y"]), int(g["rv_z"]),
                        float(g["scale"]), _p(x), _p(y))
    return y


def ref_available_proj3d() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libref_proj_3d.so"))


def _vp(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def ref_solve(kind: str, shape, b, opts: dict, dtype: int = 0, A=None, csr=None, geom=None, Ut=None,
              formats=None, submat_mb=5, vppc=1, ut_len=None) -> Result:
    """Run the reference's own tval3_cpu_2d / tval3_cpu_3d.

    kind: 'dense' (A: m x n), 'csr' (csr=(m, n, rowptr, colind, val)) or 'ray3d'
    (geom dict).  dtype 0 = float/float opts, 1 = float/double opts, 2 = double,
    3 = complex<float>/float opts, 4 = complex<double>/double opts (2D dense
    and CSR, 3D dense, CSR and rays).
    formats = (U, A, Ut) mat_format codes (0 row major, 1 col major); default is
    what the reference requires for the operator kind (2d:700-702,719,739;
    3d:1038-1039,1086-1087,1140-1141).  Raises ReferenceError with the
    reference's message on an argument error.
    """
    dims = len(shape)
    T = _DT[dtype]
    n = int(np.prod(shape))
    U = np.zeros(n, T)
    b = np.ascontiguousarray(b, T)
    Utv = np.ascontiguousarray(Ut, T).ravel() if Ut is not None else None
    utlen = ut_len if ut_len is not None else (Utv.size if Utv is not None else 0)
    ropts = _fill(RefOpts, opts)
    info = Info()
    err = C.create_string_buffer(1024)
    L = ref_lib(dims)
    if dims == 2:
        dy, dx = shape
        default = {"dense": (1, 0, 1), "csr": (1, 0, 1)}[kind]
    else:
        dz, dy, dx = shape
        default = {"dense": (0, 0, 0), "csr": (1, 0, 1), "ray3d": (0, 0, 0)}[kind]
    uf, af, utf = formats if formats is not None else default
    tail = [_vp(b), len(b), C.byref(ropts), _vp(Utv), utlen, utf, submat_mb, vppc, C.byref(info), err, 1024]
    if kind == "dense":
        A = np.ascontiguousarray(A, T)
        if dims == 2:
            rc = L.ref2d_dense(dtype, _vp(U), dy, dx, uf, _vp(A), A.shape[0], A.shape[1], af, *tail)
        else:
            rc = L.ref3d_dense(dtype, _vp(U), dy, dx, dz, uf, _vp(A), A.shape[0], A.shape[1], af, *tail)
    elif kind == "csr":
        m, ncol, rowptr, colind, val = csr
        rowptr, colind = _i32(rowptr), _i32(colind)
        val = np.ascontiguousarray(val, T)
        cptr, cind, cval = csr_to_csc(m, ncol, rowptr, colind, val)
        fmt = af if formats is not None else 2
        args = [len(colind), fmt, _p(rowptr, C.c_int), _p(colind, C.c_int), _vp(val), _p(cptr, C.c_int),
                _p(cind, C.c_int), _vp(cval)]
        if dims == 2:
            rc = L.ref2d_csr(dtype, _vp(U), dy, dx, uf, m, ncol, *args, *tail)
        else:
            rc = L.ref3d_csr(dtype, _vp(U), dy, dx, dz, uf, m, ncol, *args, *tail)
    elif kind == "ray3d":
        g = geom
        a = [_i32(g[k]) for k in ("use_path", "xe", "ye", "ze", "xr", "yr", "zr")]
        rc = L.ref3d_ray(dtype, _vp(U), dy, dx, dz, uf, int(g["numMPs"]), int(g["numPaths"]), int(g["E"]),
                         int(g["R"]), *[_p(x, C.c_int) for x in a], int(g["rv_x"]), int(g["rv_y"]),
                         int(g["rv_z"]), float(g["scale"]), *tail)
    else:
        raise ValueError(kind)
    if rc != 0:
        raise ReferenceError(err.value.decode())
    return Result(U.reshape(shape), info.secs, info.outer_iters, info.total_iters, info.rel_chg,
                  info.rel_error)


def csr_to_csc(m, n, rowptr, colind, val):
    """Stable CSR -> CSC (rows ascending within a column)."""
    rowptr = np.asarray(rowptr, np.int64)
    rows = np.repeat(np.arange(m, dtype=np.int32), np.diff(rowptr))
    order = np.lexsort((rows, np.asarray(colind)))
    cind = rows[order].astype(np.int32)
    cval = np.ascontiguousarray(np.asarray(val)[order])
    cptr = np.zeros(n + 1, np.int32)
    np.add.at(cptr, np.asarray(colind, np.int64) + 1, 1)
    cptr = np.cumsum(cptr).astype(np.int32)
    return cptr, cind, cval
