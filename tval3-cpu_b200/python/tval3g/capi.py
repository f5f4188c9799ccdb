"""ctypes binding of libtval3g.so (include/tval3g.h).

Host-buffer solves take numpy arrays; plans, operators and stencils take
device pointers (torch CUDA tensors are accepted and their data_ptr() used).
There is no fallback: if the shared library is missing or no GPU is present,
the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(os.path.dirname(HERE))
LIB_PATH = os.path.join(PKG, "lib", "libtval3g.so")

OK, ERR_ARGUMENT, ERR_CUDA, ERR_NO_DEVICE, ERR_NONFINITE, ERR_INTERNAL = 0, -1, -2, -3, -4, -5
OP_DENSE, OP_CSR, OP_RAY2D, OP_RAY3D = 0, 1, 2, 3
TV_ANISO, TV_ISO = 0, 1
DEVICE_INPUTS, GRAPH, TRACE, NO_TENSOR, TUNE, RAY_ADJ_ATOMICS, RAY_ADJ_PLAIN = 1, 2, 4, 8, 16, 32, 64

_OPT_D = ("mu", "beta", "mu0", "beta0", "tol", "tol_inn", "c", "gamma", "gam", "rate_gam", "rate_cnt",
          "skipMulRatio", "maxRelativeChange")
_OPT_I = ("maxit", "maxcnt", "nonneg", "isreal", "numInitIterations", "tv_norm")


class Options(C.Structure):
    _fields_ = [(k, C.c_double) for k in _OPT_D] + [(k, C.c_int) for k in _OPT_I]

    @staticmethod
    def from_dict(d):
        o = Options()
        for k in _OPT_D + _OPT_I:
            setattr(o, k, d[k])
        return o


class Info(C.Structure):
    _fields_ = [("secs", C.c_double), ("rel_chg", C.c_double), ("rel_error", C.c_double),
                ("outer_iters", C.c_int), ("total_iters", C.c_int), ("status", C.c_int), ("reserved", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


_IP = C.POINTER(C.c_int)
_FP = C.POINTER(C.c_float)


class Problem(C.Structure):
    _fields_ = [("dims", C.c_int), ("dim_y", C.c_int), ("dim_x", C.c_int), ("dim_z", C.c_int),
                ("op_kind", C.c_int), ("m", C.c_int), ("n_cols", C.c_int), ("layers", C.c_int),
                ("A", _FP), ("nnz", C.c_longlong), ("csr_ptr", _IP), ("csr_ind", _IP), ("csr_val", _FP),
                ("num_emitters", C.c_int), ("num_receivers", C.c_int), ("numMPs", C.c_int), ("numPaths", C.c_int),
                ("use_path", _IP), ("x_emitters", _IP), ("y_emitters", _IP), ("z_emitters", _IP),
                ("x_receivers", _IP), ("y_receivers", _IP), ("z_receivers", _IP), ("ld", C.c_int),
                ("rv_x", C.c_int), ("rv_y", C.c_int), ("rv_z", C.c_int), ("scale_factor", C.c_float),
                ("complex_data", C.c_int)]


class TVAL3Error(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise TVAL3Error(ERR_NO_DEVICE, f"{LIB_PATH} is not built (run make in the package directory)")
        L = C.CDLL(LIB_PATH)
        vp, i, d, ll = C.c_void_p, C.c_int, C.c_double, C.c_longlong
        P, O, I = C.POINTER(Problem), C.POINTER(Options), C.POINTER(Info)
        L.tval3g_last_error.restype = C.c_char_p
        L.tval3g_solve.argtypes = [P, vp, i, O, vp, i, vp, I]
        L.tval3g_solve_f64.argtypes = [P, vp, vp, i, O, vp, i, vp, I]
        L.tval3g_solve_batch.argtypes = [i, P, C.POINTER(vp), O, C.POINTER(vp), C.POINTER(vp), I, i]
        L.tval3g_plan_create.argtypes = [C.POINTER(vp), i, P, O, i]
        L.tval3g_plan_solve.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(vp), I, vp]
        L.tval3g_plan_stats.argtypes = [vp, C.POINTER(ll), C.POINTER(ll)]
        L.tval3g_plan_trace.argtypes = [vp, i, C.POINTER(C.c_double), i, C.POINTER(i)]
        L.tval3g_plan_set_target.argtypes = [vp, d]
        L.tval3g_plan_time_stencils.argtypes = [vp, i, C.POINTER(d)]
        L.tval3g_plan_destroy.argtypes = [vp]
        L.tval3g_trim_memory.argtypes = [ll]
        L.tval3g_tune_stats.argtypes = [C.POINTER(ll), C.POINTER(ll)]
        L.tval3g_op_launch_shape.argtypes = [vp, C.POINTER(i), C.POINTER(i), C.POINTER(i)]
        L.tval3g_op_create.argtypes = [C.POINTER(vp), P, i]
        L.tval3g_op_shape.argtypes = [vp, C.POINTER(ll), C.POINTER(ll), C.POINTER(ll)]
        L.tval3g_op_apply.argtypes = [vp, i, vp, vp, vp]
        L.tval3g_op_apply_n.argtypes = [vp, i, vp, vp, i, vp]
        L.tval3g_op_ray_csr.argtypes = [vp, C.POINTER(ll), _IP]
        L.tval3g_op_adjoint_index_bytes.argtypes = [vp, C.POINTER(ll)]
        L.tval3g_op_destroy.argtypes = [vp]
        L.tval3g_D.argtypes = [i, i, i, i, vp, vp, vp, vp, vp]
        L.tval3g_Dt.argtypes = [i, i, i, i, vp, vp, vp, vp, vp]
        L.tval3g_shrink.argtypes = [i, ll, i, d, vp, vp, vp, vp, vp, vp, vp, vp, vp, C.POINTER(d), vp]
        L.tval3g_unrolled_create.argtypes = [C.POINTER(vp), P, i, O, i, i]
        L.tval3g_unrolled_forward.argtypes = [vp, C.POINTER(vp), C.POINTER(d), C.POINTER(d), C.POINTER(vp), vp]
        L.tval3g_unrolled_backward.argtypes = [vp, C.POINTER(vp), C.POINTER(vp), C.POINTER(d), C.POINTER(d), vp]
        L.tval3g_unrolled_decisions.argtypes = [vp, i, C.POINTER(d), C.POINTER(i), C.POINTER(d)]
        L.tval3g_unrolled_destroy.argtypes = [vp]
        u64 = C.c_ulonglong
        L.tval3g_gaussian.argtypes = [u64, u64, ll, C.c_float, vp, vp]
        L.tval3g_gaussian_host.argtypes = [u64, u64, ll, C.c_float, vp]
        _LIB = L
    return _LIB


def _check(rc):
    if rc != OK:
        raise TVAL3Error(rc, lib().tval3g_last_error().decode())


def gaussian(d_out, seed, scale=1.0, offset=0, stream=None):
    """Fill the device tensor d_out (float32, contiguous) with the seeded
    Gaussian stream scale * z(seed, offset + i) (tval3g_gaussian)."""
    _check(lib().tval3g_gaussian(int(seed), int(offset), int(d_out.numel()), float(scale), d_out.data_ptr(),
                                 _dptr(stream)))


def gaussian_host(count, seed, scale=1.0, offset=0):
    """The same stream computed on the host (tval3g_gaussian_host)."""
    out = np.empty(int(count), np.float32)
    _check(lib().tval3g_gaussian_host(int(seed), int(offset), int(count), float(scale), out.ctypes.data))
    return out


def trim_memory(keep_bytes=0):
    """Return the library pool's cached device memory beyond keep_bytes."""
    _check(lib().tval3g_trim_memory(int(keep_bytes)))


def tune_stats():
    """(operators timed, choices taken from the cache) of the autotuner in
    this process (TVAL3G_TUNE)."""
    m, c = C.c_longlong(), C.c_longlong()
    _check(lib().tval3g_tune_stats(C.byref(m), C.byref(c)))
    return m.value, c.value


EXPORTS = ("tval3g_last_error", "tval3g_version", "tval3g_solve", "tval3g_solve_f64", "tval3g_solve_batch",
           "tval3g_plan_create",
           "tval3g_plan_solve", "tval3g_plan_stats", "tval3g_plan_trace", "tval3g_plan_set_target",
           "tval3g_plan_time_stencils",
           "tval3g_plan_destroy", "tval3g_trim_memory", "tval3g_tune_stats", "tval3g_op_launch_shape",
           "tval3g_op_create", "tval3g_op_shape",
           "tval3g_op_apply", "tval3g_op_apply_n", "tval3g_op_ray_csr", "tval3g_op_adjoint_index_bytes",
           "tval3g_op_destroy", "tval3g_D", "tval3g_Dt",
           "tval3g_shrink", "tval3g_unrolled_create", "tval3g_unrolled_forward", "tval3g_unrolled_backward",
           "tval3g_unrolled_decisions", "tval3g_unrolled_destroy")


# --------------------------------------------------------------------------
# problems (keep the numpy arrays alive with the struct)
# --------------------------------------------------------------------------
class ProblemSpec:
    """A Problem struct plus the host arrays it points to."""

    def __init__(self, shape, kind, keep=None, **fields):
        self.keep = keep or []
        p = Problem()
        dims = len(shape)
        p.dims = dims
        if dims == 2:
            p.dim_y, p.dim_x, p.dim_z = shape[0], shape[1], 1
        else:
            p.dim_z, p.dim_y, p.dim_x = shape
        p.op_kind = kind
        p.layers = 1
        for k, v in fields.items():
            setattr(p, k, v)
        self.p = p
        self.shape = tuple(shape)
        self.n = int(np.prod(shape))

    @property
    def b_len(self):
        p = self.p
        if p.op_kind == OP_RAY2D:
            return p.num_emitters * p.num_receivers
        if p.op_kind == OP_RAY3D:
            return p.numPaths * p.numMPs
        return p.m * (p.layers if p.dims == 2 else 1)


def _arr(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _ptr(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def _values(a):
    """float32 array of a real array, or the interleaved (re, im) float32
    view of a complex one; and whether it is complex"""
    if np.iscomplexobj(a):
        return _arr(a, np.complex64).view(np.float32), 1
    return _arr(a, np.float32), 0


def dense_problem(shape, A, layers=1, device_ptr=None):
    """A: (m, n_cols) float32 or complex64 host array (or device_ptr with A's
    shape, real).  A complex A makes a complex-data problem (b, Ut, U complex)."""
    m, ncols = A.shape
    if device_ptr is not None:
        return ProblemSpec(shape, OP_DENSE, [A], m=m, n_cols=ncols, layers=layers,
                           A=C.cast(C.c_void_p(device_ptr), _FP))
    A, cplx = _values(A)
    return ProblemSpec(shape, OP_DENSE, [A], m=m, n_cols=ncols, layers=layers, A=_ptr(A, C.c_float),
                       complex_data=cplx)


def csr_problem(shape, m, ncols, rowptr, colind, val, layers=1):
    """val: float32 or complex64 (a complex-data problem)."""
    rowptr, colind = _arr(rowptr, np.int32), _arr(colind, np.int32)
    val, cplx = _values(val)
    return ProblemSpec(shape, OP_CSR, [rowptr, colind, val], m=m, n_cols=ncols, layers=layers, nnz=len(colind),
                       csr_ptr=_ptr(rowptr, C.c_int), csr_ind=_ptr(colind, C.c_int), csr_val=_ptr(val, C.c_float),
                       complex_data=cplx)


def ray2d_problem(shape, g, complex_data=False):
    """complex_data: b, Ut and U are complex (the geometry is real)."""
    a = {k: _arr(g[k], np.int32) for k in ("use_path", "xe", "ye", "xr", "yr")}
    return ProblemSpec(shape, OP_RAY2D, list(a.values()), num_emitters=len(a["xe"]), num_receivers=len(a["xr"]),
                       numMPs=1, use_path=_ptr(a["use_path"], C.c_int), x_emitters=_ptr(a["xe"], C.c_int),
                       y_emitters=_ptr(a["ye"], C.c_int), x_receivers=_ptr(a["xr"], C.c_int),
                       y_receivers=_ptr(a["yr"], C.c_int), ld=int(g["ld"]), scale_factor=float(g["scale"]),
                       complex_data=int(bool(complex_data)))


def ray3d_problem(shape, g, complex_data=False):
    """complex_data: b, Ut and U are complex (the geometry is real)."""
    a = {k: _arr(g[k], np.int32) for k in ("use_path", "xe", "ye", "ze", "xr", "yr", "zr")}
    return ProblemSpec(shape, OP_RAY3D, list(a.values()), num_emitters=int(g["E"]), num_receivers=int(g["R"]),
                       numMPs=int(g["numMPs"]), numPaths=int(g["numPaths"]),
                       use_path=_ptr(a["use_path"], C.c_int), x_emitters=_ptr(a["xe"], C.c_int),
                       y_emitters=_ptr(a["ye"], C.c_int), z_emitters=_ptr(a["ze"], C.c_int),
                       x_receivers=_ptr(a["xr"], C.c_int), y_receivers=_ptr(a["yr"], C.c_int),
                       z_receivers=_ptr(a["zr"], C.c_int), rv_x=int(g["rv_x"]), rv_y=int(g["rv_y"]),
                       rv_z=int(g["rv_z"]), scale_factor=float(g["scale"]), complex_data=int(bool(complex_data)))


def problem_from_workload(w, use_csr=False):
    """ProblemSpec of a tval3g.workloads configuration dict."""
    shape = w["shape"]
    if w["kind"] == "dense":
        return dense_problem(shape, w["A"], w.get("layers", 1))
    if use_csr or w["kind"] == "csr":
        A = w["csr"]
        return csr_problem(shape, A["m"], A["n"], A["rowptr"], A["colind"], A["val"], w.get("layers", 1))
    if w["kind"] == "ray2d":
        return ray2d_problem(shape, w["geom"])
    return ray3d_problem(shape, w["geom"])


# --------------------------------------------------------------------------
# calls
# --------------------------------------------------------------------------
def solve(spec: ProblemSpec, b, opts: dict, Ut=None):
    """One solve with host buffers; returns (U as spec.shape, float32 or -
    for a complex-data problem - complex64, info dict)."""
    dt = np.complex64 if spec.p.complex_data else np.float32
    b = _arr(b, dt).ravel()
    U = np.zeros(spec.n, dt)
    Utv = _arr(Ut, dt).ravel() if Ut is not None else None
    info = Info()
    o = Options.from_dict(opts)
    rc = lib().tval3g_solve(C.byref(spec.p), b.ctypes.data, len(b), C.byref(o),
                            Utv.ctypes.data if Utv is not None else None, Utv.size if Utv is not None else 0,
                            U.ctypes.data, C.byref(info))
    _check(rc)
    return U.reshape(spec.shape), info.as_dict()


def solve_f64(spec: ProblemSpec, b, opts: dict, Ut=None, values=None):
    """One solve in double precision (tval3g_solve_f64): the FP64 engine.
    values: the operator's values in double - the dense A (m x n_cols) or the
    CSR values (nnz), float64, or complex128 for a complex-data problem; None
    for ray geometries (the spec's own float arrays A / csr_val are not read).
    Returns (U as spec.shape, float64 or complex128, info dict)."""
    dt = np.complex128 if spec.p.complex_data else np.float64
    b = _arr(b, dt).ravel()
    U = np.zeros(spec.n, dt)
    Utv = _arr(Ut, dt).ravel() if Ut is not None else None
    vals = _arr(values, dt).ravel() if values is not None else None
    info = Info()
    o = Options.from_dict(opts)
    rc = lib().tval3g_solve_f64(C.byref(spec.p), vals.ctypes.data if vals is not None else None, b.ctypes.data,
                                len(b), C.byref(o), Utv.ctypes.data if Utv is not None else None,
                                Utv.size if Utv is not None else 0, U.ctypes.data, C.byref(info))
    _check(rc)
    return U.reshape(spec.shape), info.as_dict()


def solve_batch(specs, bs, opts_list, Uts=None, graph=True, tune=False):
    n = len(specs)
    probs = (Problem * n)(*[s.p for s in specs])
    opts = (Options * n)(*[Options.from_dict(o) for o in opts_list])
    dts = [np.complex64 if s.p.complex_data else np.float32 for s in specs]
    barr = [_arr(b, dt).ravel() for b, dt in zip(bs, dts)]
    uarr = [np.zeros(s.n, dt) for s, dt in zip(specs, dts)]
    utarr = [(_arr(u, dt).ravel() if u is not None else None) for u, dt in zip(Uts or [None] * n, dts)]
    bp = (C.c_void_p * n)(*[b.ctypes.data for b in barr])
    up = (C.c_void_p * n)(*[u.ctypes.data for u in uarr])
    utp = (C.c_void_p * n)(*[(u.ctypes.data if u is not None else None) for u in utarr])
    infos = (Info * n)()
    _check(lib().tval3g_solve_batch(n, probs, bp, opts, utp, up, infos, (GRAPH if graph else 0) | (TUNE if tune else 0)))
    return [u.reshape(s.shape) for u, s in zip(uarr, specs)], [i.as_dict() for i in infos]


def _dptr(t):
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return int(t)


class Plan:
    """Device-resident solver state for a batch of problems (graph=True: the
    iteration loop is one CUDA graph with conditional nodes)."""

    def __init__(self, specs, opts_list, graph=True, device_inputs=False, trace=False, tensor=True, tune=False,
                 adj_atomics=False, adj_plain=False):
        n = len(specs)
        self.specs = specs
        self.count = n
        self.maxit = [int(o["maxit"]) for o in opts_list]
        probs = (Problem * n)(*[s.p for s in specs])
        opts = (Options * n)(*[Options.from_dict(o) for o in opts_list])
        h = C.c_void_p()
        flags = (GRAPH if graph else 0) | (DEVICE_INPUTS if device_inputs else 0) | (TRACE if trace else 0) | \
            (0 if tensor else NO_TENSOR) | (TUNE if tune else 0) | (RAY_ADJ_ATOMICS if adj_atomics else 0) | \
            (RAY_ADJ_PLAIN if adj_plain else 0)
        _check(lib().tval3g_plan_create(C.byref(h), n, probs, opts, flags))
        self.h = h

    def solve(self, d_b, d_U, d_Ut=None, stream=None):
        n = self.count
        bp = (C.c_void_p * n)(*[_dptr(x) for x in d_b])
        up = (C.c_void_p * n)(*[_dptr(x) for x in d_U])
        utp = (C.c_void_p * n)(*[_dptr(x) for x in d_Ut]) if d_Ut is not None else None
        infos = (Info * n)()
        _check(lib().tval3g_plan_solve(self.h, bp, utp, up, infos, _dptr(stream)))
        return [i.as_dict() for i in infos]

    def time_stencils(self, reps=20):
        """Mean ms per launch of the gradient epilogue, the descent and the
        shrinkage kernels (after a solve; overwrites the plan's state)."""
        ms = (C.c_double * 3)()
        _check(lib().tval3g_plan_time_stencils(self.h, int(reps), ms))
        return {"getg": ms[0], "descend": ms[1], "shrink_grad": ms[2]}

    def stats(self):
        a, b = C.c_longlong(), C.c_longlong()
        _check(lib().tval3g_plan_stats(self.h, C.byref(a), C.byref(b)))
        return {"kernel_launches": a.value, "device_bytes": b.value}

    def trace(self, index=0):
        """Per inner iteration records (tau, f, relchg, backtracks, skipped, relerr_ut, step, outer)."""
        cap = max(self.maxit[index], 1)
        buf = (C.c_double * (8 * cap))()
        cnt = C.c_int()
        _check(lib().tval3g_plan_trace(self.h, index, buf, cap, C.byref(cnt)))
        return np.array(buf[:8 * cnt.value]).reshape(cnt.value, 8)

    def set_target(self, target):
        """Time-to-solution mode: also stop once |U - Ut| <= target |Ut|."""
        _check(lib().tval3g_plan_set_target(self.h, float(target)))

    def close(self):
        if getattr(self, "h", None):
            lib().tval3g_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Operator:
    """A measurement operator on the device: apply(x, trans) with torch tensors."""

    def __init__(self, spec: ProblemSpec, tensor=True, device_inputs=False, tune=False, adj_atomics=False,
                 adj_plain=False):
        h = C.c_void_p()
        flags = (0 if tensor else NO_TENSOR) | (DEVICE_INPUTS if device_inputs else 0) | (TUNE if tune else 0) | \
            (RAY_ADJ_ATOMICS if adj_atomics else 0) | (RAY_ADJ_PLAIN if adj_plain else 0)
        _check(lib().tval3g_op_create(C.byref(h), C.byref(spec.p), flags))
        self.h = h
        r, c, z = C.c_longlong(), C.c_longlong(), C.c_longlong()
        _check(lib().tval3g_op_shape(h, C.byref(r), C.byref(c), C.byref(z)))
        self.rows, self.cols, self.nnz = r.value, c.value, z.value
        ib = C.c_longlong()
        _check(lib().tval3g_op_adjoint_index_bytes(h, C.byref(ib)))
        self.adjoint_index_bytes = ib.value

    def apply(self, x, y, trans=False, stream=None):
        _check(lib().tval3g_op_apply(self.h, int(trans), _dptr(x), _dptr(y), _dptr(stream)))
        return y

    def launch_shape(self):
        """(lanes per ray of the ray forward, 1 + gather width class of the
        forward, of the adjoint); 0 = the built-in choice."""
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        _check(lib().tval3g_op_launch_shape(self.h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def apply_n(self, x, y, reps, trans=False, stream=None):
        """Enqueue `reps` back-to-back applications on `stream`; no wait."""
        _check(lib().tval3g_op_apply_n(self.h, int(trans), _dptr(x), _dptr(y), int(reps), _dptr(stream)))
        return y

    def ray_csr(self):
        rowptr = np.zeros(self.rows + 1, np.int64)
        colind = np.zeros(max(self.nnz, 1), np.int32)
        _check(lib().tval3g_op_ray_csr(self.h, rowptr.ctypes.data_as(C.POINTER(C.c_longlong)),
                                       colind.ctypes.data_as(_IP)))
        return rowptr, colind[:self.nnz]

    def close(self):
        if getattr(self, "h", None):
            lib().tval3g_op_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def D(dims, shape, U, Ux, Uy, Uz=None):
    dz, dy, dx = (1,) + tuple(shape) if dims == 2 else shape
    _check(lib().tval3g_D(dims, dy, dx, dz, _dptr(U), _dptr(Ux), _dptr(Uy), _dptr(Uz), None))


def Dt(dims, shape, X, Y, Z, res):
    dz, dy, dx = (1,) + tuple(shape) if dims == 2 else shape
    _check(lib().tval3g_Dt(dims, dy, dx, dz, _dptr(X), _dptr(Y), _dptr(Z), _dptr(res), None))


def shrink(dims, n, tv_norm, beta, U, S, W):
    lam = C.c_double()
    Uz, Sz, Wz = (U[2], S[2], W[2]) if dims == 3 else (None, None, None)
    _check(lib().tval3g_shrink(dims, n, tv_norm, beta, _dptr(U[0]), _dptr(U[1]), _dptr(Uz), _dptr(S[0]),
                               _dptr(S[1]), _dptr(Sz), _dptr(W[0]), _dptr(W[1]), _dptr(Wz), C.byref(lam), None))
    return lam.value


class Unrolled:
    """Differentiable unrolled solve (tval3g_unrolled_*): `count` instances of
    one 2D problem, K inner iterations with per-iteration (mu_k, beta_k)."""

    def __init__(self, spec: ProblemSpec, count, opts: dict, K, ckpt=10):
        h = C.c_void_p()
        _check(lib().tval3g_unrolled_create(C.byref(h), C.byref(spec.p), int(count), C.byref(Options.from_dict(opts)),
                                            int(K), int(ckpt)))
        self.h, self.count, self.K, self.spec = h, int(count), int(K), spec

    def forward(self, d_b, mu, beta, d_U, stream=None):
        """d_b, d_U: sequences of `count` device tensors; mu, beta: K floats."""
        n = self.count
        mu = np.ascontiguousarray(mu, np.float64)
        beta = np.ascontiguousarray(beta, np.float64)
        bp = (C.c_void_p * n)(*[_dptr(x) for x in d_b])
        up = (C.c_void_p * n)(*[_dptr(x) for x in d_U])
        _check(lib().tval3g_unrolled_forward(self.h, bp, mu.ctypes.data_as(C.POINTER(C.c_double)),
                                             beta.ctypes.data_as(C.POINTER(C.c_double)), up, _dptr(stream)))

    def backward(self, d_gU, d_gb, stream=None):
        """Returns (g_mu, g_beta) as numpy arrays; gb is written to d_gb."""
        n = self.count
        gp = (C.c_void_p * n)(*[_dptr(x) for x in d_gU])
        bp = (C.c_void_p * n)(*[_dptr(x) for x in d_gb])
        gmu, gbeta = np.zeros(self.K), np.zeros(self.K)
        _check(lib().tval3g_unrolled_backward(self.h, gp, bp, gmu.ctypes.data_as(C.POINTER(C.c_double)),
                                              gbeta.ctypes.data_as(C.POINTER(C.c_double)), _dptr(stream)))
        return gmu, gbeta

    def decisions(self, index):
        steps = np.zeros(self.K)
        outer = np.zeros(self.K, np.int32)
        scl = C.c_double()
        _check(lib().tval3g_unrolled_decisions(self.h, int(index), steps.ctypes.data_as(C.POINTER(C.c_double)),
                                               outer.ctypes.data_as(C.POINTER(C.c_int)), C.byref(scl)))
        return steps, outer.astype(bool), scl.value

    def close(self):
        if getattr(self, "h", None):
            lib().tval3g_unrolled_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
