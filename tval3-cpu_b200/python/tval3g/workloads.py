"""Seeded synthetic TVAL3 workloads (phantoms, measurement operators, data).

Everything is drawn from numpy's PCG64 generator with a fixed seed, so a
workload is bit-identical on every machine with this numpy.  The shapes follow
the benchmark configurations of the TVAL3 solve path:

* ``dense2d``   plain 2D problem with a dense Gaussian A (64x64, 30 % sampling);
* ``ring2d``    2D ultrasound-tomography ring: T transducers on the inscribed
                circle, each emitter fires at the T/2 receivers on the opposite
                half; Bresenham projector and its CSR twin;
* ``hemi3d``    3D hemisphere geometry with Fibonacci-spiral transducers and
                seeded-random receiver subsets, 3D Bresenham projector;
* ``batch2d``   a mixed batch of independent 2D problems.

Ray geometries follow the reference's conventions: 2D rays are indexed
uncompacted, ray = emitter*num_receivers + receiver, with use_path marking the
traced ones (modk/tval3-cpu 2d/mat_mult.h:138-142, 2d/tval3_cpu_2d.cpp:748);
3D rays are compacted through 1-based use_path values (3d/mat_mult.h:193-202).

``bresenham_csr_*`` rasterise rays with the closed form of the reference's
error-term recurrence (pixel offset along a minor axis after j steps of the
driving axis = floor((2*j*m_minor + M - 1) / (2*M)), M = driving length); the
test-suite checks it against the sequential recurrence.
"""
from __future__ import annotations

import math

import numpy as np

# --------------------------------------------------------------------------
# options
# --------------------------------------------------------------------------


# --------------------------------------------------------------------------
# counter-based Gaussian streams (the library's tval3g_gaussian, in numpy)
# --------------------------------------------------------------------------
_PH_M0, _PH_M1, _PH_W0, _PH_W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
_M32 = np.uint64(0xFFFFFFFF)


def philox4x32_10(c, key):
    """Philox-4x32-10 (Salmon, Moraes, Dror and Shaw, SC 2011) on arrays of
    counters: c = four uint32 arrays, key = (k0, k1); returns four uint64
    arrays holding the 32-bit output words."""
    c0, c1, c2, c3 = (np.asarray(x, np.uint64) for x in c)
    k0, k1 = np.uint64(key[0]), np.uint64(key[1])
    for _ in range(10):
        p0 = np.uint64(_PH_M0) * c0
        p1 = np.uint64(_PH_M1) * c2
        c0, c1, c2, c3 = (p1 >> np.uint64(32)) ^ c1 ^ k0, p1 & _M32, (p0 >> np.uint64(32)) ^ c3 ^ k1, p0 & _M32
        k0 = (k0 + np.uint64(_PH_W0)) & _M32
        k1 = (k1 + np.uint64(_PH_W1)) & _M32
    return c0, c1, c2, c3


def philox_gaussian(seed, count, scale=1.0, offset=0):
    """float32 array: element i = scale * z(seed, offset + i), the stream of
    tval3g_gaussian (Philox-4x32-10 counter blocks, Box-Muller in FP64)."""
    e = np.arange(offset, offset + count, dtype=np.uint64)
    blocks = np.unique(e >> np.uint64(2))
    j = blocks
    x = philox4x32_10((j & _M32, j >> np.uint64(32), np.zeros_like(j), np.zeros_like(j)),
                      (seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF))
    q = 1.0 / 16777216.0
    z = np.empty((len(j), 4))
    two_pi = 6.283185307179586476925286766559
    for p in range(2):
        u1 = ((x[2 * p] >> np.uint64(8)) + np.uint64(1)).astype(np.float64) * q
        t = (x[2 * p + 1] >> np.uint64(8)).astype(np.float64) * q
        r = np.sqrt(-2.0 * np.log(u1))
        z[:, 2 * p] = r * np.cos(two_pi * t)
        z[:, 2 * p + 1] = r * np.sin(two_pi * t)
    zz = z[(e >> np.uint64(2)) - blocks[0], (e & np.uint64(3)).astype(np.int64)]
    return (zz * np.float64(np.float32(scale))).astype(np.float32)


def options(mu, beta, tol, maxit, tv_norm=1, nonneg=False, tol_inn=1e-3, maxcnt=10, **kw):
    """A full TVAL3 option set (every field set explicitly)."""
    o = dict(mu=float(mu), beta=float(beta), mu0=float(mu), beta0=float(beta), tol=float(tol),
             tol_inn=float(tol_inn), c=1e-5, gamma=0.6, gam=0.9995, rate_gam=0.9, rate_cnt=2.0,
             skipMulRatio=0.0, maxRelativeChange=0.0, maxit=int(maxit), maxcnt=int(maxcnt),
             nonneg=int(bool(nonneg)), isreal=0, numInitIterations=0, tv_norm=int(tv_norm))
    o.update(kw)
    return o


# --------------------------------------------------------------------------
# phantoms
# --------------------------------------------------------------------------


def ellipse_phantom(ny, nx, rng, count, background, values, axes, centre_radius=None):
    """Piecewise-constant image: `count` rotated ellipses painted in order.

    values: callable(rng) -> value; axes: (lo, hi) semi-axis range in pixels.
    centre_radius: if given, centres are drawn inside that radius around the
    image centre, else uniformly in the image.
    """
    img = np.full((ny, nx), background, np.float64)
    yy, xx = np.mgrid[0:ny, 0:nx].astype(np.float64)
    cy0, cx0 = (ny - 1) / 2.0, (nx - 1) / 2.0
    for _ in range(count):
        if centre_radius is None:
            cx, cy = rng.uniform(0, nx), rng.uniform(0, ny)
        else:
            rad = centre_radius * math.sqrt(rng.uniform(0, 1))
            ang = rng.uniform(0, 2 * math.pi)
            cx, cy = cx0 + rad * math.cos(ang), cy0 + rad * math.sin(ang)
        a, b = rng.uniform(*axes), rng.uniform(*axes)
        th = rng.uniform(0, math.pi)
        c, s = math.cos(th), math.sin(th)
        u = (xx - cx) * c + (yy - cy) * s
        v = -(xx - cx) * s + (yy - cy) * c
        img[(u / a) ** 2 + (v / b) ** 2 <= 1.0] = values(rng)
    return img


def ellipsoid_phantom(n, rng, count, background, values, axes):
    """(n, n, n) volume [z, y, x] with `count` random ellipsoids painted in order."""
    vol = np.full((n, n, n), background, np.float64)
    zz, yy, xx = np.mgrid[0:n, 0:n, 0:n].astype(np.float32)
    c0 = (n - 1) / 2.0
    for _ in range(count):
        ctr = c0 + rng.uniform(-n / 4, n / 4, size=3)
        ax = rng.uniform(*axes, size=3)
        # random rotation from a QR of a Gaussian matrix
        q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        d = np.stack([xx - ctr[0], yy - ctr[1], zz - ctr[2]], axis=-1)
        r = d @ q.astype(np.float32)
        inside = ((r / ax.astype(np.float32)) ** 2).sum(-1) <= 1.0
        vol[inside] = values(rng)
    return vol


def add_noise(y, rel, rng):
    """y + Gaussian noise with ||noise|| = rel * ||y||."""
    e = rng.standard_normal(y.shape)
    return y + e * (rel * np.linalg.norm(y) / max(np.linalg.norm(e), 1e-300))


# --------------------------------------------------------------------------
# Bresenham rasterisation (closed form of the reference recurrence)
# --------------------------------------------------------------------------


def _minor(j, mm, M):
    """Minor-axis offset after j driving steps (M > 0)."""
    return (2 * j * mm + M - 1) // (2 * M)


def bresenham_csr_2d(x0, y0, x1, y1, ld):
    """Pixel lists of 2D rays (arrays of endpoints) as (offsets, pixels).

    Restates the reference's recurrence (2d/mat_mult.h:145-181) in closed form:
    x drives when |dx| >= |dy|; both endpoints are included.
    """
    x0, y0, x1, y1 = (np.asarray(a, np.int64) for a in (x0, y0, x1, y1))
    dx, dy = x1 - x0, y1 - y0
    sx, sy = np.where(dx < 0, -1, 1), np.where(dy < 0, -1, 1)
    le, mm = np.abs(dx), np.abs(dy)
    xdrive = le >= mm
    M = np.where(xdrive, le, mm)
    mn = np.where(xdrive, mm, le)
    lengths = M + 1
    off = np.zeros(len(x0) + 1, np.int64)
    np.cumsum(lengths, out=off[1:])
    ray = np.repeat(np.arange(len(x0)), lengths)
    j = np.arange(off[-1], dtype=np.int64) - off[ray]
    Mr = M[ray]
    k = np.where(Mr > 0, (2 * j * mn[ray] + Mr - 1) // (2 * np.maximum(Mr, 1)), 0)
    xd = xdrive[ray]
    x = x0[ray] + sx[ray] * np.where(xd, j, k)
    y = y0[ray] + sy[ray] * np.where(xd, k, j)
    return off, (x + y * ld).astype(np.int32)


def bresenham_csr_3d(p0, p1, rvx, rvy):
    """Voxel lists of 3D rays; p0, p1: (N, 3) integer (x, y, z) endpoints.

    Closed form of 3d/mat_mult.h:241-359: x drives if mx >= my and mx >= mz,
    else y if my >= mx and my >= mz, else z; two independent minor axes.
    """
    p0, p1 = np.asarray(p0, np.int64), np.asarray(p1, np.int64)
    d = p1 - p0
    s = np.where(d < 0, -1, 1)
    a = np.abs(d)
    mx, my, mz = a[:, 0], a[:, 1], a[:, 2]
    drive = np.where((mx >= my) & (mx >= mz), 0, np.where((my >= mx) & (my >= mz), 1, 2))
    M = a[np.arange(len(a)), drive]
    lengths = M + 1
    off = np.zeros(len(a) + 1, np.int64)
    np.cumsum(lengths, out=off[1:])
    ray = np.repeat(np.arange(len(a)), lengths)
    j = np.arange(off[-1], dtype=np.int64) - off[ray]
    Mr = np.maximum(M[ray], 1)
    coord = []
    for ax in range(3):
        minor = (2 * j * a[ray, ax] + Mr - 1) // (2 * Mr)
        step = np.where(drive[ray] == ax, j, minor)
        coord.append(p0[ray, ax] + s[ray, ax] * step)
    lin = coord[0] + coord[1] * rvx + coord[2] * (rvx * rvy)
    return off, lin.astype(np.int32)


# --------------------------------------------------------------------------
# geometries
# --------------------------------------------------------------------------


def ring_geometry(side, T, receivers_per_emitter=None, scale=1.0):
    """T transducers evenly spaced on the circle inscribed in a side x side
    image (integer-rounded); emitter e fires at the receivers_per_emitter
    (default T/2) transducers centred on the opposite point."""
    c = (side - 1) / 2.0
    ang = 2 * math.pi * np.arange(T) / T
    x = np.clip(np.rint(c + c * np.cos(ang)), 0, side - 1).astype(np.int32)
    y = np.clip(np.rint(c + c * np.sin(ang)), 0, side - 1).astype(np.int32)
    R = receivers_per_emitter or T // 2
    use = np.zeros((T, T), np.int32)
    first = T // 2 - R // 2
    for e in range(T):
        use[e, (e + first + np.arange(R)) % T] = 1
    return dict(use_path=use.ravel(), xe=x, ye=y, xr=x.copy(), yr=y.copy(), ld=side, scale=float(scale),
                E=T, R=T)


def ray2d_csr(g, n_pixels):
    """CSR twin of a 2D ray geometry: rows = E*R (uncompacted, untraced rays are
    empty rows), unit weights times scale."""
    E, R = g["E"], g["R"]
    use = np.asarray(g["use_path"]).reshape(E, R)
    e, r = np.nonzero(use)
    off, pix = bresenham_csr_2d(g["xe"][e], g["ye"][e], g["xr"][r], g["yr"][r], g["ld"])
    counts = np.zeros(E * R, np.int64)
    counts[e * R + r] = np.diff(off)
    rowptr = np.zeros(E * R + 1, np.int64)
    np.cumsum(counts, out=rowptr[1:])
    assert pix.max() < n_pixels
    return dict(m=E * R, n=n_pixels, rowptr=rowptr.astype(np.int32), colind=pix,
                val=np.full(len(pix), g["scale"], np.float64))


def hemisphere_geometry(side, T, receivers_per_emitter, radius, rng, scale=1.0):
    """T transducers on a hemisphere (Fibonacci spiral) of `radius` voxels
    centred in a side^3 volume; each emitter fires at a seeded-random subset of
    receivers_per_emitter other transducers.  One measurement position."""
    c = (side - 1) / 2.0
    k = np.arange(T) + 0.5
    zc = k / T                                     # cos(polar) in (0, 1): lower hemisphere
    rr = np.sqrt(1 - zc ** 2)
    phi = k * math.pi * (3 - math.sqrt(5))
    pts = np.stack([c + radius * rr * np.cos(phi), c + radius * rr * np.sin(phi), c - radius * zc], 1)
    pts = np.clip(np.rint(pts), 0, side - 1).astype(np.int32)
    use = np.zeros((T, T), np.int32)
    nxt = 1
    for e in range(T):
        cand = np.delete(np.arange(T), e)
        recv = np.sort(rng.choice(cand, size=receivers_per_emitter, replace=False))
        use[e, recv] = np.arange(nxt, nxt + receivers_per_emitter)
        nxt += receivers_per_emitter
    return dict(numMPs=1, numPaths=nxt - 1, E=T, R=T, use_path=use.ravel(),
                xe=pts[:, 0].copy(), ye=pts[:, 1].copy(), ze=pts[:, 2].copy(),
                xr=pts[:, 0].copy(), yr=pts[:, 1].copy(), zr=pts[:, 2].copy(),
                rv_x=side, rv_y=side, rv_z=side, scale=float(scale))


def ray3d_csr(g):
    """CSR of a 3D ray geometry (rows = numPaths*numMPs compact rays)."""
    E, R, nmp, npaths = g["E"], g["R"], g["numMPs"], g["numPaths"]
    use = np.asarray(g["use_path"]).reshape(E, R)
    e, r = np.nonzero(use)
    rows_all, offs, pixs = [], [], []
    lens = np.zeros(nmp * npaths, np.int64)
    pix_by_ray = {}
    for mp in range(nmp):
        xe = np.asarray(g["xe"]).reshape(nmp, E)[mp]
        ye = np.asarray(g["ye"]).reshape(nmp, E)[mp]
        ze = np.asarray(g["ze"]).reshape(nmp, E)[mp]
        xr = np.asarray(g["xr"]).reshape(nmp, R)[mp]
        yr = np.asarray(g["yr"]).reshape(nmp, R)[mp]
        zr = np.asarray(g["zr"]).reshape(nmp, R)[mp]
        p0 = np.stack([xe[e], ye[e], ze[e]], 1)
        p1 = np.stack([xr[r], yr[r], zr[r]], 1)
        off, pix = bresenham_csr_3d(p0, p1, g["rv_x"], g["rv_y"])
        ray = mp * npaths + use[e, r] - 1
        lens[ray] = np.diff(off)
        pix_by_ray[mp] = (ray, off, pix)
    rowptr = np.zeros(nmp * npaths + 1, np.int64)
    np.cumsum(lens, out=rowptr[1:])
    colind = np.zeros(rowptr[-1], np.int32)
    for mp, (ray, off, pix) in pix_by_ray.items():
        dst = rowptr[ray]
        idx = np.repeat(dst - off[:-1], np.diff(off)) + np.arange(off[-1])
        colind[idx] = pix
    return dict(m=nmp * npaths, n=g["rv_x"] * g["rv_y"] * g["rv_z"], rowptr=rowptr.astype(np.int32),
                colind=colind, val=np.full(len(colind), g["scale"], np.float64))


def csr_matvec(csr, x):
    """y = A x for a CSR dict (float64), vectorised."""
    rowptr = np.asarray(csr["rowptr"], np.int64)
    prod = np.asarray(csr["val"], np.float64) * np.asarray(x, np.float64)[csr["colind"]]
    y = np.zeros(csr["m"])
    nz = np.diff(rowptr) > 0
    sums = np.add.reduceat(prod, rowptr[:-1][nz]) if prod.size else np.zeros(0)
    y[nz] = sums
    return y


# --------------------------------------------------------------------------
# configurations
# --------------------------------------------------------------------------


def dense2d(seed=0, side=64, sampling=0.3, noise=0.01, n_ellipses=5, tv_norm=1, maxit=300, tol=1e-4):
    """Plain 2D TVAL3 with a dense Gaussian A (m x n, N(0, 1/m))."""
    rng = np.random.default_rng(seed)
    n = side * side
    m = int(round(sampling * n))
    u = ellipse_phantom(side, side, rng, n_ellipses, 0.0, lambda r: r.uniform(0.2, 1.0), (4, 20))
    A = (rng.standard_normal((m, n)) / math.sqrt(m)).astype(np.float32)
    b = add_noise(A.astype(np.float64) @ u.ravel(), noise, rng)
    return dict(kind="dense", shape=(side, side), A=A, b=b.astype(np.float32), u_true=u,
                opts=options(2 ** 8, 2 ** 5, tol, maxit, tv_norm=tv_norm))


def sigma_max(csr, iters=40):
    """Largest singular value of a CSR operator (power iteration on A^T A from a
    seeded start; a few parts in 1e4 after 40 steps)."""
    import scipy.sparse as sp
    M = sp.csr_matrix((np.asarray(csr["val"], np.float64), csr["colind"], csr["rowptr"]), shape=(csr["m"], csr["n"]))
    x = np.random.default_rng(12345).standard_normal(csr["n"])
    lam = 0.0
    for _ in range(iters):
        y = M.T @ (M @ x)
        lam = float(np.linalg.norm(y))
        x = y / lam
    return math.sqrt(lam)


def ring2d(seed=1, side=256, T=512, receivers=None, noise=0.005, tv_norm=1, maxit=500, tol=1e-5,
           mu=2 ** 10, beta=2 ** 6, csr=True, normalize=False):
    """2D ultrasound-tomography ring (Bresenham projector + CSR twin).

    normalize: set the geometry's scale_factor (the weight of every hit) to
    1/sigma_max(A) so that A has unit spectral norm, as TVAL3's mu and beta
    assume; with unit weights (normalize=False) sigma_max(A)^2 ~ 1e5 at 256^2
    and the solve stays in its ill-conditioned transient for hundreds of
    iterations."""
    rng = np.random.default_rng(seed)
    n = side * side
    g = ring_geometry(side, T, receivers)
    u = ellipse_phantom(side, side, rng, 8, 1.0, lambda r: 1.0 + r.uniform(-0.05, 0.05),
                        (side / 32, side / 6), centre_radius=side / 3)
    yy, xx = np.mgrid[0:side, 0:side]
    c = (side - 1) / 2.0
    for _ in range(2):   # strong inclusions
        rad = side / 4 * math.sqrt(rng.uniform(0, 1))
        ang = rng.uniform(0, 2 * math.pi)
        cx, cy, r0 = c + rad * math.cos(ang), c + rad * math.sin(ang), rng.uniform(side / 40, side / 16)
        u[(xx - cx) ** 2 + (yy - cy) ** 2 <= r0 ** 2] = 1.0 + rng.choice([-1, 1]) * 0.15
    A = ray2d_csr(g, n)
    if normalize:
        s = 1.0 / sigma_max(A)
        g["scale"] = float(np.float32(s))
        A["val"] = np.full(len(A["colind"]), g["scale"], np.float64)
    y = csr_matvec(A, u.ravel())
    live = np.asarray(g["use_path"]) != 0
    b = np.zeros(A["m"])
    b[live] = add_noise(y[live], noise, rng)
    out = dict(kind="ray2d", shape=(side, side), geom=g, b=b.astype(np.float32), u_true=u,
               opts=options(mu, beta, tol, maxit, tv_norm=tv_norm))
    if csr:
        out["csr"] = A
    return out


def mrhs(seed=4, side=128, m=4096, rhs=32, noise=0.01, tv_norm=1, maxit=300, tol=1e-4):
    """Multi-right-hand-side dense problem: one Gaussian A (m x side^2,
    N(0, 1/m)) and `rhs` phantoms solved jointly as the reference's `layers`
    (the layers stacked along y: image shape (side * rhs, side))."""
    rng = np.random.default_rng(seed)
    n = side * side
    A = (rng.standard_normal((m, n), dtype=np.float32) / np.float32(math.sqrt(m))).astype(np.float32)
    us = [ellipse_phantom(side, side, rng, 5, 0.0, lambda r: r.uniform(0.2, 1.0), (side / 16, side / 3.2))
          for _ in range(rhs)]
    U = np.stack([u.ravel() for u in us])                       # rhs x n
    Y = (A.astype(np.float64) @ U.T).T                          # rhs x m
    b = np.concatenate([add_noise(y, noise, rng) for y in Y])
    return dict(kind="dense", shape=(side * rhs, side), A=A, b=b.astype(np.float32), u_true=U.reshape(side * rhs, side),
                layers=rhs, opts=options(2 ** 8, 2 ** 5, tol, maxit, tv_norm=tv_norm))


def batch_specs(seed=3, count=64, sides=(64, 96, 128, 192, 256)):
    """The mixed batch of independent 2D problems: per instance a side drawn
    from `sides`, and either a dense Gaussian A (sampling 25-40 %, the
    counter-based Gaussian stream of the instance seed, drawn on the device
    or regenerated on the host) or a ring geometry (128-512 transducers).
    Returns descriptions; batch_dense_parts / batch_dense_host / batch_ray
    materialise them."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        side = int(rng.choice(sides))
        if rng.uniform() < 0.5:
            out.append(dict(kind="dense", side=side, sampling=float(rng.uniform(0.25, 0.40)),
                            seed=int(rng.integers(1 << 30))))
        else:
            T = int(rng.choice([128, 192, 256, 384, 512]))
            out.append(dict(kind="ray2d", side=side, T=T, seed=int(rng.integers(1 << 30))))
    return out


def batch_dense_parts(d):
    """The pieces of a dense batch instance that do not need its matrix: the
    shape (side, side), m, the phantom, the options and the noise generator
    (drawn after the phantom).  Its A is the Gaussian stream of the instance
    seed, scaled by 1/sqrt(m) (philox_gaussian / tval3g_gaussian), row-major
    m x n; b = float32(A u) plus 1 % noise from the returned generator."""
    side = d["side"]
    n = side * side
    m = int(round(d["sampling"] * n))
    rng = np.random.default_rng(d["seed"])
    u = ellipse_phantom(side, side, rng, 5, 0.0, lambda r: r.uniform(0.2, 1.0), (side / 16, side / 3.2))
    return dict(shape=(side, side), m=m, n=n, u_true=u, rng=rng, scale=float(np.float32(1.0 / math.sqrt(m))),
                opts=options(2 ** 8, 2 ** 5, 1e-4, 300, tv_norm=1))


def batch_dense_host(d):
    """A dense batch instance materialised on the host (A from the numpy
    restatement of the device generator)."""
    p = batch_dense_parts(d)
    A = philox_gaussian(d["seed"], p["m"] * p["n"], p["scale"]).reshape(p["m"], p["n"])
    y = (A.astype(np.float64) @ p["u_true"].ravel()).astype(np.float32)
    b = add_noise(y.astype(np.float64), 0.01, p["rng"]).astype(np.float32)
    return dict(kind="dense", shape=p["shape"], A=A, b=b, u_true=p["u_true"], opts=p["opts"])


def batch_ray(d):
    """A ring batch instance (host geometry and data; hit weight 1/sigma_max)."""
    return ring2d(seed=d["seed"], side=d["side"], T=d["T"], tv_norm=1, maxit=500, tol=1e-5, normalize=True)


def hemi3d(seed=2, side=128, T=2048, receivers=1024, noise=0.005, tv_norm=0, maxit=400, tol=1e-5,
           n_ellipsoids=12, csr=False, forward=None, normalize=False):
    """3D hemisphere geometry (on-the-fly 3D Bresenham).

    forward: optional callable (geometry, image) -> A image; by default the
    data come from the CSR twin built here (which needs ~1 GB of host memory
    per 1e8 hits at full size).  normalize (with the CSR twin): hit weight
    scale_factor = 1/sigma_max(A), as ring2d's."""
    rng = np.random.default_rng(seed)
    radius = (side - 1) / 2.0 - 0.5
    g = hemisphere_geometry(side, T, receivers, radius, rng)
    u = ellipsoid_phantom(side, rng, n_ellipsoids, 1.0, lambda r: 1.0 + r.uniform(-0.05, 0.05),
                          (side / 16, side / 5))
    A = ray3d_csr(g) if (csr or forward is None) else None
    if normalize and A is not None:
        g["scale"] = float(np.float32(1.0 / sigma_max(A)))
        A["val"] = np.full(len(A["colind"]), g["scale"], np.float64)
    y = csr_matvec(A, u.ravel()) if forward is None else np.asarray(forward(g, u), np.float64)
    b = add_noise(y, noise, rng)
    out = dict(kind="ray3d", shape=(side, side, side), geom=g, b=b.astype(np.float32), u_true=u,
               opts=options(2 ** 10, 2 ** 6, tol, maxit, tv_norm=tv_norm))
    if csr:
        out["csr"] = A
    return out
