"""Unrolled TVAL3 and its adjoint in FP64 — test infrastructure only.

Only tests/ and bench.py's checks import this module; the product path never
does.  It restates, in numpy, the function that tval3g differentiates
(tval3g_unrolled_*): K inner iterations of the TVAL3 solve (modk/tval3-cpu
2d/tval3_cpu_2d.cpp:752-853) in 2D with per-iteration (mu_k, beta_k) in place
of the continuation, and with the decisions of a forward solve held fixed:
the step of every iteration (tau_k times the backtracking factor, the BB /
Armijo outcome of 2d:425-453,526-576) and whether the multipliers were
updated after it (2d:673-694, 2d:820-842).  With the scaled data bs = scl b:

    U_0 = A^T bs,  sigma_0 = 0,  delta_0 = 0                      (2d:767-779)
    state(k): V = D U_k, Z = V - sigma_{k-1} / beta_k, W = S(Z, 1/beta_k),
              E = V - W, r = A U_k - bs;                           (2d:588-671)
              if outer_k: sigma_k = sigma_{k-1} - beta_k E,
                          delta_k = delta_{k-1} - mu_k r          (2d:673-694)
              d_k = D^T (E - sigma_k / beta_k) + A^T ((mu_k r - delta_k) / beta_k)
                                                                   (2d:578-585)
    iteration k = 1..K: U_k = U_{k-1} - step_k d_{k-1}; state(k)   (2d:481-493)
    output U_K / scl; iteration 0 uses (mu_1, beta_1)

S is the shrinkage (anisotropic 2d:588-611, or isotropic).  The adjoint
below is derived by hand from these lines; tests check it against central
finite differences of `forward` and against torch autograd.

F is piecewise smooth: S has a kink where |Z| = 1/beta.  The adjoint is the
derivative of the piece active at the point.  On large problems a central
difference with step 1e-6 crosses some of the millions of kinks on its way
(one crossing moves the quotient by up to 1e-2), so `forward(kinks=...)`
can hold every shrinkage on the branches of a recorded point, as the step
lengths and multiplier updates already are.
"""
from __future__ import annotations

import numpy as np


def D2(U, p, q):
    U = U.reshape(p, q)
    return (np.roll(U, -1, axis=1) - U).ravel(), (np.roll(U, -1, axis=0) - U).ravel()


def Dt2(X, Y, p, q):
    X, Y = X.reshape(p, q), Y.reshape(p, q)
    return (np.roll(X, 1, axis=1) - X + np.roll(Y, 1, axis=0) - Y).ravel()


def shrink(Zx, Zy, t, iso):
    if iso:
        nrm = np.sqrt(Zx * Zx + Zy * Zy)
        s = np.where(nrm > 0, np.maximum(nrm - t, 0.0) / np.where(nrm > 0, nrm, 1.0), 0.0)
        return s * Zx, s * Zy
    return (np.sign(Zx) * np.maximum(np.abs(Zx) - t, 0.0), np.sign(Zy) * np.maximum(np.abs(Zy) - t, 0.0))


def shrink_on(Zx, Zy, t, iso):
    """Where the shrinkage is off its zero branch (iso: one mask; aniso: one per component)."""
    if iso:
        return (np.sqrt(Zx * Zx + Zy * Zy) > t,)
    return np.abs(Zx) > t, np.abs(Zy) > t


def shrink_fixed(Zx, Zy, t, iso, on):
    """The shrinkage with its branch held at `on` (from shrink_on at another
    point): the smooth piece of S that is active there."""
    if iso:
        nrm = np.sqrt(Zx * Zx + Zy * Zy)
        s = np.where(on[0], (nrm - t) / np.where(on[0], nrm, 1.0), 0.0)
        return s * Zx, s * Zy
    return (np.where(on[0], np.sign(Zx) * (np.abs(Zx) - t), 0.0),
            np.where(on[1], np.sign(Zy) * (np.abs(Zy) - t), 0.0))


def shrink_vjp(Zx, Zy, t, iso, Wbx, Wby):
    """(Zbar_x, Zbar_y, tbar) for W = S(Z, t) and the cotangent Wbar."""
    if iso:
        nrm = np.sqrt(Zx * Zx + Zy * Zy)
        on = nrm > t
        nn = np.where(on, nrm, 1.0)
        zw = (Zx * Wbx + Zy * Wby) / nn
        a = np.where(on, 1.0 - t / nn, 0.0)
        c = np.where(on, t / (nn * nn), 0.0)
        Zbx = a * Wbx + c * Zx * zw
        Zby = a * Wby + c * Zy * zw
        tbar = float(np.sum(np.where(on, -zw, 0.0)))
        return Zbx, Zby, tbar
    onx, ony = np.abs(Zx) > t, np.abs(Zy) > t
    Zbx, Zby = np.where(onx, Wbx, 0.0), np.where(ony, Wby, 0.0)
    tbar = float(np.sum(np.where(onx, -np.sign(Zx) * Wbx, 0.0)) + np.sum(np.where(ony, -np.sign(Zy) * Wby, 0.0)))
    return Zbx, Zby, tbar


class Unrolled:
    """F(b, mu, beta) = U_K / scl for fixed decisions (steps, outer, scl).

    A, At: callables (image -> measurements, measurements -> image) in FP64."""

    def __init__(self, A, At, shape, steps, outer, scl, iso):
        self.A, self.At = A, At
        self.p, self.q = shape
        self.steps = np.asarray(steps, np.float64)
        self.outer = np.asarray(outer, bool)
        self.scl = float(scl)
        self.iso = bool(iso)
        self.K = len(self.steps)

    def _state(self, U, sx, sy, dl, bs, mu, beta, o, kinks=None, k=0):
        p, q = self.p, self.q
        Vx, Vy = D2(U, p, q)
        Zx, Zy = Vx - sx / beta, Vy - sy / beta
        if kinks is None:
            Wx, Wy = shrink(Zx, Zy, 1.0 / beta, self.iso)
        elif len(kinks) == k:      # recording
            kinks.append(shrink_on(Zx, Zy, 1.0 / beta, self.iso))
            Wx, Wy = shrink(Zx, Zy, 1.0 / beta, self.iso)
        else:
            Wx, Wy = shrink_fixed(Zx, Zy, 1.0 / beta, self.iso, kinks[k])
        Ex, Ey = Vx - Wx, Vy - Wy
        r = self.A(U) - bs
        if o:
            sx, sy, dl = sx - beta * Ex, sy - beta * Ey, dl - mu * r
        d = Dt2(Ex - sx / beta, Ey - sy / beta, p, q) + self.At((mu * r - dl) / beta)
        return sx, sy, dl, d, r

    def forward(self, b, mu, beta, trajectory=False, kinks=None):
        """U_K / scl.  kinks: None, or an empty list that this call fills with
        the shrinkage branches it takes, or such a filled list, which then
        holds every shrinkage on those branches (the map's smooth piece at the
        point that recorded them, for finite differences that must not cross
        a kink)."""
        bs = self.scl * np.asarray(b, np.float64)
        n = self.p * self.q
        U = self.At(bs)
        sx, sy, dl = np.zeros(n), np.zeros(n), np.zeros(bs.size)
        traj = []
        sx, sy, dl, d, r = self._state(U, sx, sy, dl, bs, mu[0], beta[0], False, kinks, 0)
        traj.append((U, np.zeros(n), np.zeros(n), sx, sy, dl, r))
        for k in range(1, self.K + 1):
            U = U - self.steps[k - 1] * d
            s0x, s0y = sx, sy
            sx, sy, dl, d, r = self._state(U, sx, sy, dl, bs, mu[k - 1], beta[k - 1], self.outer[k - 1], kinks, k)
            traj.append((U, s0x, s0y, sx, sy, dl, r))
        out = U / self.scl
        return (out, traj) if trajectory else out

    def backward(self, b, mu, beta, gU):
        """Gradients (gb, gmu, gbeta) of <gU, F(b, mu, beta)>."""
        mu, beta = np.asarray(mu, np.float64), np.asarray(beta, np.float64)
        _, traj = self.forward(b, mu, beta, trajectory=True)
        p, q, K = self.p, self.q, self.K
        n = p * q
        Ub = np.asarray(gU, np.float64) / self.scl
        sbx, sby = np.zeros(n), np.zeros(n)
        db = np.zeros(traj[0][6].size)
        bsb = np.zeros_like(db)
        gmu, gbeta = np.zeros(K), np.zeros(K)
        dd = None   # cotangent of d_k
        for k in range(K, -1, -1):
            U, s0x, s0y, sx, sy, dl, r = traj[k]
            j = max(k, 1) - 1
            m_, b_ = mu[j], beta[j]
            o = bool(self.outer[k - 1]) if k >= 1 else False
            Vx, Vy = D2(U, p, q)
            Zx, Zy = Vx - s0x / b_, Vy - s0y / b_
            Wx, Wy = shrink(Zx, Zy, 1.0 / b_, self.iso)
            Ex, Ey = Vx - Wx, Vy - Wy
            Ebx, Eby = np.zeros(n), np.zeros(n)
            rb = np.zeros_like(r)
            if dd is not None:
                Ddx, Ddy = D2(dd, p, q)
                Ad = self.A(dd)
                Ebx, Eby = Ddx.copy(), Ddy.copy()
                sbx, sby = sbx - Ddx / b_, sby - Ddy / b_
                rb = (m_ / b_) * Ad
                db = db - Ad / b_
                gmu[j] += np.dot(Ad, r) / b_
                gbeta[j] += (np.dot(Ddx, sx) + np.dot(Ddy, sy)) / b_ ** 2 + np.dot(Ad, dl - m_ * r) / b_ ** 2
            if o:
                Ebx, Eby = Ebx - b_ * sbx, Eby - b_ * sby
                gbeta[j] -= np.dot(sbx, Ex) + np.dot(sby, Ey)
                rb = rb - m_ * db
                gmu[j] -= np.dot(db, r)
            Wbx, Wby = -Ebx, -Eby
            Zbx, Zby, tbar = shrink_vjp(Zx, Zy, 1.0 / b_, self.iso, Wbx, Wby)
            gbeta[j] += -tbar / b_ ** 2 + (np.dot(Zbx, s0x) + np.dot(Zby, s0y)) / b_ ** 2
            Vbx, Vby = Ebx + Zbx, Eby + Zby
            sbx, sby = sbx - Zbx / b_, sby - Zby / b_
            Ub = Ub + self.At(rb) + Dt2(Vbx, Vby, p, q)
            bsb = bsb - rb
            if k >= 1:
                dd = -self.steps[k - 1] * Ub
        bsb = bsb + self.A(Ub)   # U_0 = A^T bs
        return self.scl * bsb, gmu, gbeta
