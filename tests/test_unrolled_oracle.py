"""The FP64 unrolled-solve oracle (oracle/unrolled.py): its hand-written
adjoint against central finite differences and against torch autograd on a
dense-A FP64 restatement of the same iteration map."""
import numpy as np
import pytest
import torch

import unrolled as UR

FD_TOL = 1e-6       # directional derivatives, FP64 central differences (step 1e-6 relative)
AUTOGRAD_TOL = 1e-9


def _case(iso, seed=0, p=12, q=12, m=60, K=12):
    rng = np.random.default_rng(seed)
    n = p * q
    A = rng.standard_normal((m, n)) / np.sqrt(m)
    u = np.zeros((p, q))
    u[3:8, 4:9] = 1.0
    u = u.ravel()
    b = A @ u + 0.01 * rng.standard_normal(m)
    steps = 0.05 + 0.1 * rng.uniform(size=K)
    outer = np.zeros(K, bool)
    outer[[3, 7]] = True
    mu = 2.0 ** 4 * (1 + 0.1 * rng.uniform(size=K))
    beta = 2.0 ** 3 * (1 + 0.1 * rng.uniform(size=K))
    F = UR.Unrolled(lambda x: A @ x, lambda y: A.T @ y, (p, q), steps, outer, 0.7, iso)
    return F, A, b, u, mu, beta, rng


@pytest.mark.parametrize("iso", [False, True])
def test_adjoint_matches_central_differences(iso):
    F, A, b, u, mu, beta, rng = _case(iso)
    gb, gmu, gbeta = F.backward(b, mu, beta, F.forward(b, mu, beta) - u)

    def loss(b_, mu_, beta_):
        return 0.5 * np.sum((F.forward(b_, mu_, beta_) - u) ** 2)

    h, sb = 1e-6, np.abs(b).mean()
    for _ in range(64):
        vb, vm, vB = rng.standard_normal(b.size), rng.standard_normal(mu.size), rng.standard_normal(beta.size)
        fd = (loss(b + h * sb * vb, mu * (1 + h * vm), beta * (1 + h * vB)) -
              loss(b - h * sb * vb, mu * (1 - h * vm), beta * (1 - h * vB))) / (2 * h)
        an = sb * np.dot(gb, vb) + np.dot(gmu, mu * vm) + np.dot(gbeta, beta * vB)
        assert abs(fd - an) <= FD_TOL * max(abs(fd), 1e-12), (fd, an)


def _torch_map(A, shape, steps, outer, scl, iso):
    """The same iteration map in torch (FP64, dense A), differentiated by autograd."""
    p, q = shape
    At = torch.tensor(A, dtype=torch.float64)

    def D(U):
        U2 = U.reshape(p, q)
        return (torch.roll(U2, -1, 1) - U2).reshape(-1), (torch.roll(U2, -1, 0) - U2).reshape(-1)

    def Dt(X, Y):
        X2, Y2 = X.reshape(p, q), Y.reshape(p, q)
        return (torch.roll(X2, 1, 1) - X2 + torch.roll(Y2, 1, 0) - Y2).reshape(-1)

    def S(zx, zy, t):
        if iso:
            nrm = torch.sqrt(zx * zx + zy * zy + 1e-300)
            s = torch.clamp(nrm - t, min=0.0) / nrm
            return s * zx, s * zy
        return torch.sign(zx) * torch.clamp(zx.abs() - t, min=0.0), torch.sign(zy) * torch.clamp(zy.abs() - t, min=0.0)

    def F(b, mu, beta):
        bs = scl * b
        U = At.T @ bs
        sx = torch.zeros_like(U)
        sy = torch.zeros_like(U)
        dl = torch.zeros_like(bs)

        def state(U, sx, sy, dl, m_, b_, o):
            Vx, Vy = D(U)
            Wx, Wy = S(Vx - sx / b_, Vy - sy / b_, 1.0 / b_)
            Ex, Ey = Vx - Wx, Vy - Wy
            r = At @ U - bs
            if o:
                sx, sy, dl = sx - b_ * Ex, sy - b_ * Ey, dl - m_ * r
            d = Dt(Ex - sx / b_, Ey - sy / b_) + At.T @ ((m_ * r - dl) / b_)
            return sx, sy, dl, d

        sx, sy, dl, d = state(U, sx, sy, dl, mu[0], beta[0], False)
        for k in range(1, len(steps) + 1):
            U = U - float(steps[k - 1]) * d
            sx, sy, dl, d = state(U, sx, sy, dl, mu[k - 1], beta[k - 1], bool(outer[k - 1]))
        return U / scl

    return F


@pytest.mark.parametrize("iso", [False, True])
def test_adjoint_matches_torch_autograd(iso):
    F, A, b, u, mu, beta, _ = _case(iso, seed=1)
    tF = _torch_map(A, (F.p, F.q), F.steps, F.outer, F.scl, iso)
    tb = torch.tensor(b, requires_grad=True)
    tm = torch.tensor(mu, requires_grad=True)
    tB = torch.tensor(beta, requires_grad=True)
    U = tF(tb, tm, tB)
    assert np.allclose(U.detach().numpy(), F.forward(b, mu, beta), rtol=1e-12, atol=1e-12)
    (0.5 * ((U - torch.tensor(u)) ** 2).sum()).backward()
    gb, gmu, gbeta = F.backward(b, mu, beta, F.forward(b, mu, beta) - u)
    for got, ref in ((gb, tb.grad), (gmu, tm.grad), (gbeta, tB.grad)):
        ref = ref.numpy()
        assert np.linalg.norm(got - ref) <= AUTOGRAD_TOL * np.linalg.norm(ref)


def test_kinks_held_fixed_on_a_large_case():
    """128x128 ring (256 transducers x 128 receivers), K = 50 with the step
    lengths of an oracle solve: a central difference with step 1e-6 crosses
    shrinkage kinks in some directions; on the smooth piece of the point
    (kinks held fixed) it matches the adjoint, and without a kink crossing
    (step 1e-8) it matches as well."""
    import oracle as O
    from tval3g import workloads as W
    side, K = 128, 50
    w = W.ring2d(seed=11, side=side, T=256, tv_norm=1, normalize=True)
    g, b, u = w["geom"], w["b"].astype(np.float64), w["u_true"].ravel()
    op = O.Op.ray2d(g, side * side)
    opts = W.options(2 ** 8, 2 ** 5, 1e-4, K, tv_norm=1)
    r = O.solve(op, b, (side, side), opts, record=True)
    steps = np.array([it[0] * opts["gamma"] ** it[3] for it in r.iters])[:K]
    F = UR.Unrolled(lambda x: op.apply(x), lambda y: op.apply(y, True), (side, side), steps, np.zeros(K, bool),
                    1.0, True)
    mu, beta = np.full(K, 2.0 ** 8), np.full(K, 2.0 ** 5)
    kinks = []
    U = F.forward(b, mu, beta, kinks=kinks)
    assert len(kinks) == K + 1
    gb, gmu, gbeta = F.backward(b, mu, beta, U - u)
    rng = np.random.default_rng(5)
    sb = np.abs(b).mean()

    def fd(h, vb, vm, vB, kk):
        L = lambda s_: 0.5 * np.sum((F.forward(b + s_ * h * sb * vb, mu * (1 + s_ * h * vm), beta * (1 + s_ * h * vB),
                                               kinks=kk) - u) ** 2)  # noqa: E731
        return (L(1) - L(-1)) / (2 * h)

    plain_1e6 = []
    for _ in range(4):
        vb, vm, vB = rng.standard_normal(b.size), rng.standard_normal(K), rng.standard_normal(K)
        an = sb * np.dot(gb, vb) + np.dot(gmu, mu * vm) + np.dot(gbeta, beta * vB)
        assert abs(fd(1e-6, vb, vm, vB, kinks) - an) <= 1e-6 * abs(an)
        assert abs(fd(1e-8, vb, vm, vB, None) - an) <= 1e-5 * abs(an)
        plain_1e6.append(abs(fd(1e-6, vb, vm, vB, None) - an) / abs(an))
    # at least one of these directions crosses a kink with step 1e-6
    assert max(plain_1e6) > 1e-4, plain_1e6
