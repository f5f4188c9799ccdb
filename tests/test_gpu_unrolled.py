"""Differentiable unrolled solve on the GPU (tval3g_unrolled_*): the forward
against the FP64 oracle with the recorded decisions, the hand-written CUDA
adjoint against the oracle's adjoint and against FP64 central finite
differences, and the torch.autograd binding."""
import numpy as np
import pytest

import oracle as O
import unrolled as UR
from helpers import relerr
from tval3g import capi
from tval3g import workloads as W

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-4      # U_K (FP32 replay) against the FP64 oracle, relative L2
GRAD_TOL = 1e-3     # gradients (FP32 forward and adjoint) against the FP64 adjoint, relative L2
FD_TOL = 1e-4       # directional derivatives against FP64 central differences (step 1e-6 relative)


def _batch(side, T, count, iso, seed=11):
    ws = [W.ring2d(seed=seed + i, side=side, T=T, tv_norm=int(iso), normalize=True) for i in range(count)]
    g = ws[0]["geom"]
    b = np.stack([w["b"] for w in ws]).astype(np.float32)
    u = np.stack([w["u_true"].ravel() for w in ws])
    return g, b, u


def _schedule(K):
    k = np.arange(K)
    return 2.0 ** 8 * (1 + 0.2 * np.sin(k)), 2.0 ** 5 * (1 + 0.2 * np.cos(k))


def _check(torch, side, T, count, K, ckpt, iso, n_dirs, mu, beta):
    from tval3g.autograd import unrolled_tval3
    g, b, u = _batch(side, T, count, iso)
    spec = capi.ray2d_problem((side, side), g)
    opts = W.options(2 ** 8, 2 ** 5, 1e-4, K, tv_norm=int(iso))
    h = capi.Unrolled(spec, count, opts, K, ckpt=ckpt)
    tb = torch.tensor(b, device="cuda", requires_grad=True)
    tm = torch.tensor(mu, requires_grad=True)
    tB = torch.tensor(beta, requires_grad=True)
    U = unrolled_tval3(tb, tm, tB, h)
    loss = 0.5 * ((U - torch.tensor(u, device="cuda", dtype=torch.float32)) ** 2).sum()
    loss.backward()
    Ug = U.detach().cpu().numpy()
    gb = tb.grad.cpu().numpy()

    op = O.Op.ray2d(g, side * side)
    A, At = (lambda x: op.apply(x)), (lambda y: op.apply(y, True))
    gmu_ref, gbeta_ref = np.zeros(K), np.zeros(K)
    Fs = []
    errs = {"fwd": [], "gb": [], "fd": []}
    for i in range(count):
        steps, outer, scl = h.decisions(i)
        assert np.all(steps > 0) and not outer[-1]
        F = UR.Unrolled(A, At, (side, side), steps, outer, scl, iso)
        Fs.append(F)
        U64 = F.forward(b[i], mu, beta)
        errs["fwd"].append(relerr(Ug[i], U64))
        gb_i, gm_i, gB_i = F.backward(b[i], mu, beta, U64 - u[i])
        errs["gb"].append(relerr(gb[i], gb_i))
        assert errs["fwd"][-1] <= FWD_TOL and errs["gb"][-1] <= GRAD_TOL
        gmu_ref += gm_i
        gbeta_ref += gB_i
    errs["gmu"], errs["gbeta"] = relerr(tm.grad.numpy(), gmu_ref), relerr(tB.grad.numpy(), gbeta_ref)
    assert errs["gmu"] <= GRAD_TOL and errs["gbeta"] <= GRAD_TOL

    # directional derivatives against central differences of the FP64 map.
    # The map is piecewise smooth (shrinkage kinks at |Z| = 1/beta); with
    # 10^5-10^7 shrinkage evaluations a step of 1e-6 crosses a few kinks in
    # some directions, so the differences run on the smooth piece of the
    # unperturbed point: every shrinkage held on the branch it took there, as
    # the step lengths and multiplier updates are.
    rng = np.random.default_rng(5)
    kinks = []
    for i, F in enumerate(Fs):
        kinks.append([])
        F.forward(b[i], mu, beta, kinks=kinks[i])

    def L(db, fm, fB):
        return sum(0.5 * np.sum((F.forward(b[i] + db[i], mu * fm, beta * fB, kinks=kinks[i]) - u[i]) ** 2)
                   for i, F in enumerate(Fs))

    hstep, sb = 1e-6, np.abs(b).mean()
    for _ in range(n_dirs):
        vb = rng.standard_normal(b.shape)
        vm, vB = rng.standard_normal(K), rng.standard_normal(K)
        fd = (L(hstep * sb * vb, 1 + hstep * vm, 1 + hstep * vB) - L(-hstep * sb * vb, 1 - hstep * vm, 1 - hstep * vB)) \
            / (2 * hstep)
        an = sb * np.sum(gb * vb) + np.dot(tm.grad.numpy(), mu * vm) + np.dot(tB.grad.numpy(), beta * vB)
        errs["fd"].append(abs(fd - an) / abs(fd))
        assert errs["fd"][-1] <= FD_TOL, (fd, an)
    h.close()
    return errs


@pytest.mark.parametrize("iso", [False, True])
def test_unrolled_forward_and_adjoint(iso, torch_cuda):
    """32x32 ring, 3 instances, K = 20, varying (mu_k, beta_k), 64 directions."""
    mu, beta = _schedule(20)
    errs = _check(torch_cuda, 32, 32, 3, 20, 6, iso, 64, mu, beta)
    print("unrolled 32x32 iso=%d" % iso, {k: float(np.max(v)) for k, v in errs.items()})


def test_unrolled_differentiation_config(torch_cuda):
    """128x128 ring, 256 transducers x 128 receivers (m = 32768), 8 instances,
    K = 50 with a checkpoint every 10, (mu_k, beta_k) = (2^8, 2^5), 64 directions."""
    errs = _check(torch_cuda, 128, 256, 8, 50, 10, True, 64, np.full(50, 2.0 ** 8), np.full(50, 2.0 ** 5))
    print("unrolled 128x128 K=50", {k: float(np.max(v)) for k, v in errs.items()})
