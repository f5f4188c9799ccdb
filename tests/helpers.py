"""Helpers shared by the tests (paths are set up by conftest.py)."""
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def relerr(a, b):
    dt = np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64
    a = np.asarray(a, dt).ravel()
    b = np.asarray(b, dt).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))


# The FP32 noise floor of a solve.  A converged TVAL3 solve can be sensitive
# to perturbations of FP32 size: its threshold decisions (backtracking, where
# the inner loop ends) and its nonmonotone line search amplify them, so that
# two FP64 solves of the same problem whose stored vectors differ by a few
# FP32 roundings per iteration can end 1e-3 - 1e-1 apart (the spread is
# heavy-tailed).  The oracle's noise model (orc_opts.noise: every element of
# U, its differences, Au, g and g2 multiplied by 1 + eps xi after each
# descent, xi uniform in [-1, 1], eps = four FP32 unit roundoffs: an FP32
# vector comes out of a chain of several rounded operations) measures that
# sensitivity per problem; an FP32 solve is held to max(1e-3, 2 x the
# largest distance of six such perturbed FP64 solves from the unperturbed
# one).  Fixed short solves have floors near 1e-6, so their bar is 1e-3.
NOISE_EPS = 4 * 2.0 ** -24
NOISE_SEEDS = (1, 2, 3, 4, 5, 6)
BAR = 1e-3


def noise_floor(solve, U64, seeds=NOISE_SEEDS):
    """solve(extra_opts) -> oracle Result; U64 the unperturbed FP64 solution."""
    return max(relerr(solve({"noise": NOISE_EPS, "noise_seed": s}).U, U64) for s in seeds)


def solve_bar(floor):
    return max(BAR, 2.0 * floor)
