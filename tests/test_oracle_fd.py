"""Finite-difference checks of the NDT derivatives, pair by pair, in double.

For one scan point x, cell mean mu and inverse covariance C, the pair's
score is -d1 exp(-d2 v'Cv / 2) with v = T(p) x - mu and T = Trans * Rx * Ry
* Rz (the parametrisation eqs. 6.19 / 6.21 differentiate).  The oracle's
gradient (eq. 6.12) must be its derivative in both modes; the corrected
mode's Hessian (eq. 6.13) must be the derivative of that gradient.  Compat
mode keeps the reference's Hessian (kernel.cpp:486-488 accumulates another
expression, and its h_ang_d1 has the opposite sign of sin(pitch),
kernel.cpp:797), which is not one."""
import math

import numpy as np
import pytest


def _rot(p):
    a, b, c = p[3:]
    Rx = np.array([[1, 0, 0], [0, math.cos(a), -math.sin(a)], [0, math.sin(a), math.cos(a)]])
    Ry = np.array([[math.cos(b), 0, math.sin(b)], [0, 1, 0], [-math.sin(b), 0, math.cos(b)]])
    Rz = np.array([[math.cos(c), -math.sin(c), 0], [math.sin(c), math.cos(c), 0], [0, 0, 1]])
    return Rx @ Ry @ Rz, np.asarray(p[:3])


def _cases(seed, n):
    rng = np.random.default_rng(seed)
    for _ in range(n):
        p = rng.uniform(-0.4, 0.4, 6)
        x = rng.uniform(-3, 3, 3)
        A = rng.normal(size=(3, 3))
        C = A @ A.T + 0.5 * np.eye(3)
        R, t = _rot(p)
        mu = R @ x + t + rng.normal(0, 0.3, 3)
        yield p, x, C, mu


def _errors(oracle, prm, p, x, C, mu, h=1e-5):
    d1, d2 = oracle.gauss(prm)

    def offset(q):
        R, t = _rot(q)
        return R @ x + t - mu

    def score(q):
        v = offset(q)
        return -d1 * math.exp(-d2 * float(v @ C @ v) / 2)

    def grad(q):
        return oracle.update_pair(prm, q, x, offset(q), C, True)[1]

    s, g, H = oracle.update_pair(prm, p, x, offset(p), C, True)
    assert math.isclose(s, score(p), rel_tol=1e-14)
    E = np.eye(6) * h
    g_fd = np.array([(score(p + E[i]) - score(p - E[i])) / (2 * h) for i in range(6)])
    H_fd = np.array([(grad(p + E[i]) - grad(p - E[i])) / (2 * h) for i in range(6)]).T
    return np.linalg.norm(g - g_fd) / np.linalg.norm(g), np.linalg.norm(H - H_fd) / np.linalg.norm(H)


def test_corrected_gradient_and_hessian(oracle, binding_mod):
    prm = binding_mod.corrected_params()
    for p, x, C, mu in _cases(1, 60):
        eg, eh = _errors(oracle, prm, p, x, C, mu)
        assert eg < 1e-6 and eh < 1e-6, (eg, eh)


def test_compat_gradient_is_exact_hessian_is_the_references(oracle, binding_mod):
    prm = binding_mod.reference_params()
    worst_h = 0.0
    for p, x, C, mu in _cases(2, 60):
        eg, eh = _errors(oracle, prm, p, x, C, mu)
        assert eg < 1e-6, eg
        worst_h = max(worst_h, eh)
    assert worst_h > 1e-2  # the reference's Hessian is not the derivative of its gradient


@pytest.mark.parametrize("pitch", [0.3, -0.7])
def test_pitch_second_derivative_known_answer(oracle, binding_mod, pitch):
    """H[4][4] of a pure-pitch pose for the point (0, 0, 1): the term the modes differ in.  With
    x' = (sin b, 0, cos b): J4 = (cos b, 0, -sin b) and d^2x'/db^2 = (-sin b, 0, -cos b), so eq. 6.13 gives
    H44 = d1 d2 e (-d2 (v.J4)^2 + J4.J4 + v.(-sin b, 0, -cos b))."""
    prm = binding_mod.corrected_params()
    d1, d2 = oracle.gauss(prm)
    x = np.array([0.0, 0.0, 1.0])
    p = np.array([0.0, 0.0, 0.0, 0.0, pitch, 0.0])
    v = np.array([0.2, -0.1, 0.15])  # offset of the transformed point from the cell mean
    H = oracle.update_pair(prm, p, x, v, np.eye(3), True)[2]
    e = math.exp(-d2 * float(v @ v) / 2)
    J4 = np.array([math.cos(pitch), 0.0, -math.sin(pitch)])
    d44 = np.array([-math.sin(pitch), 0.0, -math.cos(pitch)])
    h44 = d1 * d2 * e * (-d2 * float(v @ J4) ** 2 + float(J4 @ J4) + float(v @ d44))
    assert math.isclose(H[4, 4], h44, rel_tol=1e-12)
