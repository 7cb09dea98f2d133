"""The face-flux expansion of the stage kernels (face_expand in
nexd-3d_b200/csrc/stage_kernel.cuh), restated in numpy and checked against the
rank-3 coefficient form it replaces:

  stresses   A0 [n n^T + c (s s^T + t t^T)] + A1 (n s^T + s n^T) + A2 (n t^T + t n^T)
  velocities -(A0 n / Zp + (A1 s + A2 t) / Zs)
  anelastic  A0 n n^T / (lambda + 2 mu) + (A1 (n s^T + s n^T) + A2 (n t^T + t n^T)) / (2 mu)

The kernel evaluates the stresses as n v^T + v n^T + c A0 I with
v = (1-c)/2 A0 n + A1 s + A2 t, which uses s s^T + t t^T = I - n n^T for an
orthonormal face frame.  CPU only.
"""
import numpy as np

VOIGT = [(0, 0), (1, 1), (2, 2), (0, 1), (1, 2), (0, 2)]


def frame(rng):
    n = rng.standard_normal(3)
    n /= np.linalg.norm(n)
    s = np.cross(n, rng.standard_normal(3))
    s /= np.linalg.norm(s)
    return n, s, np.cross(n, s)


def coefficient_form(n, s, t, c, izp, izs, ap, as_, A0, A1, A2):
    sym = lambda a, b: np.outer(a, b) + np.outer(b, a)
    sig = A0 * (np.outer(n, n) + c * (np.outer(s, s) + np.outer(t, t))) + A1 * sym(n, s) + A2 * sym(n, t)
    vel = -(izp * A0 * n + izs * (A1 * s + A2 * t))
    an = A0 * ap * np.outer(n, n) + as_ * (A1 * sym(n, s) + A2 * sym(n, t))
    return np.array([sig[i, j] for i, j in VOIGT]), vel, np.array([an[i, j] for i, j in VOIGT])


def compact_form(n, s, t, c, izp, izs, ap, as_, A0, A1, A2):
    """The arithmetic of face_expand, operation for operation (in FP64)."""
    m = A1 * s + A2 * t
    v = 0.5 * (1.0 - c) * A0 * n + m
    b = c * A0
    sig = np.array([2 * n[0] * v[0] + b, 2 * n[1] * v[1] + b, 2 * n[2] * v[2] + b,
                    n[0] * v[1] + v[0] * n[1], n[1] * v[2] + v[1] * n[2], n[0] * v[2] + v[0] * n[2]])
    vel = -(izp * A0 * n + izs * m)
    u = 0.5 * ap * A0 * n + as_ * m
    an = np.array([2 * n[0] * u[0], 2 * n[1] * u[1], 2 * n[2] * u[2],
                   n[0] * u[1] + u[0] * n[1], n[1] * u[2] + u[1] * n[2], n[0] * u[2] + u[0] * n[2]])
    return sig, vel, an


def test_compact_expansion_equals_coefficient_form():
    rng = np.random.default_rng(7)
    for _ in range(200):
        n, s, t = frame(rng)
        rho, vp = rng.uniform(2000, 3000), rng.uniform(2500, 6000)
        vs = vp / rng.uniform(1.5, 2.0)
        mu, lam = rho * vs * vs, rho * vp * vp - 2 * rho * vs * vs
        c, izp, izs = lam / (lam + 2 * mu), 1 / (rho * vp), 1 / (rho * vs)
        ap, as_ = 1 / (lam + 2 * mu), 1 / (2 * mu)
        A = rng.standard_normal(3) * 10.0 ** rng.uniform(-3, 3, 3)
        ref = coefficient_form(n, s, t, c, izp, izs, ap, as_, *A)
        got = compact_form(n, s, t, c, izp, izs, ap, as_, *A)
        for r, g in zip(ref, got):
            assert np.allclose(g, r, rtol=1e-12, atol=1e-12 * np.abs(r).max())


def test_frame_identity_needs_orthonormal_frame():
    """The identity s s^T + t t^T = I - n n^T behind the compact form."""
    rng = np.random.default_rng(8)
    n, s, t = frame(rng)
    assert np.allclose(np.outer(s, s) + np.outer(t, t), np.eye(3) - np.outer(n, n), atol=1e-14)
