"""CPU oracle of the anisotropic extension (TEST INFRASTRUCTURE ONLY: the product never
imports this module).

Follows the derivation of doc/linear_elasticity.tex:372-402 and doc/anisotropic.py:
21 independent entries of the symmetric 6 x 6 Voigt stiffness numbered as
doc/anisotropic.py:150-185, stress sigma_a = sum_b C_ab w_b eps_b (w = 1, 1, 1, 2, 2, 2),
acoustic matrix K_ki = C^0_kjil xi_j xi_l of the normalised modified wave vector,
Gamma^0 tau = sym(xi (x) K^-1 tau xi) (doc/anisotropic.py:98-128, for an isotropic C^0 equal
to fourier.py:115-186), r = -Gamma^0 tau, zero where xi has no direction. The reference has
no anisotropic solver; it derives these formulas symbolically in doc/anisotropic.py. This
oracle is pinned to that derivation: its stress law, acoustic matrix and Gamma^0 equal the
reference's sympy expressions evaluated in FP64 on seeded stiffnesses and wave vectors
(tests/golden/reference_aniso.npz, made by tests/golden/make_aniso_golden.py), and an
isotropic stiffness reproduces ls_oracle, which is pinned to the reference's solver.
"""

import numpy as np

from . import ls_oracle

C21_PAIRS = ((0, 0), (1, 1), (2, 2), (3, 3), (4, 4), (5, 5), (0, 1), (0, 2), (1, 2), (0, 3),
             (0, 4), (0, 5), (1, 3), (1, 4), (1, 5), (2, 3), (2, 4), (2, 5), (3, 4), (3, 5),
             (4, 5))
VOIGT = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))


def voigt_of(p, q):
    return VOIGT.index(tuple(sorted((p, q))))


def matrix_from_c21(c21):
    """(6, 6, ...) symmetric Voigt matrix from (21, ...) entries."""
    c21 = np.asarray(c21)
    m = np.zeros((6, 6) + c21.shape[1:], dtype=c21.dtype)
    for k, (a, b) in enumerate(C21_PAIRS):
        m[a, b] = c21[k]
        m[b, a] = c21[k]
    return m


def isotropic_c21(lmbda, mu):
    """Entries of an isotropic stiffness: C_0..2 = lambda + 2 mu, C_3..5 = mu, C_6..8 =
    lambda (doc/linear_elasticity.tex:381-387), others 0."""
    lmbda = np.asarray(lmbda)
    c = np.zeros((21,) + lmbda.shape, dtype=np.result_type(lmbda, mu))
    c[0:3] = lmbda + 2 * mu
    c[3:6] = mu
    c[6:9] = lmbda
    return c


def stress(c21, eps):
    m = matrix_from_c21(c21)
    w = np.array([1.0, 1.0, 1.0, 2.0, 2.0, 2.0]).reshape((6,) + (1,) * (eps.ndim - 1))
    return np.einsum("ab...,b...->a...", m, w * eps).astype(eps.dtype)


def acoustic_matrix(c0, xizero):
    """K_ki = C^0_kjil xi_j xi_l (doc/anisotropic.py:46-95) for a constant reference
    stiffness c0 (21,) and wave vectors xizero (3, ...); shape (..., 3, 3)."""
    m = matrix_from_c21(np.asarray(c0, dtype=np.float64))
    c4 = np.zeros((3, 3, 3, 3))
    for p in range(3):
        for q in range(3):
            for r in range(3):
                for s in range(3):
                    c4[p, q, r, s] = m[voigt_of(p, q), voigt_of(r, s)]
    z = np.asarray(xizero, dtype=np.float64)
    return np.einsum("kjil,j...,l...->...ki", c4, z, z)


def gamma_solve(tau_hat, c0, xizero):
    """r_hat = -Gamma^0 tau_hat for a constant reference stiffness c0 (21,)."""
    z = np.asarray(xizero, dtype=np.float64)
    k = acoustic_matrix(c0, z)
    nrm2 = np.sum(z * z, axis=0)
    ok = nrm2 > 0.5  # unit vectors; the zero mode and guarded modes have |xi| ~ 0
    kk = np.where(ok[..., None, None], k, np.eye(3))
    n = np.linalg.inv(kk)
    t = tau_hat
    tau = np.stack([np.stack([t[0], t[3], t[4]]), np.stack([t[3], t[1], t[5]]),
                    np.stack([t[4], t[5], t[2]])])
    v = np.einsum("kj...,j...->k...", tau, z)
    u = np.einsum("...ki,i...->k...", n, v)
    r = np.stack([-z[0] * u[0], -z[1] * u[1], -z[2] * u[2], -0.5 * (z[0] * u[1] + z[1] * u[0]),
                  -0.5 * (z[0] * u[2] + z[2] * u[0]), -0.5 * (z[1] * u[2] + z[2] * u[1])])
    return np.where(ok, r, 0.0).astype(tau_hat.dtype)


def reference_c0(c21):
    """(min + max) / 2 of every entry over the field."""
    c = np.asarray(c21, dtype=np.float64).reshape(21, -1)
    return 0.5 * (c.min(axis=1) + c.max(axis=1))


def lippmann_schwinger(c21, epsilon_bar, grid, rtol=1e-6, atol=1e-20, depth=0, maxiter=32,
                       dtype=np.float64, c0=None, spectrum="half"):
    """The Anderson-accelerated fixed point with the anisotropic law and Gamma^0; returns
    (epsilon, sigma, iterations)."""
    c21 = np.asarray(c21, dtype=dtype)
    c0 = reference_c0(c21) if c0 is None else np.asarray(c0, dtype=np.float64)
    dummy = np.ones(grid.shape, dtype=dtype)
    return ls_oracle.lippmann_schwinger(
        dummy, dummy, epsilon_bar, grid, rtol=rtol, atol=atol, depth=depth, maxiter=maxiter,
        dtype=dtype, spectrum=spectrum, stress=lambda lm, m, e: stress(c21, e),
        gamma=lambda sh, xz: gamma_solve(sh, c0, xz))
