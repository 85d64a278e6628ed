"""NumPy/SciPy restatement of the reference Lippmann-Schwinger solver.

TEST INFRASTRUCTURE ONLY. This module is the checker for the CUDA path in
``jaxmaterials_b200``; it is imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` and by nothing in the product.

Every function follows a function of the reference (yang-chen-2022/JaxMaterials)
and cites the file:line it restates:

* ``src/jaxmaterials/solver/lippmann_schwinger.py`` -- stress, criteria, solver loop
  with Anderson acceleration (``lippmann_schwinger_jax``);
* ``src/jaxmaterials/solver/fourier.py`` -- modified wave vectors and Gamma^0;
* ``src/jaxmaterials/solver/derivatives.py`` -- real-space backward divergence;
* ``cuda/src/fourier.cu`` -- Hermitian weights of the half-spectrum norm;
* ``src/jaxmaterials/data/data.py`` -- C_eff assembly from six unit loads.

One function restates a published scheme instead of the reference's:
``conjugate_gradient`` (Zeman et al. 2010) solves the same equation with the reference's
Gamma^0, criterion and stopping rule; it is the checker for a conjugate-gradient solver
mode.

Pinned against the reference itself: ``tests/golden/make_golden.py`` runs the
reference's Python solver on seeded inputs and stores its outputs, and
``tests/test_oracle.py`` checks this module against those fixtures and against every
known-answer assertion of the reference's own test suites.

Conventions: Voigt order (xx, yy, zz, xy, xz, yz) with tensor (not engineering) shear
entries; fields are arrays of shape (6, nx, ny, nz) with z fastest.
"""

from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np
import scipy.fft as sfft

VOIGT_WEIGHTS = np.array([1.0, 1.0, 1.0, 2.0, 2.0, 2.0])


@dataclass(frozen=True)
class Grid:
    """Periodic grid with nx x ny x nz voxels on a Lx x Ly x Lz box
    (``src/jaxmaterials/common.py:6-29``, ``cuda/src/common.hh:73-91``)."""

    nx: int
    ny: int
    nz: int
    Lx: float
    Ly: float
    Lz: float

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)

    @property
    def number_of_voxels(self):
        return self.nx * self.ny * self.nz


def _workers(workers):
    return os.cpu_count() if workers is None else workers


# ------------------------------------------------------------------ Fourier vectors
def get_xi(grid, dtype=np.float64):
    """Modified wave vectors tilde(xi) on the full spectrum, computed in FP64 and cast
    (``src/jaxmaterials/solver/fourier.py:9-58``)::

        tilde(xi)_0 = 2 nx/Lx sin(xi_0/2) cos(xi_1/2) cos(xi_2/2),  xi_d = 2 pi k_d / N_d

    with unsigned k_d in [0, N_d)."""
    k = [2 * np.pi * np.arange(n) / n for n in (grid.nx, grid.ny, grid.nz)]
    x = np.meshgrid(*k, indexing="ij")
    xi = np.stack(
        [
            2 * grid.nx / grid.Lx * np.sin(x[0] / 2) * np.cos(x[1] / 2) * np.cos(x[2] / 2),
            2 * grid.ny / grid.Ly * np.cos(x[0] / 2) * np.sin(x[1] / 2) * np.cos(x[2] / 2),
            2 * grid.nz / grid.Lz * np.cos(x[0] / 2) * np.cos(x[1] / 2) * np.sin(x[2] / 2),
        ]
    )
    return xi.astype(dtype)


def get_xizero(grid, dtype=np.float64):
    """Normalised wave vectors xi/|xi| in FP64 with norms below 1e-12 replaced by 1
    (``src/jaxmaterials/solver/fourier.py:61-85``)."""
    xi = get_xi(grid, dtype=np.float64)
    nrm = np.linalg.norm(xi, axis=0)
    nrm[nrm < 1.0e-12] = 1.0
    return (xi / nrm).astype(dtype)


def get_xizero_cuda32(grid, dtype=np.float32):
    """Normalised wave vectors as the reference CUDA library builds them: FP32 sin/cos of
    pi k/N, FP32 norm, norms below 1e-6 replaced by 1 (``cuda/src/fourier.cu:47-77``).
    On even grids the modes with two Nyquist indices get |xi| ~ 1e-5 from FP32 round-off
    and pass this guard, so the reference CUDA applies a nonzero Gamma^0 there, unlike
    the Python path (``get_xizero``)."""
    # xi_d / 2 = M_PI * k / N evaluated in double and stored as float
    h = [(np.pi * np.arange(m) / m).astype(np.float32) for m in grid.shape]
    x = np.meshgrid(*h, indexing="ij")
    s = [np.sin(v).astype(np.float32) for v in x]
    c = [np.cos(v).astype(np.float32) for v in x]
    sc = [np.float32(2 * n) / np.float32(ln)
          for n, ln in zip(grid.shape, (grid.Lx, grid.Ly, grid.Lz))]
    t = [sc[0] * s[0] * c[1] * c[2], sc[1] * c[0] * s[1] * c[2], sc[2] * c[0] * c[1] * s[2]]
    nrm = np.sqrt(t[0] ** 2 + t[1] ** 2 + t[2] ** 2).astype(np.float32)
    nrm[nrm < 1.0e-6] = 1.0
    return np.stack([v / nrm for v in t]).astype(dtype)


def half(a, grid):
    """Restrict a full-spectrum array to the R2C half spectrum k_z in [0, nz/2]."""
    return a[..., : grid.nz // 2 + 1]


def hermitian_weights(nz, dtype=np.float64):
    """Weights that turn a half-spectrum sum into the full-spectrum sum: 1 at k_z = 0
    and, for even nz, at k_z = nz/2; 2 elsewhere (``cuda/src/fourier.cu:155-159``)."""
    w = np.full(nz // 2 + 1, 2.0, dtype=dtype)
    w[0] = 1.0
    if nz % 2 == 0:
        w[nz // 2] = 1.0
    return w


# ------------------------------------------------------------------ Green operator
def fourier_solve(tau_hat, lmbda0, mu0, xizero):
    """r_hat = -Gamma^0 : tau_hat for the isotropic reference medium (lambda0, mu0)
    (``src/jaxmaterials/solver/fourier.py:115-186``)."""
    x0, x1, x2 = xizero[0], xizero[1], xizero[2]
    t = tau_hat
    eps_a = np.stack(
        [
            x0**2 * t[0] + x0 * (x2 * t[4] + x1 * t[3]),
            x1**2 * t[1] + x1 * (x2 * t[5] + x0 * t[3]),
            x2**2 * t[2] + x2 * (x1 * t[5] + x0 * t[4]),
            0.5 * (x0 * x1 * (t[0] + t[1]) + (x0**2 + x1**2) * t[3] + x2 * (x0 * t[5] + x1 * t[4])),
            0.5 * (x0 * x2 * (t[0] + t[2]) + (x0**2 + x2**2) * t[4] + x1 * (x0 * t[5] + x2 * t[3])),
            0.5 * (x1 * x2 * (t[1] + t[2]) + (x1**2 + x2**2) * t[5] + x0 * (x1 * t[4] + x2 * t[3])),
        ]
    )
    xi_xi = np.stack([x0**2, x1**2, x2**2, x0 * x1, x0 * x2, x1 * x2])
    xi_dot_tau = (
        x0**2 * t[0]
        + x1**2 * t[1]
        + x2**2 * t[2]
        + 2 * (x0 * x1 * t[3] + x0 * x2 * t[4] + x1 * x2 * t[5])
    )
    return 1 / mu0 * (-eps_a + (lmbda0 + mu0) / (lmbda0 + 2 * mu0) * xi_xi * xi_dot_tau)


# ------------------------------------------------------------------ pointwise law
def compute_sigma(lmbda, mu, epsilon):
    """sigma = lambda tr(eps) I + 2 mu eps in Voigt form
    (``src/jaxmaterials/solver/lippmann_schwinger.py:20-33``)."""
    tr = epsilon[0] + epsilon[1] + epsilon[2]
    zero = np.zeros(epsilon.shape[-3:], dtype=epsilon.dtype)
    return 2 * mu * epsilon + lmbda * np.stack(3 * [tr] + 3 * [zero])


# ------------------------------------------------------------------ derivatives
def backward_derivative(g, grid, direction):
    """8-point backward difference D^- on the staggered grid, periodic
    (``src/jaxmaterials/solver/derivatives.py:8-63``)."""
    r = np.roll
    if direction == 0:
        s = 0.25 * grid.nx / grid.Lx
        d = (g + r(g, 1, axis=-2) + r(g, 1, axis=-1) + r(g, (1, 1), axis=(-2, -1))
             - r(g, 1, axis=-3) - r(g, (1, 1), axis=(-3, -2)) - r(g, (1, 1), axis=(-3, -1))
             - r(g, (1, 1, 1), axis=(-3, -2, -1)))
    elif direction == 1:
        s = 0.25 * grid.ny / grid.Ly
        d = (g + r(g, 1, axis=-3) + r(g, 1, axis=-1) + r(g, (1, 1), axis=(-3, -1))
             - r(g, 1, axis=-2) - r(g, (1, 1), axis=(-3, -2)) - r(g, (1, 1), axis=(-2, -1))
             - r(g, (1, 1, 1), axis=(-3, -2, -1)))
    else:
        s = 0.25 * grid.nz / grid.Lz
        d = (g + r(g, 1, axis=-3) + r(g, 1, axis=-2) + r(g, (1, 1), axis=(-3, -2))
             - r(g, 1, axis=-1) - r(g, (1, 1), axis=(-3, -1)) - r(g, (1, 1), axis=(-2, -1))
             - r(g, (1, 1, 1), axis=(-3, -2, -1)))
    return s * d


def backward_divergence(sigma, grid):
    """Discrete divergence D^-_j sigma_ij of a Voigt tensor field
    (``src/jaxmaterials/solver/derivatives.py:66-95``)."""
    bd = backward_derivative
    return np.stack(
        [
            bd(sigma[0], grid, 0) + bd(sigma[3], grid, 1) + bd(sigma[4], grid, 2),
            bd(sigma[3], grid, 0) + bd(sigma[1], grid, 1) + bd(sigma[5], grid, 2),
            bd(sigma[4], grid, 0) + bd(sigma[5], grid, 1) + bd(sigma[2], grid, 2),
        ]
    )


# ------------------------------------------------------------------ criteria
def relative_divergence(sigma, grid):
    """|D^- sigma| / (sqrt(N) |<sigma>|_w), shear entries weighted x2 in the norm
    (``src/jaxmaterials/solver/lippmann_schwinger.py:103-115``)."""
    ds = backward_divergence(sigma, grid)
    ds_nrm = np.sqrt(np.sum(ds**2))
    avg = np.mean(sigma, axis=(1, 2, 3))
    avg_nrm = np.sqrt(np.sum(avg[:3] ** 2) + 2 * np.sum(avg[3:] ** 2))
    return ds_nrm / (np.sqrt(grid.number_of_voxels) * avg_nrm)


def divergence_fourier(sigma_hat, xi):
    """xi . sigma_hat, the Fourier-space divergence
    (``src/jaxmaterials/solver/lippmann_schwinger.py:125-137``,
    ``cuda/src/fourier.cu:206-249``)."""
    s = sigma_hat
    return np.stack(
        [
            xi[0] * s[0] + xi[1] * s[3] + xi[2] * s[4],
            xi[0] * s[3] + xi[1] * s[1] + xi[2] * s[5],
            xi[0] * s[4] + xi[1] * s[5] + xi[2] * s[2],
        ]
    )


def relative_divergence_fourier(sigma_hat, xi, grid):
    """Fourier form of the criterion on the FULL spectrum
    (``src/jaxmaterials/solver/lippmann_schwinger.py:118-143``)."""
    ds = divergence_fourier(sigma_hat, xi)
    ds_nrm = np.sqrt(np.sum(np.abs(ds) ** 2))
    s0 = np.real(sigma_hat[:, 0, 0, 0])
    s0_nrm = np.sqrt(np.sum(s0[:3] ** 2) + 2 * np.sum(s0[3:] ** 2))
    return ds_nrm / s0_nrm


def relative_divergence_half(sigma_hat_half, xi_half, grid, accum=np.float64):
    """Same criterion on the R2C half spectrum with Hermitian weights
    (``cuda/src/fourier.cu:140-203`` for the weighted norm and
    ``cuda/src/lippmann_schwinger.cu:95-109`` with ``cuda/src/common.cc:48-59`` for
    the zero mode)."""
    ds = divergence_fourier(sigma_hat_half, xi_half)
    w = hermitian_weights(grid.nz, dtype=accum)
    ds_nrm2 = np.sum(np.sum(np.abs(ds).astype(accum) ** 2, axis=(0, 1, 2)) * w)
    s0 = sigma_hat_half[:, 0, 0, 0].astype(np.complex128)
    s0_nrm2 = np.sum(np.abs(s0[:3]) ** 2) + 2 * np.sum(np.abs(s0[3:]) ** 2)
    return float(np.sqrt(ds_nrm2) / np.sqrt(s0_nrm2))


# ------------------------------------------------------------------ solver
def lame_reference(lmbda, mu):
    """Reference medium: half of (min + max) of each Lame field, in the field dtype
    (``src/jaxmaterials/solver/lippmann_schwinger.py:171-172``,
    ``cuda/src/lippmann_schwinger.cu:172-173``)."""
    mu0 = 0.5 * (np.min(mu) + np.max(mu))
    lmbda0 = 0.5 * (np.min(lmbda) + np.max(lmbda))
    return lmbda0, mu0


def lippmann_schwinger(lmbda, mu, epsilon_bar, grid, rtol=1e-6, atol=1e-20, depth=0,
                       maxiter=32, dtype=np.float32, spectrum="half", workers=None,
                       epsilon0=None, history=None, xizero_fn=None, stress=None, gamma=None):
    """Moulinec-Suquet fixed point with Anderson acceleration of depth ``depth``
    (``src/jaxmaterials/solver/lippmann_schwinger.py:146-265``).

    ``spectrum="full"`` uses complex FFTs over the full spectrum exactly as the reference;
    ``spectrum="half"`` uses R2C/C2R transforms (same fixed point, half the work).
    ``epsilon0`` optionally replaces the cold start eps = epsilon_bar by a warm start.
    ``history``, if a list, receives the criterion value after every evaluation.
    ``xizero_fn(grid, dtype)`` replaces ``get_xizero`` (e.g. ``get_xizero_cuda32`` for
    the reference CUDA library's construction). ``stress(lmbda, mu, eps)`` replaces the
    linear law (the damage extension's ``elasticity_solve``, lippmann_schwinger.py:330-455);
    ``gamma(sigma_hat, xizero)`` replaces the isotropic Gamma^0 (the anisotropic extension).

    Returns ``(epsilon, sigma, iterations)`` with sigma = sigma(epsilon); the loop stops
    when e <= atol or e <= rtol * e0 (e0 at the first iterate) or after maxiter updates.
    """
    w = _workers(workers)
    shape = grid.shape
    axes = (-3, -2, -1)
    lmbda = np.asarray(lmbda, dtype=dtype)
    mu = np.asarray(mu, dtype=dtype)
    lmbda0, mu0 = lame_reference(lmbda, mu)
    xizero = (xizero_fn or get_xizero)(grid, dtype=dtype)
    xi = get_xi(grid, dtype=dtype)
    if spectrum == "half":
        xizero = half(xizero, grid)
        xi = half(xi, grid)

        def fwd(f):
            return sfft.rfftn(f, axes=axes, workers=w)

        def inv(fh):
            return sfft.irfftn(fh, s=shape, axes=axes, workers=w)

        def crit(sh):
            return relative_divergence_half(sh, xi, grid)
    else:

        def fwd(f):
            return sfft.fftn(f, axes=axes, workers=w)

        def inv(fh):
            return np.real(sfft.ifftn(fh, axes=axes, workers=w))

        def crit(sh):
            return float(relative_divergence_fourier(sh, xi, grid))

    eps = np.zeros((depth + 1, 6) + shape, dtype=dtype)
    if epsilon0 is None:
        eps[0] = np.asarray(epsilon_bar, dtype=dtype)[:, None, None, None]
    else:
        eps[0] = np.asarray(epsilon0, dtype=dtype)
    res = np.zeros((depth + 1, 6) + shape, dtype=dtype)
    a_mat = np.eye(depth + 1, dtype=dtype)
    u_rhs = np.zeros(depth + 1, dtype=dtype)
    law = stress or compute_sigma
    sigma = law(lmbda, mu, eps[0])
    sigma_hat = fwd(sigma)
    e = crit(sigma_hat)
    e0 = e
    if history is not None:
        history.append(e)
    it = 0
    scale = np.array([1.0, 1.0, 1.0, 2.0, 2.0, 2.0], dtype=dtype)
    while e > atol and e > rtol * e0 and it < maxiter:
        r_hat = (gamma(sigma_hat, xizero) if gamma is not None
                 else fourier_solve(sigma_hat, lmbda0, mu0, xizero))
        r = np.asarray(inv(r_hat), dtype=dtype)
        res = np.roll(res, 1, axis=0)
        res[0] = r
        a_mat = np.roll(a_mat, (1, 1), axis=(0, 1))
        a_mat[0, :] = np.einsum("aijk,saijk,a->s", r, res, scale)
        a_mat[:, 0] = a_mat[0, :]
        u_rhs = np.roll(u_rhs, 1)
        u_rhs[0] = 1
        v = np.linalg.solve(a_mat, u_rhs)
        alpha = (v / np.dot(v, u_rhs)).astype(dtype)
        eps_new = np.einsum("s,saijk", alpha, eps + res).astype(dtype)
        eps = np.roll(eps, 1, axis=0)
        eps[0] = eps_new
        sigma = law(lmbda, mu, eps[0])
        sigma_hat = fwd(sigma)
        e = crit(sigma_hat)
        if history is not None:
            history.append(e)
        it += 1
    return eps[0], sigma, it


def conjugate_gradient(lmbda, mu, epsilon_bar, grid, rtol=1e-6, atol=1e-20, maxiter=1000,
                       dtype=np.float64, workers=None, history=None, restart=0, stress=None):
    """Conjugate gradients on the Lippmann-Schwinger equation (J. Zeman, J. Vondrejc,
    J. Novak, I. Marek, J. Comput. Phys. 229 (2010) 8065-8071).

    The strain is eps = eps_bar + x with x a compatible zero-mean field solving
    G[C : x] = -G[C : eps_bar], where G is the projection onto compatible zero-mean strains
    (the Gamma^0 of ``fourier_solve`` for the reference medium lambda0 = 0, mu0 = 1/2, i.e.
    C0 the identity). On compatible fields G C is symmetric positive definite in the inner
    product sum_ij a_ij b_ij (Voigt weights 1, 1, 1, 2, 2, 2), so plain CG applies; every
    update costs one stress evaluation and one forward/inverse transform pair, as a
    Moulinec-Suquet update does. Criterion and stop are those of ``lippmann_schwinger``
    (e <= atol or e <= rtol * e0, e0 the criterion of eps_bar; the criterion is evaluated on
    the stress of eps_bar + x after every update). Inner products accumulate in FP64.
    ``restart`` > 0: every ``restart`` updates the recursively updated residual is replaced
    by the true one, -G[C : (eps_bar + x)], and the search direction by it (beta = 0): in
    FP32 fields the recursive residual drifts and plain CG stalls near 2e-6 and then
    diverges, while with this replacement every 20 updates it converges as in FP64.
    ``stress``: a linear law ``stress(lmbda, mu, eps)`` with a symmetric positive definite
    stiffness in place of the isotropic one (as in ``lippmann_schwinger``).
    Returns ``(epsilon, sigma, iterations)``.
    """
    w = _workers(workers)
    shape = grid.shape
    axes = (-3, -2, -1)
    lmbda = np.asarray(lmbda, dtype=dtype)
    mu = np.asarray(mu, dtype=dtype)
    xizero = half(get_xizero(grid, dtype=dtype), grid)
    xi = half(get_xi(grid, dtype=dtype), grid)
    wv = VOIGT_WEIGHTS.astype(dtype)[:, None, None, None]
    law = stress or compute_sigma

    def project(tau):
        tau_hat = sfft.rfftn(tau, axes=axes, workers=w)
        return -np.asarray(sfft.irfftn(fourier_solve(tau_hat, 0.0, 0.5, xizero), s=shape,
                                       axes=axes, workers=w), dtype=dtype)

    def dot(a, b):
        return float(np.sum(a * b * wv, dtype=np.float64))

    def crit(sig):
        return relative_divergence_half(sfft.rfftn(sig, axes=axes, workers=w), xi, grid)

    eb = np.broadcast_to(np.asarray(epsilon_bar, dtype=dtype)[:, None, None, None], (6,) + shape)
    x = np.zeros((6,) + shape, dtype=dtype)
    sigma = law(lmbda, mu, eb)
    e = crit(sigma)
    e0 = e
    if history is not None:
        history.append(e)
    r = -project(sigma)
    p = r.copy()
    rr = dot(r, r)
    it = 0
    while e > atol and e > rtol * e0 and it < maxiter:
        q = project(law(lmbda, mu, p))
        alpha = dtype(rr / dot(p, q))
        x += alpha * p
        r -= alpha * q
        sigma = law(lmbda, mu, eb + x)
        e = crit(sigma)
        if history is not None:
            history.append(e)
        it += 1
        if restart and it % restart == 0:
            r = -project(sigma)
            p = r.copy()
            rr = dot(r, r)
        else:
            rr_new = dot(r, r)
            p = r + dtype(rr_new / rr) * p
            rr = rr_new
    return eb + x, sigma, it


def c_eff(lmbda, mu, grid, rtol=1e-6, atol=1e-20, depth=0, maxiter=1000,
          dtype=np.float64, workers=None):
    """Effective stiffness from six unit macroscopic strains: row k is the mean stress
    for eps_bar = e_k (``src/jaxmaterials/data/data.py:178-186``). Shear entries are
    tensor strains, so C[3,3] = 2 mu_eff for an isotropic medium.

    Returns ``(C, iterations)`` with C of shape (6, 6)."""
    c = np.zeros((6, 6))
    its = []
    for k in range(6):
        e = np.zeros(6)
        e[k] = 1.0
        _, sigma, it = lippmann_schwinger(lmbda, mu, e, grid, rtol=rtol, atol=atol,
                                          depth=depth, maxiter=maxiter, dtype=dtype,
                                          workers=workers)
        c[k] = np.mean(sigma.astype(np.float64), axis=(1, 2, 3))
        its.append(it)
    return c, its
