"""CPU oracle of the reference's damage extension (TEST INFRASTRUCTURE ONLY: the product
never imports this module).

Restates in NumPy, with the reference's evaluation order:
* ``voigt_to_tensor`` / ``tensor_to_voigt`` (src/jaxmaterials/utilities.py:65-85): Voigt
  components (v0..v5) sit in the tensor as [[v0, v5, v4], [v5, v1, v3], [v4, v3, v2]];
* ``compute_sigma_damaged`` (src/jaxmaterials/solver/lippmann_schwinger.py:36-75): spectral
  split of the strain into tension and compression parts (eigh), stress of each part with
  the trace split at zero, tension part degraded by (1 - d)^2 + k;
* ``compute_strain_energy`` (:78-100): tensile energy 1/2 lambda <tr eps>_+^2 + mu sum
  <eig>_+^2;
* ``elasticity_solve`` (:330-455): the Anderson-accelerated Lippmann-Schwinger iteration of
  ``lippmann_schwinger_jax`` with the damaged stress law (``ls_oracle.lippmann_schwinger``
  with that law);
* ``phase_field_solve`` (:457-547): the polarisation fixed point
  d = F^-1[F[chi] / (A0 + |xi~|^2)], chi = B - (A - A0) d with A = 1/lc^2 + 2H/(gc lc),
  B = 2H/(gc lc), A0 = (min A + max A)/2, stopped when ||chi_new - chi|| / ||chi_new|| <=
  tolerance.
Pinned against the reference's own outputs in tests/golden/reference_damage.npz.
"""

import numpy as np

from . import ls_oracle


def voigt_to_tensor(v):
    row0 = np.stack([v[0], v[5], v[4]], axis=-1)
    row1 = np.stack([v[5], v[1], v[3]], axis=-1)
    row2 = np.stack([v[4], v[3], v[2]], axis=-1)
    return np.stack([row0, row1, row2], axis=-2)


def tensor_to_voigt(t):
    return np.stack([t[..., 0, 0], t[..., 1, 1], t[..., 2, 2], t[..., 1, 2], t[..., 0, 2],
                     t[..., 0, 1]], axis=0)


def compute_sigma_damaged(lmbda, mu, epsilon, d=None, k=1e-12):
    t = voigt_to_tensor(epsilon)
    tr = np.trace(t, axis1=-2, axis2=-1)
    tr_p, tr_m = np.maximum(tr, 0.0), np.minimum(tr, 0.0)
    w, v = np.linalg.eigh(t)
    e_p = tensor_to_voigt(np.einsum("...ia,...a,...ja->...ij", v, np.maximum(w, 0.0), v))
    e_m = tensor_to_voigt(np.einsum("...ia,...a,...ja->...ij", v, np.minimum(w, 0.0), v))
    one = np.ones_like(tr_p)
    zero = np.zeros_like(tr_p)
    ident = np.stack([one, one, one, zero, zero, zero], axis=0)
    s_p = lmbda * tr_p * ident + 2.0 * mu * e_p
    s_m = lmbda * tr_m * ident + 2.0 * mu * e_m
    if d is not None:
        return ((1.0 - d) ** 2 + k) * s_p + s_m
    return s_p + s_m


def compute_strain_energy(lmbda, mu, epsilon):
    t = voigt_to_tensor(epsilon)
    tr_p = np.maximum(np.trace(t, axis1=-2, axis2=-1), 0.0)
    w = np.maximum(np.linalg.eigvalsh(t), 0.0)
    return 0.5 * lmbda * tr_p ** 2 + mu * np.sum(w ** 2, axis=-1)


def elasticity_solve(lmbda, mu, epsilon_bar, dvar, kk, grid, rtol=1e-6, atol=1e-20, depth=0,
                     maxiter=32, dtype=np.float64, history=None, spectrum="full"):
    """Returns (epsilon, sigma, iterations) like the reference."""
    def law(lm, m, e):
        return compute_sigma_damaged(lm, m, e, dvar, kk).astype(e.dtype)

    return ls_oracle.lippmann_schwinger(lmbda, mu, epsilon_bar, grid, rtol=rtol, atol=atol,
                                        depth=depth, maxiter=maxiter, dtype=dtype,
                                        spectrum=spectrum, history=history, stress=law)


def phase_field_solve(hh, d_old, gc, lc, grid, tolerance=1e-6, maxiter=1000, dtype=np.float64):
    """Returns (d, iterations) like the reference."""
    hh = np.asarray(hh, dtype=dtype)
    a = 1.0 / (lc ** 2) + 2.0 * hh / (gc * lc)
    b = 2.0 * hh / (gc * lc)
    a0 = 0.5 * (np.min(a) + np.max(a))
    xi = ls_oracle.get_xi(grid, dtype=dtype)
    xixi = xi[0] ** 2 + xi[1] ** 2 + xi[2] ** 2
    d = np.asarray(d_old, dtype=dtype)
    chi = b - (a - a0) * d
    residual, it = 1.0, 0
    while residual > tolerance and it < maxiter:
        d = np.real(np.fft.ifftn(np.fft.fftn(chi) / (a0 + xixi)))
        chi_new = b - (a - a0) * d
        nrm = np.linalg.norm(chi_new)
        residual = np.linalg.norm(chi_new - chi) / nrm if nrm > 1e-12 else 0.0
        chi = chi_new
        it += 1
    return d, it
