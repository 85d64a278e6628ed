"""Anisotropic linear elasticity: the Lippmann-Schwinger solve with a general stiffness
(21 independent entries per voxel) and the Gamma^0 operator of an anisotropic reference
medium, as derived in the reference's doc/linear_elasticity.tex:372-402 and
doc/anisotropic.py (the reference itself has no solver for this case).

Entry numbering (doc/anisotropic.py:150-185): C_0..C_5 the diagonal of the 6 x 6 Voigt
matrix, then (0,1), (0,2), (1,2), (0,3), (0,4), (0,5), (1,3), (1,4), (1,5), (2,3), (2,4),
(2,5), (3,4), (3,5), (4,5); Voigt order (xx, yy, zz, xy, xz, yz), tensor shear strains:
sigma_a = sum_b C_ab w_b eps_b with w = (1, 1, 1, 2, 2, 2). Runs on the GPU through
``lsb_set_anisotropic`` (generic passes).
"""

import numpy as np

from .lippmann_schwinger import RULE_JAX, Solver

__all__ = ["isotropic_stiffness", "lippmann_schwinger_anisotropic", "C21_PAIRS"]

C21_PAIRS = ((0, 0), (1, 1), (2, 2), (3, 3), (4, 4), (5, 5), (0, 1), (0, 2), (1, 2), (0, 3),
             (0, 4), (0, 5), (1, 3), (1, 4), (1, 5), (2, 3), (2, 4), (2, 5), (3, 4), (3, 5),
             (4, 5))


def isotropic_stiffness(lmbda, mu):
    """Entries of the isotropic stiffness of Lame fields (doc/linear_elasticity.tex:381-387):
    C_0..2 = lambda + 2 mu, C_3..5 = mu, C_6..8 = lambda, the rest 0; shape (21,) + shape of
    the fields."""
    lmbda = np.asarray(lmbda, dtype=np.float64)
    mu = np.asarray(mu, dtype=np.float64)
    c = np.zeros((21,) + lmbda.shape)
    c[0:3] = lmbda + 2 * mu
    c[3:6] = mu
    c[6:9] = lmbda
    return c


def lippmann_schwinger_anisotropic(stiffness, epsilon_bar, grid_spec, rtol=1e-6, atol=1e-20,
                                   depth=0, maxiter=32, dtype=np.float32, c0=None, rule=RULE_JAX,
                                   solver=None):
    """Fixed point of the anisotropic problem for every row of ``epsilon_bar`` ((B, 6) or
    (6,)); stiffness (21, nx, ny, nz), or (S, 21, nx, ny, nz) with instance b reading
    structure b // (B // S). c0: reference stiffness (21,), default the mid-range of every
    entry. Returns ``(epsilon, sigma, iterations)`` as NumPy arrays ((6, ...) and an int for
    a single row)."""
    import torch

    eb = np.atleast_2d(np.asarray(epsilon_bar, dtype=np.float64))
    f64 = np.dtype(dtype) == np.float64
    tdt = torch.float64 if f64 else torch.float32
    g = grid_spec
    c = torch.as_tensor(stiffness, dtype=tdt, device="cuda").contiguous()
    s = solver or Solver(g, batch=eb.shape[0], depth=depth)
    try:
        s.set_anisotropic(c, c0, np.float64 if f64 else np.float32)
        # the Lame arguments do not enter the law; two stiffness entries serve as arrays of
        # the right layout
        lam = c[0] if c.dim() == 4 else c[:, 0].contiguous()
        mu = c[3] if c.dim() == 4 else c[:, 3].contiguous()
        r = s.solve(lam, mu, eb, rtol=rtol, atol=atol, maxiter=maxiter, rule=rule,
                    want_sigma=True, dtype=np.float64 if f64 else np.float32)
    finally:
        s.set_anisotropic(None)
        if solver is None:
            s.close()
    eps, sig = r.epsilon.cpu().numpy(), r.sigma.cpu().numpy()
    if np.ndim(epsilon_bar) == 1:
        return eps[0], sig[0], int(r.iters[0])
    return eps, sig, r.iters.copy()
