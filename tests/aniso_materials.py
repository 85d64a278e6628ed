"""Seeded anisotropic stiffness fields for the anisotropic tests: two phases, each an
isotropic tensor plus a fibre term beta (a (x) a (x) a (x) a) along its own direction a
(positive definite), written as the 21 Voigt entries of jaxmaterials_b200.solver.anisotropic."""

import numpy as np

VOIGT = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))
C21_PAIRS = ((0, 0), (1, 1), (2, 2), (3, 3), (4, 4), (5, 5), (0, 1), (0, 2), (1, 2), (0, 3),
             (0, 4), (0, 5), (1, 3), (1, 4), (1, 5), (2, 3), (2, 4), (2, 5), (3, 4), (3, 5),
             (4, 5))


def fibre_tensor(lmbda, mu, beta, a):
    a = np.asarray(a, dtype=np.float64)
    a = a / np.linalg.norm(a)
    d = np.eye(3)
    c = (lmbda * np.einsum("ij,kl->ijkl", d, d)
         + mu * (np.einsum("ik,jl->ijkl", d, d) + np.einsum("il,jk->ijkl", d, d))
         + beta * np.einsum("i,j,k,l->ijkl", a, a, a, a))
    return c


def c21_of_tensor(c4):
    return np.array([c4[VOIGT[p][0], VOIGT[p][1], VOIGT[q][0], VOIGT[q][1]] for p, q in C21_PAIRS])


def two_phase_field(shape, seed=0):
    rng = np.random.default_rng(seed)
    m = c21_of_tensor(fibre_tensor(1.2, 0.8, 0.6, rng.normal(size=3)))
    f = c21_of_tensor(fibre_tensor(3.0, 2.5, 9.0, rng.normal(size=3)))
    mask = rng.uniform(size=shape) < 0.35
    return np.where(mask[None], f[:, None, None, None], m[:, None, None, None])
