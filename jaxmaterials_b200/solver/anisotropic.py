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


def two_phase_stiffness(n, seed=0):
    """A seeded two-phase anisotropic field on an n^3 grid: each phase an isotropic tensor
    plus a fibre term beta a(x)a(x)a(x)a along its own random direction a (the stiffer phase
    at 35% of the voxels, in random voxels)."""
    rng = np.random.default_rng(seed)

    def tensor(lmbda, mu, beta, a):
        a = a / np.linalg.norm(a)
        d = np.eye(3)
        return (lmbda * np.einsum("ij,kl->ijkl", d, d)
                + mu * (np.einsum("ik,jl->ijkl", d, d) + np.einsum("il,jk->ijkl", d, d))
                + beta * np.einsum("i,j,k,l->ijkl", a, a, a, a))

    voigt = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))

    def c21(c4):
        return np.array([c4[voigt[p][0], voigt[p][1], voigt[q][0], voigt[q][1]]
                         for p, q in C21_PAIRS])

    m = c21(tensor(1.2, 0.8, 0.6, rng.normal(size=3)))
    f = c21(tensor(3.0, 2.5, 9.0, rng.normal(size=3)))
    mask = rng.uniform(size=(n, n, n)) < 0.35
    return np.where(mask[None], f[:, None, None, None], m[:, None, None, None]).astype(np.float32)


def benchmark(n=128, depth=5, seed=0):
    """C_eff of a two-phase anisotropic n^3 field: the six unit loads as one batch (Anderson
    depth ``depth``, rtol 1e-6, mixed precision), fields resident on the device, CUDA events
    on the current stream around the solve."""
    import torch

    from .. import GridSpec

    g = GridSpec(n, n, n, float(n), float(n), float(n))
    c = torch.as_tensor(two_phase_stiffness(n, seed), device="cuda")
    eye = np.eye(6)
    s = Solver(g, batch=6, depth=depth)
    s.set_anisotropic(c)

    def run():
        return s.solve(c[0], c[3], eye, rtol=1e-6, atol=1e-20, maxiter=2000, rule=RULE_JAX,
                       want_sigma=False)

    run()
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    r = run()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    s.set_anisotropic(None)
    s.close()
    iters = r.iters
    return {"grid": [n, n, n], "anderson_depth": depth, "loads": 6, "ms": ms,
            "iters": [int(i) for i in iters], "solves_per_s": 6 / (ms / 1000.0),
            "voxel_iter_per_s": float(np.sum(iters)) * n ** 3 / (ms / 1000.0),
            "ms_per_iteration": ms / max(int(np.max(iters)), 1),
            "c_eff_diag": [float(r.mean_sigma[k, k]) for k in range(6)]}


def main(argv=None):
    """``python -m jaxmaterials_b200.solver.anisotropic [--n 128]``: timing of the C_eff of a
    two-phase anisotropic field as one JSON line."""
    import argparse
    import json

    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, default=128)
    a = p.parse_args(argv)
    print(json.dumps(benchmark(a.n)))


if __name__ == "__main__":
    main()
