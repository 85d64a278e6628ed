"""Generate the golden fixtures by running the REFERENCE's own Python solver.

Run from the repository root in an environment that holds the reference checkout:

    python tests/golden/make_golden.py <reference checkout>   (or JAXMATERIALS_REF in the environment)

JAX is not installed here, so ``tests/golden/_jaxshim`` provides a NumPy-backed stand-in
for the handful of jax calls the reference solver makes; the reference modules
``src/jaxmaterials/solver/{lippmann_schwinger,fourier,derivatives}.py`` and
``src/jaxmaterials/common.py`` are imported and executed unchanged. The outputs land in
``tests/golden/reference_ls.npz``; the tests read only that file.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def reference_material(shape, seed=784173):
    """Inputs of tests/test_lippmann_schwinger.py:37-47,75: initialise_material returns
    (first draw, second draw) and the test binds them as (lmbda, mu)."""
    rng = np.random.default_rng(seed=seed)
    first = np.ones(shape) + rng.uniform(size=shape, low=-0.2, high=0.2)
    second = np.ones(shape) + rng.uniform(size=shape, low=-0.2, high=0.2)
    return first, second


def main(ref_root):
    sys.path.insert(0, os.path.join(HERE, "_jaxshim"))
    sys.path.insert(0, os.path.join(ref_root, "src"))
    sys.path.insert(0, ROOT)
    from jaxmaterials.common import GridSpec
    from jaxmaterials.solver import fourier as rf
    from jaxmaterials.solver import lippmann_schwinger as rls
    from jaxmaterials_b200.data import fibres

    out = {}
    ext = (1.2, 0.8, 0.9)
    small = {"even": (12, 10, 8), "odd": (11, 9, 7)}

    # Fourier vectors (fourier.py:9-85)
    for tag, n in {"even": (8, 6, 4), "odd": (7, 5, 3)}.items():
        g = GridSpec(*n, *ext)
        out[f"xi_{tag}"] = np.asarray(rf.get_xi(g, dtype=np.float64))
        out[f"xizero_{tag}"] = np.asarray(rf.get_xizero(g, dtype=np.float64))

    # Gamma^0 application (fourier.py:115-186), lambda0 = 0.8, mu0 = 1.3 as in the
    # reference's CUDA Fourier tests
    for tag, n in small.items():
        g = GridSpec(*n, *ext)
        rng = np.random.default_rng(5150)
        tau = rng.normal(size=(6,) + n)
        tau_hat = np.fft.fftn(tau, axes=(-3, -2, -1))
        xz = rf.get_xizero(g, dtype=np.float64)
        out[f"gamma_tau_{tag}"] = tau
        out[f"gamma_out_{tag}"] = np.asarray(rls.fourier_solve(tau_hat, 0.8, 1.3, xz))

    # Criteria on N(0,1) stress, seed of tests/test_lippmann_schwinger.py:55
    for tag, n in small.items():
        g = GridSpec(*n, *ext)
        rng = np.random.default_rng(seed=8741823)
        sigma = rng.normal(size=(6,) + n)
        sh = np.fft.fftn(sigma, axes=(-3, -2, -1))
        out[f"crit_sigma_{tag}"] = sigma
        out[f"crit_real_{tag}"] = np.float64(rls.relative_divergence(sigma, g))
        out[f"crit_fourier_{tag}"] = np.float64(
            rls.relative_divergence_fourier(sh, rf.get_xi(g), g))

    # Solver runs with the inputs of tests/test_lippmann_schwinger.py:31-99
    eps_bar = np.array([2.1, 0.9, 0.8, 0.4, 0.9, 0.5])
    for tag, n in small.items():
        g = GridSpec(*n, *ext)
        lm, mu = reference_material(n)
        out[f"ls_lambda_{tag}"] = lm
        out[f"ls_mu_{tag}"] = mu
        for dt, dname in ((np.float32, "f32"), (np.float64, "f64")):
            atol = 1.0e-5 if dt == np.float32 else 1.0e-12
            for depth in (0, 2, 4):
                eps, sig, it = rls.lippmann_schwinger_jax(
                    np.array(lm, dtype=dt), np.array(mu, dtype=dt), eps_bar, g,
                    rtol=1e-20, atol=atol, depth=depth, maxiter=32, dtype=dt)
                key = f"ls_{tag}_{dname}_d{depth}"
                out[key + "_eps"] = np.asarray(eps)
                out[key + "_sigma"] = np.asarray(sig)
                out[key + "_iter"] = np.int64(it)

    # Same test inputs at the reference suite's own grid sizes: scalars only
    for tag, n in {"even": (64, 48, 32), "odd": (57, 43, 37)}.items():
        g = GridSpec(*n, *ext)
        lm, mu = reference_material(n)
        for dt, dname in ((np.float32, "f32"), (np.float64, "f64")):
            atol = 1.0e-5 if dt == np.float32 else 1.0e-12
            for depth in (0, 2, 4):
                eps, sig, it = rls.lippmann_schwinger_jax(
                    np.array(lm, dtype=dt), np.array(mu, dtype=dt), eps_bar, g,
                    rtol=1e-20, atol=atol, depth=depth, maxiter=32, dtype=dt)
                key = f"big_{tag}_{dname}_d{depth}"
                out[key + "_iter"] = np.int64(it)
                out[key + "_reldiv"] = np.float64(rls.relative_divergence(sig, g))
                out[key + "_sigma_mean"] = np.mean(np.asarray(sig, np.float64), axis=(1, 2, 3))
                out[key + "_eps_mean"] = np.mean(np.asarray(eps, np.float64), axis=(1, 2, 3))

    # High-contrast fibre composite, 16^3, contrast ~26, tol 1e-6, FP64
    st = fibres.generate_layered_fibres(16, 2, 2.0, 0.40, seed=7)
    lm, mu = fibres.lame_fields(st, dtype=np.float64)
    g = GridSpec(16, 16, 16, 16.0, 16.0, 16.0)
    out["fib_lambda"] = lm
    out["fib_mu"] = mu
    for depth in (0, 5):
        c = np.zeros((6, 6))
        its = []
        for k in range(6):
            e = np.zeros(6)
            e[k] = 1.0
            eps, sig, it = rls.lippmann_schwinger_jax(
                lm, mu, e, g, rtol=1e-6, atol=1e-20, depth=depth, maxiter=1000,
                dtype=np.float64)
            c[k] = np.mean(np.asarray(sig), axis=(1, 2, 3))
            its.append(int(it))
            if k == 0:
                out[f"fib_d{depth}_eps0"] = np.asarray(eps)
                out[f"fib_d{depth}_sigma0"] = np.asarray(sig)
        out[f"fib_d{depth}_ceff"] = c
        out[f"fib_d{depth}_iters"] = np.array(its)

    np.savez_compressed(os.path.join(HERE, "reference_ls.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["JAXMATERIALS_REF"])
