"""Pins the CPU oracle (oracle/ls_oracle.py) to the reference.

Two kinds of evidence:
* golden fixtures produced by the reference's own Python solver
  (tests/golden/make_golden.py);
* every known-answer assertion of the reference's test suites
  (tests/test_lippmann_schwinger.py, cuda/src/tests/test_fourier.hh,
  cuda/src/tests/test_lippmann_schwinger.hh), re-run on the oracle at the suites' grid
  sizes.
"""

import numpy as np
import pytest
import scipy.fft as sfft

from oracle import ls_oracle as O
from tests.conftest import reference_material

EXT = (1.2, 0.8, 0.9)
SMALL = {"even": (12, 10, 8), "odd": (11, 9, 7)}
PY_SIZES = {"even": (64, 48, 32), "odd": (57, 43, 37)}      # test_lippmann_schwinger.py:18
CU_SIZES = {"even": (48, 64, 32), "odd": (47, 61, 37)}      # test_*.hh SetUp
CU_EXT = (1.1, 0.9, 0.7)
EPS_BAR = np.array([2.1, 0.9, 0.8, 0.4, 0.9, 0.5])


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max()


@pytest.mark.parametrize("tag,n", [("even", (8, 6, 4)), ("odd", (7, 5, 3))])
def test_xi_matches_reference(golden, tag, n):
    g = O.Grid(*n, *EXT)
    assert rel(O.get_xi(g), golden[f"xi_{tag}"]) < 1e-15
    assert rel(O.get_xizero(g), golden[f"xizero_{tag}"]) < 1e-15


@pytest.mark.parametrize("tag", ["even", "odd"])
def test_gamma_matches_reference(golden, tag):
    g = O.Grid(*SMALL[tag], *EXT)
    tau_hat = np.fft.fftn(golden[f"gamma_tau_{tag}"], axes=(-3, -2, -1))
    out = O.fourier_solve(tau_hat, 0.8, 1.3, O.get_xizero(g))
    assert rel(out, golden[f"gamma_out_{tag}"]) < 1e-14


@pytest.mark.parametrize("tag", ["even", "odd"])
def test_criteria_match_reference(golden, tag):
    g = O.Grid(*SMALL[tag], *EXT)
    sigma = golden[f"crit_sigma_{tag}"]
    assert abs(O.relative_divergence(sigma, g) / golden[f"crit_real_{tag}"] - 1) < 1e-13
    full = O.relative_divergence_fourier(np.fft.fftn(sigma, axes=(-3, -2, -1)), O.get_xi(g), g)
    assert abs(full / golden[f"crit_fourier_{tag}"] - 1) < 1e-13
    half = O.relative_divergence_half(sfft.rfftn(sigma, axes=(-3, -2, -1)),
                                      O.half(O.get_xi(g), g), g)
    assert abs(half / full - 1) < 1e-12


@pytest.mark.parametrize("depth", [0, 2, 4])
@pytest.mark.parametrize("dname", ["f32", "f64"])
@pytest.mark.parametrize("tag", ["even", "odd"])
@pytest.mark.parametrize("spectrum", ["full", "half"])
def test_solver_matches_reference(golden, tag, dname, depth, spectrum):
    g = O.Grid(*SMALL[tag], *EXT)
    dt = np.float32 if dname == "f32" else np.float64
    atol = 1e-5 if dt == np.float32 else 1e-12
    eps, sig, it = O.lippmann_schwinger(golden[f"ls_lambda_{tag}"], golden[f"ls_mu_{tag}"],
                                        EPS_BAR, g, rtol=1e-20, atol=atol, depth=depth,
                                        maxiter=32, dtype=dt, spectrum=spectrum, workers=1)
    key = f"ls_{tag}_{dname}_d{depth}"
    assert it == int(golden[key + "_iter"])
    tol = 2e-6 if dt == np.float32 else 1e-13
    assert rel(eps, golden[key + "_eps"]) < tol
    assert rel(sig, golden[key + "_sigma"]) < tol


@pytest.mark.parametrize("depth", [0, 5])
def test_fibre_ceff_matches_reference(golden, depth):
    g = O.Grid(16, 16, 16, 16.0, 16.0, 16.0)
    lm, mu = golden["fib_lambda"], golden["fib_mu"]
    c = np.zeros((6, 6))
    its = []
    for k in range(6):
        e = np.zeros(6)
        e[k] = 1.0
        eps, sig, it = O.lippmann_schwinger(lm, mu, e, g, rtol=1e-6, atol=1e-20, depth=depth,
                                            maxiter=1000, dtype=np.float64, workers=1)
        c[k] = sig.mean(axis=(1, 2, 3))
        its.append(it)
        if k == 0:
            assert rel(eps, golden[f"fib_d{depth}_eps0"]) < 1e-10
    assert its == list(golden[f"fib_d{depth}_iters"])
    assert np.linalg.norm(c - golden[f"fib_d{depth}_ceff"]) / np.linalg.norm(c) < 1e-10


# ------------------------------------------------ reference assertions, re-run on the oracle
@pytest.mark.parametrize("tag", ["even", "odd"])
def test_relative_convergence(tag):
    """tests/test_lippmann_schwinger.py:50-61"""
    g = O.Grid(*PY_SIZES[tag], *EXT)
    rng = np.random.default_rng(seed=8741823)
    sigma = rng.normal(size=(6,) + g.shape)
    real = O.relative_divergence(sigma, g)
    four = O.relative_divergence_fourier(np.fft.fftn(sigma, axes=(-3, -2, -1)), O.get_xi(g), g)
    assert abs((real - four) / real) < 1e-5


@pytest.mark.parametrize("depth", [0, 2, 4])
@pytest.mark.parametrize("dname", ["f32", "f64"])
@pytest.mark.parametrize("tag", ["even", "odd"])
def test_convergence(golden, tag, dname, depth):
    """tests/test_lippmann_schwinger.py:64-99, plus the iteration count and mean stress
    of the reference run on the same inputs."""
    g = O.Grid(*PY_SIZES[tag], *EXT)
    dt = np.float32 if dname == "f32" else np.float64
    lm, mu = reference_material(g.shape)
    atol = 1.0e-5 if dt == np.float32 else 1.0e-12
    _, sigma, it = O.lippmann_schwinger(lm, mu, EPS_BAR, g, rtol=1e-20, atol=atol, depth=depth,
                                        maxiter=32, dtype=dt)
    rel_div = O.relative_divergence(sigma.astype(np.float64), g)
    if dt == np.float32:
        assert it < 8
    else:
        assert it < {0: 16, 2: 14, 4: 13}[depth]
    assert rel_div < atol
    key = f"big_{tag}_{dname}_d{depth}"
    assert it == int(golden[key + "_iter"])
    mean = sigma.astype(np.float64).mean(axis=(1, 2, 3))
    assert rel(mean, golden[key + "_sigma_mean"]) < (1e-6 if dt == np.float32 else 1e-12)


@pytest.mark.parametrize("tag", ["even", "odd"])
def test_homogeneous_material(tag):
    """cuda/src/tests/test_lippmann_schwinger.hh:104-128: converges in zero iterations."""
    g = O.Grid(*CU_SIZES[tag], *CU_EXT)
    lm = np.full(g.shape, 1.2)
    mu = np.full(g.shape, 1.2)
    eb = np.array([1.0, 0.4, 0.3, 0.1, -0.4, 0.7])
    _, _, it = O.lippmann_schwinger(lm, mu, eb, g, rtol=1e-20, atol=1e-4, maxiter=100)
    assert it == 0


@pytest.mark.parametrize("tag", ["even", "odd"])
def test_div_sigma_zero(tag):
    """cuda/src/tests/test_fourier.hh:267-316: eps = -Gamma^0 tau makes
    sigma = C^0 eps + tau divergence free (lambda0 = 0.8, mu0 = 1.3)."""
    g = O.Grid(*CU_SIZES[tag], *CU_EXT)
    rng = np.random.default_rng(7812481)
    tau = rng.normal(size=(6,) + g.shape)
    eps = sfft.irfftn(O.fourier_solve(sfft.rfftn(tau, axes=(-3, -2, -1)), 0.8, 1.3,
                                      O.half(O.get_xizero(g), g)), s=g.shape, axes=(-3, -2, -1))
    sigma = O.compute_sigma(np.full(g.shape, 0.8), np.full(g.shape, 1.3), eps) + tau
    div = O.backward_divergence(sigma, g)
    tnorm = np.sqrt(np.sum(sigma[:3] ** 2) + 2 * np.sum(sigma[3:] ** 2))
    assert np.sqrt(np.sum(div**2)) / tnorm < 5e-5


@pytest.mark.parametrize("tag", ["even", "odd"])
def test_fourier_divergence_parseval(tag):
    """cuda/src/tests/test_fourier.hh:182-254: |D^- eps| = |xi . eps_hat| / sqrt(N)."""
    g = O.Grid(*CU_SIZES[tag], *CU_EXT)
    rng = np.random.default_rng(11)
    eps = rng.normal(size=(6,) + g.shape)
    real = np.sqrt(np.sum(O.backward_divergence(eps, g) ** 2))
    d = O.divergence_fourier(sfft.rfftn(eps, axes=(-3, -2, -1)), O.half(O.get_xi(g), g))
    w = O.hermitian_weights(g.nz)
    four = np.sqrt(np.sum(np.sum(np.abs(d) ** 2, axis=(0, 1, 2)) * w)) / np.sqrt(g.number_of_voxels)
    assert abs(four - real) / real < 1e-10


@pytest.mark.parametrize("tag", ["even", "odd"])
def test_hermitian_norm(tag):
    """cuda/src/tests/test_fourier.hh:146-178: weighted half-spectrum norm = full norm."""
    g = O.Grid(*CU_SIZES[tag], *CU_EXT)
    rng = np.random.default_rng(3)
    f = rng.normal(size=(6,) + g.shape)
    full = np.sum(np.abs(np.fft.fftn(f, axes=(-3, -2, -1))) ** 2)
    h = sfft.rfftn(f, axes=(-3, -2, -1))
    half = np.sum(np.sum(np.abs(h) ** 2, axis=(0, 1, 2)) * O.hermitian_weights(g.nz))
    assert abs(half / full - 1) < 1e-12


@pytest.mark.parametrize("tag", ["even", "odd"])
def test_cuda_suite_convergence(tag):
    """cuda/src/tests/test_lippmann_schwinger.hh:132-180 with lambda, mu ~ U(0.8, 0.9)."""
    g = O.Grid(*CU_SIZES[tag], *CU_EXT)
    rng = np.random.default_rng(1)
    mu = rng.uniform(0.8, 0.9, size=g.shape)
    lm = rng.uniform(0.8, 0.9, size=g.shape)
    eb = np.array([1.0, 0.4, 0.3, 0.1, -0.4, 0.7])
    _, sigma, it = O.lippmann_schwinger(lm, mu, eb, g, rtol=1e-20, atol=1e-4, maxiter=100)
    div = np.sqrt(np.sum(O.backward_divergence(sigma.astype(np.float64), g) ** 2))
    avg = sigma.astype(np.float64).mean(axis=(1, 2, 3))
    assert it < 10
    assert div / np.sqrt(np.sum(avg[:3] ** 2) + 2 * np.sum(avg[3:] ** 2)) < 1e-2
