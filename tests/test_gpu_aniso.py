"""The anisotropic solve on the GPU (lsb_set_anisotropic) against the anisotropic oracle and
against the isotropic solver for isotropic stiffnesses."""

import numpy as np
import pytest

from tests.aniso_materials import two_phase_field

pytestmark = pytest.mark.gpu


def relmax(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


EB = np.array([1e-3, -4e-4, 2e-4, 3e-4, -1e-4, 2e-4])


@pytest.mark.parametrize("n", [(12, 10, 8), (32, 16, 16)])
@pytest.mark.parametrize("depth", [0, 3])
def test_fixed_iterations_match_oracle_fp64(n, depth):
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.solver.anisotropic import lippmann_schwinger_anisotropic
    from oracle import aniso_oracle as A
    from oracle import ls_oracle as O

    c = two_phase_field(n, seed=sum(n))
    ext = (1.0, 0.8, 0.7)
    e, s, it = lippmann_schwinger_anisotropic(c, EB, GridSpec(*n, *ext), rtol=0.0, atol=0.0,
                                              depth=depth, maxiter=20, dtype=np.float64)
    assert it == 20
    e64, s64, _ = A.lippmann_schwinger(c, EB, O.Grid(*n, *ext), rtol=0.0, atol=0.0, depth=depth,
                                       maxiter=20)
    assert relmax(e, e64) < 1e-10
    assert relmax(s, s64) < 1e-10


@pytest.mark.parametrize("n", [(12, 10, 8), (32, 16, 16), (48, 96, 32)])
def test_fp32_matches_oracle(n):
    """FP32 fields (generic passes on the first grid, the compile-time-size passes' anisotropic
    variants on the power-of-two one) after equal updates, and converged to the same
    solution."""
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.solver.anisotropic import lippmann_schwinger_anisotropic
    from oracle import aniso_oracle as A
    from oracle import ls_oracle as O

    c = two_phase_field(n, seed=7)
    g, og = GridSpec(*n, 1.0, 1.0, 1.0), O.Grid(*n, 1.0, 1.0, 1.0)
    e, _, it = lippmann_schwinger_anisotropic(c, EB, g, rtol=0.0, atol=0.0, depth=3, maxiter=15)
    e64, _, _ = A.lippmann_schwinger(c, EB, og, rtol=0.0, atol=0.0, depth=3, maxiter=15)
    assert it == 15
    assert relmax(e, e64) < 2e-5
    e, s, it = lippmann_schwinger_anisotropic(c, EB, g, rtol=1e-6, depth=3, maxiter=500)
    e64, s64, it64 = A.lippmann_schwinger(c, EB, og, rtol=1e-6, depth=3, maxiter=500)
    assert abs(it - it64) <= 2
    assert relmax(s.mean(axis=(1, 2, 3)), s64.mean(axis=(1, 2, 3))) < 1e-5


@pytest.mark.parametrize("n", [(12, 10, 8), (32, 16, 16)])
def test_isotropic_stiffness_equals_isotropic_solver(n):
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.solver import lippmann_schwinger
    from jaxmaterials_b200.solver.anisotropic import (isotropic_stiffness,
                                                      lippmann_schwinger_anisotropic)

    rng = np.random.default_rng(3)
    lm, mu = 1 + rng.uniform(-0.3, 0.3, (2,) + n)
    g = GridSpec(*n, 1.2, 0.8, 0.9)
    lam0 = 0.5 * (lm.min() + lm.max())
    mu0 = 0.5 * (mu.min() + mu.max())
    c0 = isotropic_stiffness(np.array(lam0), np.array(mu0))
    e1, _, it1 = lippmann_schwinger_anisotropic(isotropic_stiffness(lm, mu), EB, g, rtol=1e-8,
                                                depth=3, maxiter=300, dtype=np.float64, c0=c0)
    e2, _, it2 = lippmann_schwinger(lm, mu, EB, g, rtol=1e-8, depth=3, maxiter=300,
                                    dtype=np.float64)
    assert it1 == it2
    assert relmax(e1, e2) < 1e-12


def test_solver_returns_to_the_isotropic_law():
    """A solver that ran an anisotropic solve gives the isotropic results afterwards."""
    import torch

    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.solver import Solver
    from jaxmaterials_b200.solver.anisotropic import lippmann_schwinger_anisotropic

    n = (32, 16, 16)
    g = GridSpec(*n, 1.0, 1.0, 1.0)
    rng = np.random.default_rng(4)
    lm, mu = (1 + rng.uniform(-0.3, 0.3, (2,) + n)).astype(np.float32)
    s = Solver(g, batch=1, depth=3)
    r0 = s.solve(lm, mu, EB, rtol=1e-6, maxiter=300)
    e0 = r0.epsilon.cpu().numpy()
    lippmann_schwinger_anisotropic(two_phase_field(n), EB, g, rtol=1e-6, depth=3, maxiter=300,
                                   solver=s)
    r1 = s.solve(lm, mu, EB, rtol=1e-6, maxiter=300)
    assert np.array_equal(r1.iters, r0.iters)
    assert np.array_equal(r1.epsilon.cpu().numpy(), e0)
    s.close()
    torch.cuda.synchronize()


@pytest.mark.parametrize("n", [(12, 10, 8), (32, 16, 16)])
def test_grouped_structures_equal_separate_solves(n):
    """Two structures x six loads in one batch (instance b reads structure b // 6, each with its
    own C^0) give the same fields as separate solves."""
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.solver.anisotropic import lippmann_schwinger_anisotropic

    g = GridSpec(*n, 1.0, 0.9, 0.8)
    c = np.stack([two_phase_field(n, seed=1), two_phase_field(n, seed=2) * 1.7])
    eb = np.tile(np.eye(6) * 1e-3, (2, 1))
    e, s, it = lippmann_schwinger_anisotropic(c, eb, g, rtol=1e-6, depth=3, maxiter=300)
    for k in range(2):
        e1, s1, it1 = lippmann_schwinger_anisotropic(c[k], np.eye(6) * 1e-3, g, rtol=1e-6,
                                                     depth=3, maxiter=300)
        assert np.array_equal(it[6 * k:6 * k + 6], it1)
        assert np.array_equal(e[6 * k:6 * k + 6], e1)
