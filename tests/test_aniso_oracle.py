"""The anisotropic oracle (oracle/aniso_oracle.py): its stress law, acoustic matrix and
Gamma^0 equal the reference's own symbolic derivation (doc/anisotropic.py, evaluated by
tests/golden/make_aniso_golden.py into tests/golden/reference_aniso.npz); it reduces to
the pinned isotropic oracle for isotropic stiffnesses, and its Gamma^0 has the defining
properties of the Green operator of the reference medium (no GPU)."""

import os

import numpy as np
import pytest

from tests.conftest import ROOT

from tests.aniso_materials import c21_of_tensor, fibre_tensor, two_phase_field


def test_isotropic_reduction():
    from oracle import aniso_oracle as A
    from oracle import ls_oracle as O

    rng = np.random.default_rng(1)
    n = (10, 8, 6)
    g = O.Grid(*n, 1.2, 0.8, 0.9)
    lm, mu = 1 + rng.uniform(-0.2, 0.2, (2,) + n)
    eb = np.array([1e-3, -5e-4, 2e-4, 1e-4, 0.0, 3e-4])
    lam0, mu0 = O.lame_reference(lm, mu)
    c0 = A.isotropic_c21(np.array(lam0), np.array(mu0))
    for depth in (0, 3):
        e1, s1, it1 = A.lippmann_schwinger(A.isotropic_c21(lm, mu), eb, g, rtol=1e-8, depth=depth,
                                           maxiter=200, c0=c0)
        e2, s2, it2 = O.lippmann_schwinger(lm, mu, eb, g, rtol=1e-8, depth=depth, maxiter=200,
                                           dtype=np.float64)
        assert it1 == it2
        assert np.abs(e1 - e2).max() < 1e-13 * np.abs(e2).max()
        assert np.abs(s1 - s2).max() < 1e-13 * np.abs(s2).max()


def test_gamma_is_the_green_operator_of_the_reference_medium():
    """For unit xi: Gamma C0 Gamma = Gamma, and xi . (C0 : Gamma tau - tau) = 0."""
    from oracle import aniso_oracle as A

    rng = np.random.default_rng(2)
    c0 = c21_of_tensor(fibre_tensor(1.5, 0.9, 4.0, rng.normal(size=3)))
    z = rng.normal(size=(3, 50))
    z /= np.linalg.norm(z, axis=0)
    tau = rng.normal(size=(6, 50))
    g_tau = -A.gamma_solve(tau, c0, z)                        # Gamma tau
    c_g = A.stress(np.repeat(c0[:, None], 50, axis=1), g_tau)  # C0 : Gamma tau
    assert np.allclose(-A.gamma_solve(c_g, c0, z), g_tau, rtol=0, atol=1e-12)
    d = c_g - tau
    div = np.stack([d[0] * z[0] + d[3] * z[1] + d[4] * z[2], d[3] * z[0] + d[1] * z[1] + d[5] * z[2],
                    d[4] * z[0] + d[5] * z[1] + d[2] * z[2]])
    assert np.abs(div).max() < 1e-12
    # zero-direction modes give zero
    assert np.array_equal(A.gamma_solve(tau[:, :3], c0, np.zeros((3, 3))), np.zeros((6, 3)))


def test_anisotropic_solve_converges_and_c_eff_is_symmetric():
    from oracle import aniso_oracle as A
    from oracle import ls_oracle as O

    n = (8, 8, 8)
    g = O.Grid(*n, 1.0, 1.0, 1.0)
    c = two_phase_field(n, seed=3)
    rows = []
    for k in range(6):
        eb = np.zeros(6)
        eb[k] = 1.0
        e, s, it = A.lippmann_schwinger(c, eb, g, rtol=1e-9, depth=4, maxiter=400)
        assert it < 400
        rows.append(s.mean(axis=(1, 2, 3)))
    ceff = np.array(rows)  # row k: mean stress for e_k (tensor shear)
    w = np.diag([1, 1, 1, 2, 2, 2])
    b = ceff @ w  # symmetric in the energy pairing
    assert np.abs(b - b.T).max() < 1e-6 * np.abs(b).max()


@pytest.fixture(scope="module")
def aniso_gold():
    with np.load(os.path.join(ROOT, "tests", "golden", "reference_aniso.npz")) as d:
        return {k: d[k] for k in d.files}


def test_stress_law_matches_reference_derivation(aniso_gold):
    from oracle import aniso_oracle as A

    g = aniso_gold
    got = A.stress(g["c21"].T, g["eps"].T).T
    assert np.abs(got - g["sigma"]).max() < 1e-13 * np.abs(g["sigma"]).max()


def test_acoustic_matrix_matches_reference_derivation(aniso_gold):
    from oracle import aniso_oracle as A

    g = aniso_gold
    for s in range(g["c0"].shape[0]):
        k = A.acoustic_matrix(g["c0"][s], g["xi"][s])
        assert np.abs(k - g["K"][s]).max() < 1e-13 * np.abs(g["K"][s]).max()


def test_gamma_matches_reference_derivation(aniso_gold):
    """Column b of Gamma^0 (Voigt pairs, the reference's Gamma^0_klij) is -r for
    tau = e_b / w_b, since (Gamma^0 tau)_a = sum_b Gamma_ab w_b tau_b with tensor shear."""
    from oracle import aniso_oracle as A

    g = aniso_gold
    w = np.array([1.0, 1.0, 1.0, 2.0, 2.0, 2.0])
    for s in range(g["c0"].shape[0]):
        tau = np.diag(1.0 / w)                       # column b: e_b / w_b
        z = np.repeat(g["xi"][s][:, None], 6, axis=1)
        cols = -A.gamma_solve(tau, g["c0"][s], z)    # (6, 6): [a, b]
        assert np.abs(cols - g["gamma"][s]).max() < 1e-12 * np.abs(g["gamma"][s]).max()
