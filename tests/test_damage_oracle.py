"""The damage oracle (oracle/damage_oracle.py) against the reference's own outputs
(tests/golden/reference_damage.npz, made by tests/golden/make_damage_golden.py)."""

import os

import numpy as np
import pytest

from tests.conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_damage.npz")


@pytest.fixture(scope="module")
def gold():
    with np.load(GOLDEN) as d:
        return {k: d[k] for k in d.files}


def grid_of(g):
    from oracle import ls_oracle as O

    return O.Grid(int(g[0]), int(g[1]), int(g[2]), g[3], g[4], g[5])


def test_pointwise_laws(gold):
    from oracle import damage_oracle as D

    e, lm, mu, d = gold["pt_eps"], gold["pt_lambda"], gold["pt_mu"], gold["pt_d"]
    assert np.array_equal(D.compute_sigma_damaged(lm, mu, e, d, 1e-6), gold["pt_sigma_d"])
    assert np.array_equal(D.compute_sigma_damaged(lm, mu, e), gold["pt_sigma_nod"])
    assert np.array_equal(D.compute_strain_energy(lm, mu, e), gold["pt_psi"])
    # without damage the split law is the linear law
    from oracle import ls_oracle as O

    assert np.allclose(gold["pt_sigma_nod"], O.compute_sigma(lm, mu, e), rtol=0, atol=1e-15)


@pytest.mark.parametrize("tag", ["a", "b"])
@pytest.mark.parametrize("depth", [0, 3])
def test_elasticity_solve(gold, tag, depth):
    from oracle import damage_oracle as D

    g = grid_of(gold[f"el_{tag}_grid"])
    e, s, it = D.elasticity_solve(gold[f"el_{tag}_lambda"], gold[f"el_{tag}_mu"],
                                  gold[f"el_{tag}_ebar"], gold[f"el_{tag}_d"], 1e-6, g, rtol=1e-6,
                                  atol=1e-20, depth=depth, maxiter=300)
    assert it == int(gold[f"el_{tag}_d{depth}_iters"])
    ref = gold[f"el_{tag}_d{depth}_eps"]
    assert np.abs(e - ref).max() <= 1e-9 * np.abs(ref).max()
    ref_s = gold[f"el_{tag}_d{depth}_sigma"]
    assert np.abs(s - ref_s).max() <= 1e-9 * np.abs(ref_s).max()


@pytest.mark.parametrize("tag", ["a", "b"])
def test_phase_field_solve(gold, tag):
    from oracle import damage_oracle as D

    g = grid_of(gold[f"pf_{tag}_grid"])
    d, it = D.phase_field_solve(gold[f"pf_{tag}_H"], gold[f"pf_{tag}_dold"], 2.7e-3, 0.05, g,
                                tolerance=1e-9, maxiter=10000)
    assert it == int(gold[f"pf_{tag}_iters"])
    assert np.abs(d - gold[f"pf_{tag}_d"]).max() <= 1e-14
