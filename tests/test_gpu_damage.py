"""The damage extension on the GPU (lsb_damage_stress, lsb_strain_energy, lsb_set_damage,
lsb_phase_field_solve) against the CPU oracle and the reference's own outputs."""

import numpy as np
import pytest

from tests.test_damage_oracle import GOLDEN, grid_of

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gold():
    with np.load(GOLDEN) as d:
        return {k: d[k] for k in d.files}


def gspec(g):
    from jaxmaterials_b200 import GridSpec

    return GridSpec(int(g[0]), int(g[1]), int(g[2]), g[3], g[4], g[5])


def relmax(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


def random_strains(rng, shape, n=6):
    """Mixed-sign strains including degenerate tensors (zero, uniaxial, hydrostatic) whose
    eigenvalues coincide."""
    e = rng.normal(size=(n,) + shape) * 1e-3
    flat = e.reshape(n, -1)
    flat[:, 0] = 0.0
    flat[:, 1] = [1e-3, 0, 0, 0, 0, 0]
    flat[:, 2] = [-2e-3, -2e-3, -2e-3, 0, 0, 0]
    flat[:, 3] = [1e-3, 1e-3, -1e-3, 0, 0, 0]
    flat[:, 4] = [0, 0, 0, 1e-3, 0, 0]
    return flat.reshape(e.shape)


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 2e-5)])
def test_pointwise_laws_match_oracle(dtype, tol):
    from jaxmaterials_b200.solver import damage as dm
    from oracle import damage_oracle as D

    rng = np.random.default_rng(7)
    shape = (9, 7, 5)
    e = random_strains(rng, shape)
    lm, mu = rng.uniform(0.5, 2.0, size=(2,) + shape)
    d = rng.uniform(0.0, 1.0, size=shape)
    cast = lambda a: np.asarray(a, dtype)  # noqa: E731
    for dd in (d, None):
        got = dm.compute_sigma_damaged(cast(lm), cast(mu), cast(e), None if dd is None else cast(dd),
                                       1e-6)
        ref = D.compute_sigma_damaged(lm, mu, e, dd, 1e-6)
        assert got.dtype == dtype
        assert relmax(got, ref) < tol
    psi = dm.compute_strain_energy(cast(lm), cast(mu), cast(e))
    assert relmax(psi, D.compute_strain_energy(lm, mu, e)) < tol


def test_pointwise_laws_match_reference(gold):
    from jaxmaterials_b200.solver import damage as dm

    e, lm, mu, d = gold["pt_eps"], gold["pt_lambda"], gold["pt_mu"], gold["pt_d"]
    assert relmax(dm.compute_sigma_damaged(lm, mu, e, d, 1e-6), gold["pt_sigma_d"]) < 1e-12
    assert relmax(dm.compute_sigma_damaged(lm, mu, e), gold["pt_sigma_nod"]) < 1e-12
    assert relmax(dm.compute_strain_energy(lm, mu, e), gold["pt_psi"]) < 1e-12


def test_history_update_is_a_running_maximum():
    import torch

    from jaxmaterials_b200.solver import damage as dm

    rng = np.random.default_rng(3)
    shape = (6, 5, 4)
    lm, mu = rng.uniform(0.5, 2.0, size=(2,) + shape)
    e1, e2 = rng.normal(size=(2, 6) + shape) * 1e-3
    h = torch.zeros(shape, dtype=torch.float64, device="cuda")
    dm.update_history(h, lm, mu, e1)
    dm.update_history(h, lm, mu, e2)
    ref = np.maximum(dm.compute_strain_energy(lm, mu, e1), dm.compute_strain_energy(lm, mu, e2))
    assert np.array_equal(h.cpu().numpy(), ref)


@pytest.mark.parametrize("tag", ["a", "b"])
@pytest.mark.parametrize("depth", [0, 3])
def test_damaged_solve_fixed_iterations_match_oracle(gold, tag, depth):
    """FP64 end to end: fields after the same number of updates agree to round-off."""
    from jaxmaterials_b200.solver import damage as dm
    from oracle import damage_oracle as D

    g = gold[f"el_{tag}_grid"]
    args = (gold[f"el_{tag}_lambda"], gold[f"el_{tag}_mu"], gold[f"el_{tag}_ebar"],
            gold[f"el_{tag}_d"], 1e-6)
    e, s, it = dm.elasticity_solve(*args, gspec(g), rtol=0.0, atol=0.0, depth=depth, maxiter=25,
                                   dtype=np.float64)
    assert it == 25
    e64, s64, _ = D.elasticity_solve(*args, grid_of(g), rtol=0.0, atol=0.0, depth=depth, maxiter=25)
    assert relmax(e, e64) < 1e-10
    assert relmax(s, s64) < 1e-10


def test_damaged_solve_matches_reference_to_convergence(gold):
    from jaxmaterials_b200.solver import damage as dm

    g = gold["el_b_grid"]
    e, s, it = dm.elasticity_solve(gold["el_b_lambda"], gold["el_b_mu"], gold["el_b_ebar"],
                                   gold["el_b_d"], 1e-6, gspec(g), rtol=1e-6, atol=1e-20, depth=3,
                                   maxiter=300, dtype=np.float64)
    assert abs(it - int(gold["el_b_d3_iters"])) <= 2
    assert relmax(e, gold["el_b_d3_eps"]) < 1e-6
    assert relmax(s, gold["el_b_d3_sigma"]) < 1e-6


@pytest.mark.parametrize("depth", [0, 5])
def test_damaged_solve_on_the_fast_passes(depth):
    """A grid of the compile-time-size FP32 passes (32 x 16 x 16) with a damage field, against
    the FP64 oracle after equal updates."""
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.solver import damage as dm
    from oracle import damage_oracle as D
    from oracle import ls_oracle as O

    rng = np.random.default_rng(11)
    n = (32, 16, 16)
    lm = (1.0 + rng.uniform(-0.3, 0.3, n)).astype(np.float32)
    mu = (1.0 + rng.uniform(-0.3, 0.3, n)).astype(np.float32)
    d = np.clip(rng.uniform(-0.5, 1.2, n), 0, 1).astype(np.float32)
    eb = np.array([0.0, 1e-3, -2e-4, 0.0, 1e-4, 0.0])
    e, s, it = dm.elasticity_solve(lm, mu, eb, d, 1e-6, GridSpec(*n, 1.0, 0.5, 0.5), rtol=0.0,
                                   atol=0.0, depth=depth, maxiter=12, dtype=np.float32)
    e64, _, _ = D.elasticity_solve(lm, mu, eb, d, 1e-6, O.Grid(*n, 1.0, 0.5, 0.5), rtol=0.0,
                                   atol=0.0, depth=depth, maxiter=12, spectrum="half")
    assert it == 12
    assert relmax(e, e64) < 2e-4


def test_no_damage_equals_linear_solver():
    """d = 0, k = 0 gives g = 1 and the split law sums to the linear law."""
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.solver import damage as dm
    from jaxmaterials_b200.solver import lippmann_schwinger

    rng = np.random.default_rng(5)
    n = (12, 10, 8)
    lm = (1.0 + rng.uniform(-0.2, 0.2, n))
    mu = (1.0 + rng.uniform(-0.2, 0.2, n))
    eb = np.array([1e-3, -5e-4, 2e-4, 1e-4, 0.0, 3e-4])
    g = GridSpec(*n, 1.2, 0.8, 0.9)
    e1, _, it1 = dm.elasticity_solve(lm, mu, eb, np.zeros(n), 0.0, g, rtol=1e-8, depth=0,
                                     maxiter=200, dtype=np.float64)
    e2, _, it2 = lippmann_schwinger(lm, mu, eb, g, rtol=1e-8, depth=0, maxiter=200, dtype=np.float64)
    assert it1 == it2
    assert relmax(e1, e2) < 1e-12


@pytest.mark.parametrize("tag", ["a", "b"])
def test_phase_field_matches_reference(gold, tag):
    from jaxmaterials_b200.solver import damage as dm

    g = gold[f"pf_{tag}_grid"]
    d, it = dm.phase_field_solve(gold[f"pf_{tag}_H"], gold[f"pf_{tag}_dold"], 2.7e-3, 0.05,
                                 gspec(g), tolerance=1e-9, maxiter=10000, dtype=np.float64)
    assert it == int(gold[f"pf_{tag}_iters"])
    assert np.abs(d - gold[f"pf_{tag}_d"]).max() < 1e-12


@pytest.mark.parametrize("shape", [(32, 16, 16), (20, 15, 1), (17, 9, 12)])
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 2e-5)])
def test_phase_field_matches_oracle(shape, dtype, tol):
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.solver import damage as dm
    from oracle import damage_oracle as D
    from oracle import ls_oracle as O

    rng = np.random.default_rng(sum(shape))
    hh = rng.uniform(0.0, 3e-3, size=shape)
    d0 = rng.uniform(0.0, 0.2, size=shape)
    ext = (1.0, 0.7, 0.5)
    d, it = dm.phase_field_solve(hh.astype(dtype), d0.astype(dtype), 2.7e-3, 0.04,
                                 GridSpec(*shape, *ext), tolerance=1e-7, maxiter=500, dtype=dtype)
    dr, itr = D.phase_field_solve(hh, d0, 2.7e-3, 0.04, O.Grid(*shape, *ext), tolerance=1e-7,
                                  maxiter=500)
    assert abs(it - itr) <= (0 if dtype == np.float64 else 2)
    assert np.abs(d - dr).max() <= tol * np.abs(dr).max()


def test_grouped_damage_fields_equal_separate_solves():
    """Damage fields of shape (S, nx, ny, nz) follow the Lame grouping: two structures x two
    loads in one batch equal separate solves."""
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.solver import Solver

    rng = np.random.default_rng(9)
    n = (32, 16, 16)
    g = GridSpec(*n, 1.0, 0.5, 0.5)
    lm = (1.0 + rng.uniform(-0.3, 0.3, (2,) + n)).astype(np.float32)
    mu = (1.0 + rng.uniform(-0.3, 0.3, (2,) + n)).astype(np.float32)
    d = np.clip(rng.uniform(-0.5, 1.2, (2,) + n), 0, 1).astype(np.float32)
    eb = np.array([[0, 1e-3, 0, 0, 0, 0], [1e-3, 0, 0, 0, 2e-4, 0]] * 2, dtype=np.float32)
    s = Solver(g, batch=4, depth=3)
    s.set_damage(d, 1e-6)
    r = s.solve(lm, mu, eb, rtol=1e-6, maxiter=300)
    e = r.epsilon.cpu().numpy()
    for k in range(2):
        s1 = Solver(g, batch=2, depth=3)
        s1.set_damage(d[k], 1e-6)
        r1 = s1.solve(lm[k], mu[k], eb[2 * k:2 * k + 2], rtol=1e-6, maxiter=300)
        assert np.array_equal(r.iters[2 * k:2 * k + 2], r1.iters)
        assert np.array_equal(e[2 * k:2 * k + 2], r1.epsilon.cpu().numpy())
        s1.close()
    s.close()
