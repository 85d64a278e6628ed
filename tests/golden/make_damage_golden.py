"""Generate the damage / phase-field fixtures by running the REFERENCE's own Python code.

Run from the repository root in an environment that holds the reference checkout:

    python tests/golden/make_damage_golden.py <reference checkout>   (or JAXMATERIALS_REF in the environment)

Imports ``src/jaxmaterials/solver/lippmann_schwinger.py`` (with ``tests/golden/_jaxshim``
standing in for jax, NumPy doing the arithmetic) and runs, unchanged,
``compute_sigma_damaged``, ``compute_strain_energy``, ``elasticity_solve`` and
``phase_field_solve`` on small seeded inputs. Output: ``tests/golden/reference_damage.npz``.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def material(shape, rng):
    """Matrix with a stiffer inclusion and a soft slit (the kind of field the reference's
    phase-field driver builds, tests/phasefield.py:45-145)."""
    lm = np.full(shape, 121.15)
    mu = np.full(shape, 80.77)
    nx, ny, nz = shape
    lm[nx // 3: nx // 2, ny // 3: 2 * ny // 3] *= 2.0
    mu[nx // 3: nx // 2, ny // 3: 2 * ny // 3] *= 2.0
    lm[: nx // 2, ny // 2] = 1.0
    mu[: nx // 2, ny // 2] = 1.0
    return lm, mu


def main(ref_root):
    sys.path.insert(0, os.path.join(HERE, "_jaxshim"))
    sys.path.insert(0, os.path.join(ref_root, "src"))
    from jaxmaterials.common import GridSpec
    from jaxmaterials.solver import lippmann_schwinger as rls

    out = {}
    rng = np.random.default_rng(4711)
    # pointwise laws: mixed-sign strains, with and without damage
    eps = rng.normal(size=(6, 5, 4, 3)) * 1e-3
    lm = rng.uniform(0.5, 2.0, size=(5, 4, 3))
    mu = rng.uniform(0.5, 2.0, size=(5, 4, 3))
    d = rng.uniform(0.0, 1.0, size=(5, 4, 3))
    out["pt_eps"], out["pt_lambda"], out["pt_mu"], out["pt_d"] = eps, lm, mu, d
    out["pt_sigma_d"] = np.asarray(rls.compute_sigma_damaged(lm, mu, eps, d, 1e-6))
    out["pt_sigma_nod"] = np.asarray(rls.compute_sigma_damaged(lm, mu, eps))
    out["pt_psi"] = np.asarray(rls.compute_strain_energy(lm, mu, eps))

    # damaged elasticity solves (FP64, plain and Anderson depth 3)
    for tag, shape in (("a", (9, 8, 1)), ("b", (8, 6, 5))):
        g = GridSpec(*shape, 1.0, 1.0, 0.1 if shape[2] == 1 else 0.6)
        lmf, muf = material(shape, rng)
        dmg = np.clip(rng.uniform(-0.5, 1.2, size=shape), 0.0, 1.0)
        ebar = np.array([0.0, 1e-3, 0.0, 0.0, 0.0, 0.0])
        out[f"el_{tag}_lambda"], out[f"el_{tag}_mu"], out[f"el_{tag}_d"] = lmf, muf, dmg
        out[f"el_{tag}_ebar"] = ebar
        out[f"el_{tag}_grid"] = np.array([*shape, g.Lx, g.Ly, g.Lz])
        for depth in (0, 3):
            e, s, it = rls.elasticity_solve(lmf, muf, ebar, dmg, 1e-6, g, rtol=1e-6, atol=1e-20,
                                            depth=depth, maxiter=300, dtype=np.float64)
            out[f"el_{tag}_d{depth}_eps"] = np.asarray(e)
            out[f"el_{tag}_d{depth}_sigma"] = np.asarray(s)
            out[f"el_{tag}_d{depth}_iters"] = np.asarray(it)

    # phase-field solves (FP64): a 2-d slice like the driver's and a 3-d grid
    for tag, shape in (("a", (12, 10, 1)), ("b", (8, 6, 5))):
        g = GridSpec(*shape, 1.0, 1.0, 0.015 if shape[2] == 1 else 0.6)
        hh = rng.uniform(0.0, 2e-3, size=shape)
        d_old = rng.uniform(0.0, 0.3, size=shape)
        dd, it = rls.phase_field_solve(hh, d_old, 2.7e-3, 0.05, g, tolerance=1e-9, maxiter=10000,
                                       dtype=np.float64)
        out[f"pf_{tag}_H"], out[f"pf_{tag}_dold"] = hh, d_old
        out[f"pf_{tag}_grid"] = np.array([*shape, g.Lx, g.Ly, g.Lz])
        out[f"pf_{tag}_d"] = np.asarray(dd)
        out[f"pf_{tag}_iters"] = np.asarray(it)
    np.savez_compressed(os.path.join(HERE, "reference_damage.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["JAXMATERIALS_REF"])
