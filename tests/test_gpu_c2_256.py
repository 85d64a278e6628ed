"""Config 2 at 256^3 (4 cross-ply layers, fibre radius 4 voxels, vf 0.45, six unit loads,
tol 1e-6): the mixed-precision FP32 solve, Anderson m = 5 and plain, gives C_eff within
1e-5 (relative Frobenius) of an FP64 Anderson run of the same solver on the same structure
(the FP64 path is pinned to the FP64 oracle at small sizes in test_gpu_parity.py) and, when
tests/golden/bench_c2_256.npz holds it, of the FP64 CPU oracle's C_eff.
"""

import os

import numpy as np
import pytest

from tests.conftest import ROOT

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem(built_library):
    import torch

    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.data import fibres
    from jaxmaterials_b200.solver import CONVERGED, Solver

    st = fibres.config_structure("c2_256", seed=0)
    lm, mu = fibres.lame_fields(st)
    g = GridSpec(*st.n, *st.extents)
    lm_d = torch.as_tensor(lm, device="cuda")
    mu_d = torch.as_tensor(mu, device="cuda")
    s64 = Solver(g, batch=6, depth=5, precision="fp64")
    r64 = s64.solve(lm_d.double(), mu_d.double(), np.eye(6), rtol=1e-6, atol=1e-20,
                    maxiter=3000, want_sigma=False)
    assert np.all(r64.status == CONVERGED)
    c64 = np.asarray(r64.mean_sigma, np.float64)
    s64.close()
    torch.cuda.empty_cache()
    path = os.path.join(ROOT, "tests", "golden", "bench_c2_256.npz")
    oracle = np.load(path)["ceff_d5"] if os.path.exists(path) else None
    return g, lm_d, mu_d, c64, oracle


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - b) / np.linalg.norm(b))


@pytest.mark.parametrize("depth", [5, 0])
def test_c2_256_ceff_vs_fp64(problem, depth):
    import torch

    from jaxmaterials_b200.solver import CONVERGED, Solver

    g, lm_d, mu_d, c64, oracle = problem
    s = Solver(g, batch=6, depth=depth)
    r = s.solve(lm_d, mu_d, np.eye(6, dtype=np.float32), rtol=1e-6, atol=1e-20, maxiter=3000,
                want_sigma=False)
    assert np.all(r.status == CONVERGED), r.status
    assert rel(r.mean_sigma, c64) < 1e-5
    if oracle is not None:
        assert rel(r.mean_sigma, oracle) < 1e-5
        assert rel(c64, oracle) < 1e-6
    # rows are mean stresses for unit tensor strains, so diag(1/w) M (w = 1,1,1,2,2,2) is the
    # engineering stiffness, symmetric to solver tolerance
    d = np.diag([1.0, 1.0, 1.0, 0.5, 0.5, 0.5]) @ np.asarray(r.mean_sigma)
    assert np.abs(d - d.T).max() < 1e-5 * np.abs(d).max()
    s.close()
    torch.cuda.empty_cache()
