"""GPU voxelisation of layered fibre composites (lsb_voxelise_fibres) against the reference's
own fields (tests/golden/reference_fibres.npz) and the CPU oracle, bit for bit; and the
dataset generator end to end."""

import numpy as np
import pytest

from tests.test_fibres import GOLDEN, VALUES, generator, layers_of

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gold():
    with np.load(GOLDEN) as d:
        return {k: d[k] for k in d.files}


@pytest.mark.parametrize("tag,dtype,seed", [("f32", np.float32, 5713853), ("f64", np.float64, 91)])
def test_fields_match_reference(gold, tag, dtype, seed):
    gen = generator(gold, tag, dtype, seed)
    for s in range(2):
        _, pos, rad, ori = layers_of(gold, f"lay_{tag}_{s}_")
        lame = gen.material_properties(pos, rad, ori)
        ref = gold[f"lay_{tag}_{s}_lame"]
        assert lame.dtype == ref.dtype
        assert np.array_equal(lame, ref)


def random_sample(rng, g, nlayers):
    """Layers of random fibres (overlapping each other, reaching into the void layers and
    across the in-plane ends) for a stress test of the predicate and the additions."""
    ext = (g.Lx, g.Ly)
    pos, rad, ori = [], [], []
    for k in range(nlayers):
        o = int(rng.integers(0, 2))
        n = int(rng.integers(1, 40))
        u = rng.uniform(-0.1, 1.1, n) * ext[o]
        z = rng.uniform(-0.05, 1.05, n) * g.Lz
        pos.append(np.stack([u, z], axis=1))
        rad.append(rng.uniform(0.02, 0.25, n) * min(ext[o], g.Lz))
        ori.append(o)
    return pos, rad, ori


@pytest.mark.parametrize("shape", [(17, 23, 11), (32, 16, 48), (5, 64, 9)])
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_random_fibres_match_oracle(shape, dtype):
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.data.layered import voxelise
    from oracle import fibres_oracle

    rng = np.random.default_rng(sum(shape))
    g = GridSpec(*shape, 1.3, 0.7, 0.9)
    vals = (0.11, 3.0, 7.3, 0.2, 1.7, 0.9)
    samples = [random_sample(rng, g, int(rng.integers(1, 5))) for _ in range(4)]
    got = voxelise(samples, g, 0.07, vals, dtype).cpu().numpy()
    for s, (pos, rad, ori) in enumerate(samples):
        ref = fibres_oracle.material_properties((*shape, g.Lx, g.Ly, g.Lz), 0.07, vals, pos, rad,
                                                ori, dtype=dtype)
        assert np.array_equal(got[s], ref), s


def test_voxelise_rejects_bad_input():
    from jaxmaterials_b200 import GridSpec, _lib
    from jaxmaterials_b200.data.layered import voxelise

    g = GridSpec(8, 8, 8, 1.0, 1.0, 1.0)
    bad = [([np.array([[0.5, 0.5]])], [np.array([0.1])], [2])]  # orientation 2
    with pytest.raises(_lib.LibraryError, match="orientation"):
        voxelise(bad, g, 0.1, VALUES)
    assert voxelise([], g, 0.1, VALUES).shape == (0, 2, 8, 8, 8)


def test_dataset_generation_end_to_end(tmp_path):
    import torch

    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.data.dataset import LayeredFibresDataset
    from jaxmaterials_b200.data.distributions_fibres import FibreRadiusDistribution
    from jaxmaterials_b200.data.layered import LayeredFibresDatasetGenerator
    from jaxmaterials_b200.solver import c_eff

    g = GridSpec(32, 32, 16, 0.5, 0.5, 0.2)

    def make():
        rd = FibreRadiusDistribution(r_avg=7.5e-3, r_min=5.0e-3, r_max=10.0e-3, sigma=0.5e-3,
                                     gaussian=True)
        return LayeredFibresDatasetGenerator(g, 3, 0.01, 3, rd, volume_fraction=0.3,
                                             mu_fibre=0.5, mu_material=1.0, mu_void=0.1,
                                             lambda_fibre=0.1, lambda_material=0.5,
                                             lambda_void=1.0, dtype=np.float32,
                                             rng=np.random.default_rng(1))

    gen = make()
    lame, sigma = gen.generate(structures_per_batch=2)
    assert lame.shape == (3, 2, 32, 32, 16) and sigma.shape == (3, 6, 6)
    # the fields are the voxelisation of the positions a fresh generator draws first
    gen2 = make()
    _, pos, rad, ori = gen2.generate_fibre_positions()
    assert np.array_equal(gen2.material_properties(pos, rad, ori), lame[0])
    # C_eff of sample 1 equals a separate solve to the same tolerance
    c, _, _ = c_eff(lame[1, 1], lame[1, 0], g, rtol=1e-4, atol=1e-4, maxiter=100)
    assert np.allclose(sigma[1], c, rtol=2e-3, atol=2e-4)
    path = tmp_path / "fibres.npz"
    gen.save_hdf5(str(path))
    ds = LayeredFibresDataset(str(path))
    x, y = ds[2]
    assert np.array_equal(x, lame[2]) and np.array_equal(y, sigma[2])
    torch.cuda.synchronize()
