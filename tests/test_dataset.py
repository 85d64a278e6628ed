"""Dataset files: the reference's key names and channel order, save/load round trip,
the loader's interface (no GPU)."""

import numpy as np

from jaxmaterials_b200.data import dataset as D


def test_save_load_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    lame = rng.standard_normal((3, 2, 4, 5, 6)).astype(np.float32)
    sig = rng.standard_normal((3, 6, 6)).astype(np.float32)
    path = tmp_path / "fibres.npz"
    D.save(path, lame, sig, [4.0, 5.0, 6.0])
    with np.load(path) as f:
        assert set(f.files) == {"base/lame_parameters", "base/sigma_bar", "domain_size"}
    ds = D.LayeredFibresDataset(path)
    assert len(ds) == 3 and ds.number_of_cells == [4, 5, 6]
    x, y = ds[1]
    np.testing.assert_array_equal(x, lame[1])
    np.testing.assert_array_equal(y, sig[1])
    np.testing.assert_array_equal(ds.domain_size, [4.0, 5.0, 6.0])
    m, s = ds.mean
    np.testing.assert_allclose(m, lame.mean(axis=0))
    np.testing.assert_allclose(s, sig.mean(axis=0))
    ds2 = D.LayeredFibresDataset(path, features_last=True)
    assert ds2[0][0].shape == (4, 5, 6, 2)
    np.testing.assert_array_equal(ds2[0][0][..., 0], lame[0, 0])
