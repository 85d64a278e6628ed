"""C_eff datasets of layered fibre composites: generation with the batched solver, storage,
loading.

Mirrors the reference's dataset pipeline (src/jaxmaterials/data/data.py:15-60 and
:148-186, :316-331): per sample the Lame fields in channel order [mu, lambda] with shape
(2, nx, ny, nz) and the effective stiffness `sigma_bar` (6, 6) whose row k is the mean
stress for the unit strain e_k, plus the domain size. The reference writes HDF5 with the
datasets "base/lame_parameters", "base/sigma_bar" and the attribute "domain_size"; h5py is
not part of this environment, so files here are NumPy .npz archives with exactly those
keys (an .h5 name is read or written with h5py when it is installed). The reference solves
one structure and one load case at a time; here the whole dataset goes through
lsb_c_eff_batch (six loads per structure, structures batched on the GPU).
"""

import numpy as np

from .. import GridSpec
from . import fibres

KEY_LAME = "base/lame_parameters"
KEY_SIGMA = "base/sigma_bar"
KEY_DOMAIN = "domain_size"


def generate(n_samples, n=32, seed=0, nlayers=(2, 6), radius=(2.0, 5.0),
             volume_fraction=(0.30, 0.55), rtol=1e-6, depth=5, maxiter=5000, dtype=np.float32,
             memory_gb=0.0):
    """Seeded cross-ply structures on an n^3 grid (cubic voxels of unit size) and their C_eff.

    Returns (lame_parameters (n_samples, 2, n, n, n) [mu, lambda], sigma_bar
    (n_samples, 6, 6), domain_size (3,), iterations (n_samples, 6))."""
    from ..solver import c_eff_batch

    rng = np.random.default_rng(seed)
    lame = np.empty((n_samples, 2, n, n, n), dtype=dtype)
    lms, mus = [], []
    for j in range(n_samples):
        st = fibres.generate_layered_fibres(
            n, int(rng.integers(nlayers[0], nlayers[1] + 1)), float(rng.uniform(*radius)),
            float(rng.uniform(*volume_fraction)), int(rng.integers(0, 2**31 - 1)))
        lm, mu = fibres.lame_fields(st)
        lame[j, 0], lame[j, 1] = mu, lm
        lms.append(lm)
        mus.append(mu)
    g = GridSpec(n, n, n, float(n), float(n), float(n))
    c, iters, _ = c_eff_batch(lms, mus, g, rtol=rtol, depth=depth, maxiter=maxiter,
                              memory_gb=memory_gb)
    return lame, c.astype(dtype), np.array([g.Lx, g.Ly, g.Lz]), iters


def save(filename, lame_parameters, sigma_bar, domain_size):
    """Write a dataset (.npz with the reference's HDF5 names; .h5 through h5py)."""
    if str(filename).endswith((".h5", ".hdf5")):
        import h5py

        with h5py.File(filename, "w") as f:
            group = f.create_group("base")
            group.create_dataset("lame_parameters", data=lame_parameters)
            group.create_dataset("sigma_bar", data=sigma_bar)
            f.attrs[KEY_DOMAIN] = list(domain_size)
        return
    np.savez(filename, **{KEY_LAME: lame_parameters, KEY_SIGMA: sigma_bar,
                          KEY_DOMAIN: np.asarray(domain_size, dtype=np.float64)})


def _load(filename):
    if str(filename).endswith((".h5", ".hdf5")):
        import h5py

        with h5py.File(filename, "r") as f:
            return (np.array(f[KEY_LAME]), np.array(f[KEY_SIGMA]),
                    np.array(f.attrs[KEY_DOMAIN]))
    with np.load(filename) as d:
        return np.array(d[KEY_LAME]), np.array(d[KEY_SIGMA]), np.array(d[KEY_DOMAIN])


class LayeredFibresDataset:
    """A dataset as loaded from disk (the reference's ``LayeredFibresDataset`` interface):
    item idx is (lame parameters (2, nx, ny, nz) [mu, lambda] or, with features_last,
    (nx, ny, nz, 2), and sigma_bar (6, 6)). Usable as a torch Dataset."""

    def __init__(self, filename, features_last=False):
        lame, sigma, domain = _load(filename)
        self.number_of_cells = list(lame.shape[-3:])
        if features_last:
            lame = np.transpose(lame, axes=(0, 2, 3, 4, 1))
        self._lame_parameters = lame
        self._sigma_bar = sigma
        self.domain_size = domain
        self.n_samples = lame.shape[0]

    def __len__(self):
        return self.n_samples

    def __getitem__(self, idx):
        return self._lame_parameters[idx, ...], self._sigma_bar[idx, ...]

    @property
    def mean(self):
        """Pointwise means over the samples."""
        return np.mean(self._lame_parameters, axis=(0,)), np.mean(self._sigma_bar, axis=(0,))

    @property
    def std(self):
        """Pointwise standard deviations over the samples."""
        return np.std(self._lame_parameters, axis=(0,)), np.std(self._sigma_bar, axis=(0,))
