"""Layered cross-ply fibre composites: the reference's ``LayeredFibresDatasetGenerator``
(``src/jaxmaterials/data/data.py:63-331``) with its fibre placement on all host cores
(``libfibres.so``) and its voxelisation and C_eff solves on the GPU.

* ``generate_fibre_positions`` consumes the NumPy generators exactly as the reference does
  (layer boundaries, orientation offset, per-layer seed, radius draws; data.py:188-265) and
  places the fibres with the reference's shaking algorithm (bit-identical positions).
* ``material_properties`` returns the reference's (mu, lambda) fields (data.py:267-314)
  bit for bit, computed by ``lsb_voxelise_fibres`` on the GPU.
* ``generate`` builds the whole dataset: all layers of all samples are shaken in one
  threaded call, all samples voxelised on the device, and the six unit-strain solves of
  every sample run as grouped GPU batches (data.py:148-186: plain iteration, rtol = atol =
  1e-4, at most 100 updates; a solve that reaches 100 raises, as the reference's wrapper
  does). The fields go to the solver as labelled: the reference's wrapper hands mu to the
  lambda argument of its library (src/jaxmaterials/solver/lippmann_schwinger.py:310-312).
"""

import ctypes

import numpy as np

from .. import _lib
from .distributions_fibres import initial_lattice, place_batch

__all__ = ["LayeredFibresDatasetGenerator", "voxelise", "voxelise_records", "fibre_records"]

_ELEM = {np.dtype(np.float32): 4, np.dtype(np.float64): 8}


def _records(fibre_positions, fibre_radii, fibre_orientations):
    """(u0, z0, r^2, orientation) per fibre, layer by layer; r^2 evaluated as the reference
    evaluates ``r**2`` on a NumPy scalar (data.py:309-311)."""
    rows = []
    for x, r, o in zip(fibre_positions, fibre_radii, fibre_orientations):
        for p, rr in zip(x, r):
            rows.append((p[0], p[1], rr ** 2, float(o)))
    return np.asarray(rows, dtype=np.float64).reshape(-1, 4)


def fibre_records(samples):
    """Offsets (S + 1,) and records (total, 4) of the fibres of many samples, the inputs of
    ``lsb_voxelise_fibres``."""
    recs = [_records(*s) for s in samples]
    off = np.zeros(len(samples) + 1, dtype=np.int32)
    off[1:] = np.cumsum([len(r) for r in recs])
    fib = np.ascontiguousarray(np.concatenate(recs, axis=0) if recs else np.zeros((0, 4)))
    return off, fib


def voxelise_records(off, fib, grid_spec, d_void, values, dtype=np.float32, device=None):
    """``voxelise`` from prepared records (``fibre_records``)."""
    import torch

    dt = np.dtype(dtype)
    if dt not in _ELEM:
        raise ValueError("dtype must be float32 or float64")
    g = grid_spec
    n = len(off) - 1
    device = torch.device(device) if device is not None else torch.device("cuda")
    out = torch.empty((n, 2, g.nx, g.ny, g.nz),
                      dtype=torch.float32 if dt == np.float32 else torch.float64, device=device)
    if n == 0:
        return out
    off = np.ascontiguousarray(off, dtype=np.int32)
    fib = np.ascontiguousarray(fib, dtype=np.float64)
    voxels = np.array([g.nx, g.ny, g.nz], dtype=np.int32)
    extents = np.array([g.Lx, g.Ly, g.Lz], dtype=np.float64)
    vals = np.asarray(values, dtype=np.float64)
    lib = _lib.load()
    with torch.cuda.device(device):
        stream = torch.cuda.current_stream(device).cuda_stream
        rc = lib.lsb_voxelise_fibres(
            n, voxels.ctypes.data_as(_lib.c_int_p), extents.ctypes.data_as(_lib.c_double_p),
            float(d_void), float(g.Lz - d_void), vals.ctypes.data_as(_lib.c_double_p),
            off.ctypes.data_as(_lib.c_int_p), fib.ctypes.data_as(_lib.c_double_p), _ELEM[dt],
            ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    _lib.check(rc, "lsb_voxelise_fibres")
    return out


def voxelise(samples, grid_spec, d_void, values, dtype=np.float32, device=None):
    """(mu, lambda) fields of many samples on the GPU: a torch tensor of shape
    (S, 2, nx, ny, nz) on ``device``.

    samples: list of (fibre_positions, fibre_radii, fibre_orientations) as returned by
    ``generate_fibre_positions`` (without the boundaries); values = (mu_void, lambda_void,
    mu_fibre, lambda_fibre, mu_material, lambda_material)."""
    off, fib = fibre_records(samples)
    return voxelise_records(off, fib, grid_spec, d_void, values, dtype, device)


class LayeredFibresDatasetGenerator:
    """Samples (X, y): X = Lame fields (mu, lambda) of shape (2, nx, ny, nz), y = C_eff (6,
    6) with row k the mean stress for the unit strain e_k. Between void layers of thickness
    d_void at the bottom and top, ``nlayers`` layers of random depths hold fibres along x and
    y alternately (data.py:63-146; same arguments and defaults)."""

    def __init__(self, grid_spec, nlayers, d_void, n_samples, radius_distribution,
                 volume_fraction=0.3, mu_fibre=1.0, mu_material=0.5, mu_void=0.1,
                 lambda_fibre=0.1, lambda_material=0.1, lambda_void=0.01, rng=None,
                 dtype=np.float64, verbose=False):
        self.grid_spec = grid_spec
        self.nlayers = nlayers
        self.d_void = d_void
        self.n_samples = n_samples
        self.radius_distribution = radius_distribution
        self.volume_fraction = volume_fraction
        self.mu_fibre = mu_fibre
        self.mu_material = mu_material
        self.mu_void = mu_void
        self.lambda_fibre = lambda_fibre
        self.lambda_material = lambda_material
        self.lambda_void = lambda_void
        self.rng = np.random.default_rng(seed=64217) if rng is None else rng
        self.dtype = dtype
        self.verbose = verbose

    # ---- fibre positions
    def _draw_layers(self):
        """The random draws of one sample, in the reference's order (data.py:205-234):
        layer boundaries (redrawn until every layer is at least 3 r_max deep), orientation
        offset, then per layer a seed and the radii of its start lattice."""
        r_max = self.radius_distribution.r_max
        g = self.grid_spec
        depths = np.asarray([0.5 * r_max])
        while np.any(depths < 3 * r_max):
            bounds = np.asarray(sorted(
                [self.d_void, g.Lz - self.d_void]
                + [float(z) for z in self.rng.uniform(size=self.nlayers - 1, low=self.d_void,
                                                      high=g.Lz - self.d_void)]))
            depths = bounds[1:] - bounds[:-1]
        offset = self.rng.integers(low=0, high=2, size=1)[0]
        extent = [g.Lx, g.Ly, g.Lz]
        layers = []
        for k in range(self.nlayers):
            orientation = (k + offset) % 2
            self.rng.integers(low=0, high=2, size=1)  # the per-layer seed (unused by the C++ path)
            box = np.asarray([extent[orientation], depths[k] - 2 * r_max], dtype=np.float64)
            lattice = initial_lattice(box, self.radius_distribution.r_avg, self.volume_fraction)
            radii = self.radius_distribution.draw(lattice.shape[0])
            layers.append((orientation, box, lattice, radii))
        return bounds, layers

    def _assemble(self, bounds, layers, moved):
        """Periodic copies across the in-plane ends and the shift to the layer's height
        (data.py:236-264)."""
        r_max = self.radius_distribution.r_max
        extent = [self.grid_spec.Lx, self.grid_spec.Ly, self.grid_spec.Lz]
        positions, radii, orientations = [], [], []
        for k, ((orientation, _, _, r), x) in enumerate(zip(layers, moved)):
            length = extent[orientation]
            lower = (np.less_equal(x[..., 0], r_max),)
            upper = np.greater_equal(x[..., 0], length - r_max)
            x = np.concatenate([x, x[lower] + np.asarray([length, 0]),
                                x[upper] - np.asarray([length, 0])], axis=0)
            r = np.concatenate([r, r[lower], r[upper]], axis=0)
            x += (np.asarray([0, bounds[k] + r_max]),)
            positions.append(x)
            radii.append(r)
            orientations.append(orientation)
        return bounds, positions, radii, orientations

    def generate_fibre_positions(self):
        """(layer boundaries, fibre positions per layer (n_j, 2) projected on the plane
        across the fibres, radii per layer, orientation per layer) of one new sample."""
        return self.generate_fibre_positions_batch(1)[0]

    def generate_fibre_positions_batch(self, n):
        """``generate_fibre_positions`` for n samples, their layers shaken in one threaded
        call. Identical to n consecutive single calls."""
        drawn = [self._draw_layers() for _ in range(n)]
        flat = [layer for _, layers in drawn for layer in layers]
        moved = place_batch([b for _, b, _, _ in flat], [r for _, _, _, r in flat],
                            [x for _, _, x, _ in flat])
        out, i = [], 0
        for bounds, layers in drawn:
            out.append(self._assemble(bounds, layers, moved[i:i + len(layers)]))
            i += len(layers)
        return out

    # ---- fields
    @property
    def _values(self):
        return (self.mu_void, self.lambda_void, self.mu_fibre, self.lambda_fibre,
                self.mu_material, self.lambda_material)

    def material_properties(self, fibre_positions, fibre_radii, fibre_orientations):
        """(mu, lambda) at the voxel centres, shape (2, nx, ny, nz), dtype ``self.dtype``
        (computed on the GPU, equal to the reference's NumPy evaluation)."""
        t = voxelise([(fibre_positions, fibre_radii, fibre_orientations)], self.grid_spec,
                     self.d_void, self._values, self.dtype)
        return t[0].cpu().numpy()

    # ---- dataset
    def generate(self, structures_per_batch=0, device=None):
        """Lame fields and C_eff of ``n_samples`` samples (``_lame_parameters``,
        ``_sigma_bar``)."""
        import torch

        from ..solver import CONVERGED, Solver

        g = self.grid_spec
        device = torch.device(device) if device is not None else torch.device("cuda")
        samples = [s[1:] for s in self.generate_fibre_positions_batch(self.n_samples)]
        lame = voxelise(samples, g, self.d_void, self._values, self.dtype, device)
        self._lame_parameters = lame.cpu().numpy()
        # six instances per structure at about 50 B per voxel each (FP32 strain and
        # spectrum): about 8 GB of solver state per batch
        s_max = structures_per_batch or int(np.clip(8e9 // (300 * g.number_of_voxels), 1, 256))
        s_max = min(s_max, max(self.n_samples, 1))
        self._sigma_bar = np.empty((self.n_samples, 6, 6), dtype=self.dtype)
        solver = Solver(g, batch=6 * min(s_max, self.n_samples), depth=0, precision="mixed")
        try:
            for j0 in range(0, self.n_samples, s_max):
                s = min(s_max, self.n_samples - j0)
                lm = lame[j0:j0 + s, 1].to(torch.float32).contiguous()
                mu = lame[j0:j0 + s, 0].to(torch.float32).contiguous()
                eb = np.tile(np.eye(6, dtype=np.float32), (s, 1))
                r = solver.solve(lm, mu, eb, rtol=1.0e-4, atol=1.0e-4, maxiter=100,
                                 want_sigma=False)
                bad = np.flatnonzero(r.status != CONVERGED)
                if len(bad):
                    b = int(bad[0])
                    raise RuntimeError(f"sample {j0 + b // 6}, load case {b % 6}: no convergence "
                                       f"in {int(r.iters[b])} iterations")
                self._sigma_bar[j0:j0 + s] = r.mean_sigma.reshape(s, 6, 6)
        finally:
            solver.close()
        return self._lame_parameters, self._sigma_bar

    def save_hdf5(self, filename):
        """Write the dataset in the reference's layout (see ``dataset.save``)."""
        from .dataset import save

        assert hasattr(self, "_lame_parameters") and hasattr(self, "_sigma_bar"), \
            "Data not generated yet, call generate() first."
        g = self.grid_spec
        save(filename, self._lame_parameters, self._sigma_bar, [g.Lx, g.Ly, g.Lz])


def reference_config_generator(n_samples, seed=5713853, dtype=np.float32):
    """The reference's dataset script configuration (src/generate_data.py:14-56): 160 x 160 x
    64 voxels on 0.5 x 0.5 x 0.2, 3 fibre layers, void layers 0.01, volume fraction 0.3,
    radii normal 7.5e-3 +- 0.5e-3 in [5e-3, 1e-2]."""
    from .. import GridSpec
    from .distributions_fibres import FibreRadiusDistribution

    rd = FibreRadiusDistribution(r_avg=7.5e-3, r_min=5.0e-3, r_max=10.0e-3, sigma=0.5e-3,
                                 gaussian=True)
    return LayeredFibresDatasetGenerator(
        GridSpec(160, 160, 64, 0.5, 0.5, 0.2), 3, 0.01, n_samples, rd, volume_fraction=0.3,
        mu_fibre=0.5, mu_material=1.0, mu_void=0.1, lambda_fibre=0.1, lambda_material=0.5,
        lambda_void=1.0, dtype=dtype, rng=np.random.default_rng(seed))


def benchmark(n_samples, seed=5713853, pipeline=True, keep_first=False):
    """Timings of the reference configuration for ``n_samples`` samples: fibre placement on
    all host cores and on one, GPU voxelisation (CUDA events around the library call:
    record upload and kernels), and (``pipeline``) the whole ``generate`` (wall clock)."""
    import time

    import torch

    from .distributions_fibres import place_batch

    gen = reference_config_generator(n_samples, seed)
    g = gen.grid_spec
    t = time.perf_counter()
    samples = [smp[1:] for smp in gen.generate_fibre_positions_batch(n_samples)]
    t_place = time.perf_counter() - t
    gen1 = reference_config_generator(n_samples, seed)
    flat = [layer for _ in range(n_samples) for layer in gen1._draw_layers()[1]]
    t = time.perf_counter()
    place_batch([b for _, b, _, _ in flat], [r for _, _, _, r in flat],
                [x for _, _, x, _ in flat], threads=1)
    t_place1 = time.perf_counter() - t
    off, fib = fibre_records(samples)
    vals = gen._values
    voxelise_records(off, fib, g, gen.d_void, vals)  # warm-up (sizes the device scratch)
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    out = voxelise_records(off, fib, g, gen.d_void, vals)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    res = {"samples": n_samples, "grid": [g.nx, g.ny, g.nz], "layers": gen.nlayers,
           "volume_fraction": gen.volume_fraction, "fibres_per_sample": len(fib) / n_samples,
           "placement_s_per_sample": t_place / n_samples,
           "placement_s_per_sample_1_thread": t_place1 / n_samples,
           "voxelise_ms_per_sample": ms / n_samples,
           "voxelise_bytes_per_sample": 2 * g.number_of_voxels * 4}
    first = (samples[0], out[0].cpu().numpy()) if keep_first else None
    del out
    if pipeline:
        gen2 = reference_config_generator(n_samples, seed)
        t = time.perf_counter()
        gen2.generate()
        res["pipeline_samples_per_s"] = n_samples / (time.perf_counter() - t)
    return res, first


def main(argv=None):
    """``python -m jaxmaterials_b200.data.layered --samples N [--no-pipeline]``: timings of the
    reference dataset configuration as one JSON line."""
    import argparse
    import json

    p = argparse.ArgumentParser()
    p.add_argument("--samples", type=int, default=16)
    p.add_argument("--no-pipeline", action="store_true")
    a = p.parse_args(argv)
    res, _ = benchmark(a.samples, pipeline=not a.no_pipeline)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
