"""Generate the fibre-placement and voxelisation fixtures by running the REFERENCE's own
Python code (and, through it, its C++ fibre library, which it compiles with g++).

Run from the repository root in an environment that holds the reference checkout:

    python tests/golden/make_fibres_golden.py <reference checkout>   (or JAXMATERIALS_REF in the environment)

``src/jaxmaterials/data/distributions_fibres.py`` and ``src/jaxmaterials/data/data.py`` are
imported and executed unchanged. data.py imports modules that are not installed here and
that the called functions do not use: jax (``tests/golden/_jaxshim``), h5py and
matplotlib (empty stand-ins below). The outputs land in ``tests/golden/reference_fibres.npz``;
the tests read only that file.
"""

import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _stand_ins():
    sys.modules.setdefault("h5py", types.ModuleType("h5py"))
    mpl = types.ModuleType("matplotlib")
    mpl.pyplot = types.ModuleType("matplotlib.pyplot")
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", mpl.pyplot)


def _flatten(prefix, out, positions, radii, orientations, bounds):
    out[prefix + "bounds"] = np.asarray(bounds)
    out[prefix + "orient"] = np.asarray(orientations, dtype=np.int64)
    out[prefix + "counts"] = np.asarray([len(r) for r in radii], dtype=np.int64)
    out[prefix + "pos"] = np.concatenate(positions, axis=0)
    out[prefix + "rad"] = np.concatenate(radii, axis=0)


def main(ref_root):
    sys.path.insert(0, os.path.join(HERE, "_jaxshim"))
    sys.path.insert(0, os.path.join(ref_root, "src"))
    _stand_ins()
    from jaxmaterials.common import GridSpec
    from jaxmaterials.data import data as rdata
    from jaxmaterials.data import distributions_fibres as rdf

    out = {}
    # 1. 2-d fibre sets: the C++ path, two consecutive draws of one instance (the C++
    # generator state carries over), at three volume fractions and box shapes
    cases = [((0.25, 0.05), 0.30, 11), ((0.12, 0.12), 0.45, 12), ((0.30, 0.03), 0.55, 13)]
    for i, (box, vf, seed) in enumerate(cases):
        rd = rdf.FibreRadiusDistribution(r_avg=7.5e-3, r_min=5.0e-3, r_max=10.0e-3,
                                         sigma=0.5e-3, gaussian=True, seed=100 + i)
        fd = rdf.FibreDistribution2d(box, volume_fraction=vf, r_fibre_dist=rd, seed=seed)
        it = iter(fd)
        out[f"d2_{i}_box"] = np.asarray(box)
        out[f"d2_{i}_vf"] = np.asarray(vf)
        out[f"d2_{i}_lattice"] = np.array(fd._initial_fibre_locations)
        for draw in range(2):
            x, r = next(it)
            out[f"d2_{i}_x{draw}"] = x
            out[f"d2_{i}_r{draw}"] = r
    # the NumPy path (fast_code=False) on a small set
    rd = rdf.FibreRadiusDistribution(r_avg=7.5e-3, r_min=5.0e-3, r_max=10.0e-3, sigma=0.5e-3,
                                     gaussian=True, seed=7)
    fd = rdf.FibreDistribution2d((0.08, 0.04), volume_fraction=0.3, r_fibre_dist=rd, seed=5,
                                 fast_code=False)
    x, r = next(iter(fd))
    out["np_box"] = np.asarray((0.08, 0.04))
    out["np_x"] = x
    out["np_r"] = r
    # constant radii
    rd = rdf.FibreRadiusDistribution(r_avg=7.5e-3, r_min=5.0e-3, r_max=10.0e-3, sigma=0.5e-3,
                                     gaussian=False)
    out["const_r"] = rd.draw(5)

    # 2. layered samples: positions and (mu, lambda) fields, float32 and float64
    g = GridSpec(40, 40, 16, 0.5, 0.5, 0.2)
    for tag, dtype, seed in (("f32", np.float32, 5713853), ("f64", np.float64, 91)):
        rd = rdf.FibreRadiusDistribution(r_avg=7.5e-3, r_min=5.0e-3, r_max=10.0e-3,
                                         sigma=0.5e-3, gaussian=True, seed=856219)
        gen = rdata.LayeredFibresDatasetGenerator(
            g, 3, 0.01, 2, rd, volume_fraction=0.3, mu_fibre=0.5, mu_material=1.0,
            mu_void=0.1, lambda_fibre=0.1, lambda_material=0.5, lambda_void=1.0, dtype=dtype,
            rng=np.random.default_rng(seed=seed))
        for s in range(2):
            bounds, pos, rad, ori = gen.generate_fibre_positions()
            _flatten(f"lay_{tag}_{s}_", out, pos, rad, ori, bounds)
            out[f"lay_{tag}_{s}_lame"] = gen.material_properties(pos, rad, ori)
    out["lay_grid"] = np.asarray([g.nx, g.ny, g.nz, g.Lx, g.Ly, g.Lz])
    np.savez_compressed(os.path.join(HERE, "reference_fibres.npz"), **out)
    print("wrote", os.path.join(HERE, "reference_fibres.npz"), len(out), "arrays")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["JAXMATERIALS_REF"])
