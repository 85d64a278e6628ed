"""Fibre placement (libfibres.so) and the voxelisation oracle against the reference's own
outputs (tests/golden/reference_fibres.npz, made by tests/golden/make_fibres_golden.py) and
against the reference's C++ library built from its sources (oracle/_ref/libfibres.so).
No GPU needed."""

import ctypes
import os

import numpy as np
import pytest

from tests.conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_fibres.npz")
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libfibres.so")
VALUES = (0.1, 1.0, 0.5, 0.1, 1.0, 0.5)  # mu/lambda of void, fibre, matrix in the fixture


@pytest.fixture(scope="module")
def gold():
    with np.load(GOLDEN) as d:
        return {k: d[k] for k in d.files}


@pytest.fixture(scope="module")
def fibres_lib(built_library):
    from jaxmaterials_b200 import _lib

    return _lib.load_fibres()


def radius_dist(seed, gaussian=True):
    from jaxmaterials_b200.data.distributions_fibres import FibreRadiusDistribution

    return FibreRadiusDistribution(r_avg=7.5e-3, r_min=5.0e-3, r_max=10.0e-3, sigma=0.5e-3,
                                   gaussian=gaussian, seed=seed)


def layers_of(gold, prefix):
    counts = gold[prefix + "counts"]
    cut = np.cumsum(counts)[:-1]
    return (gold[prefix + "bounds"], np.split(gold[prefix + "pos"], cut),
            np.split(gold[prefix + "rad"], cut), [int(o) for o in gold[prefix + "orient"]])


@pytest.mark.parametrize("case", [0, 1, 2])
def test_fibre_sets_match_reference(fibres_lib, gold, case):
    from jaxmaterials_b200.data.distributions_fibres import FibreDistribution2d

    box = tuple(gold[f"d2_{case}_box"])
    fd = FibreDistribution2d(box, volume_fraction=float(gold[f"d2_{case}_vf"]),
                             r_fibre_dist=radius_dist(100 + case), seed=11 + case)
    assert np.array_equal(fd._initial_fibre_locations, gold[f"d2_{case}_lattice"])
    it = iter(fd)
    for draw in range(2):  # the second draw continues the first one's C++ random stream
        x, r = next(it)
        assert np.array_equal(r, gold[f"d2_{case}_r{draw}"])
        assert np.array_equal(x, gold[f"d2_{case}_x{draw}"])


def test_numpy_path_matches_reference(gold):
    """The oracle's restatement of the reference's NumPy shaking path (fast_code=False)
    reproduces the reference's positions bit for bit."""
    from jaxmaterials_b200.data.distributions_fibres import initial_lattice
    from oracle import fibres_oracle

    box = np.asarray(gold["np_box"], dtype=np.float64)
    rd = radius_dist(7)
    x0 = initial_lattice(box, rd.r_avg, 0.3)
    r = rd.draw(x0.shape[0])
    x = fibres_oracle.move_fibres(np.random.default_rng(5), np.array(x0), r, box)
    assert np.array_equal(r, gold["np_r"])
    assert np.array_equal(x, gold["np_x"])


def test_numpy_shaking_path_is_not_in_the_product():
    from jaxmaterials_b200.data.distributions_fibres import FibreDistribution2d

    with pytest.raises(ValueError):
        FibreDistribution2d((0.1, 0.1), fast_code=False)


def test_constant_radii(gold):
    assert np.array_equal(radius_dist(0, gaussian=False).draw(5), gold["const_r"])


def generator(gold, tag, dtype, seed):
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.data.layered import LayeredFibresDatasetGenerator

    nx, ny, nz, Lx, Ly, Lz = gold["lay_grid"]
    g = GridSpec(int(nx), int(ny), int(nz), Lx, Ly, Lz)
    return LayeredFibresDatasetGenerator(
        g, 3, 0.01, 2, radius_dist(856219), volume_fraction=0.3, mu_fibre=0.5,
        mu_material=1.0, mu_void=0.1, lambda_fibre=0.1, lambda_material=0.5, lambda_void=1.0,
        dtype=dtype, rng=np.random.default_rng(seed=seed))


@pytest.mark.parametrize("tag,dtype,seed", [("f32", np.float32, 5713853), ("f64", np.float64, 91)])
@pytest.mark.parametrize("batched", [False, True])
def test_layer_positions_match_reference(fibres_lib, gold, tag, dtype, seed, batched):
    gen = generator(gold, tag, dtype, seed)
    got = gen.generate_fibre_positions_batch(2) if batched else \
        [gen.generate_fibre_positions() for _ in range(2)]
    for s in range(2):
        bounds, pos, rad, ori = layers_of(gold, f"lay_{tag}_{s}_")
        b2, p2, r2, o2 = got[s]
        assert np.array_equal(b2, bounds)
        assert o2 == ori
        assert all(np.array_equal(a, b) for a, b in zip(p2, pos))
        assert all(np.array_equal(a, b) for a, b in zip(r2, rad))


@pytest.mark.parametrize("tag,dtype", [("f32", np.float32), ("f64", np.float64)])
def test_voxel_oracle_matches_reference(gold, tag, dtype):
    from oracle import fibres_oracle

    for s in range(2):
        _, pos, rad, ori = layers_of(gold, f"lay_{tag}_{s}_")
        lame = fibres_oracle.material_properties(tuple(gold["lay_grid"]), 0.01, VALUES, pos, rad,
                                                 ori, dtype=dtype)
        ref = gold[f"lay_{tag}_{s}_lame"]
        assert lame.dtype == ref.dtype
        assert np.array_equal(lame, ref)


def _load_ref():
    lib = ctypes.CDLL(REF_LIB)
    D = ctypes.POINTER(ctypes.c_double)
    lib.initialise_rng.argtypes = [ctypes.c_uint, ctypes.POINTER(ctypes.c_uint), ctypes.c_char_p]
    lib.move_fibres.argtypes = [ctypes.c_uint, D, D, D, ctypes.c_uint, ctypes.c_double,
                                ctypes.c_uint, ctypes.POINTER(ctypes.c_uint), ctypes.c_char_p]
    lib.dist_periodic.argtypes = [ctypes.c_uint, D, D, D, D]
    return lib


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference library not built")
def test_matches_reference_library_on_random_sets(fibres_lib):
    from jaxmaterials_b200.data.distributions_fibres import initial_lattice

    ref = _load_ref()
    D = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
    rng = np.random.default_rng(2024)
    for trial in range(12):
        box = np.array([rng.uniform(0.04, 0.3), rng.uniform(0.03, 0.08)])
        vf = rng.uniform(0.2, 0.42)
        x0 = initial_lattice(box, 7.5e-3, vf)
        if x0.shape[0] < 3:
            continue
        r = rng.uniform(5e-3, 1e-2, size=x0.shape[0])
        seed = int(rng.integers(0, 2**31))
        res = []
        for lib in (ref, fibres_lib):
            n = ctypes.c_uint()
            st = ctypes.create_string_buffer(10000)
            lib.initialise_rng(seed, ctypes.byref(n), st)
            x = np.ascontiguousarray(x0.copy())
            lib.move_fibres(x.shape[0], D(box), D(r), D(x), 30, 3e-4, 5000, ctypes.byref(n), st)
            res.append((x, st.raw[:n.value]))
        assert np.array_equal(res[0][0], res[1][0]), trial
        assert res[0][1] == res[1][1], trial
        p = np.ascontiguousarray(rng.uniform(0, 1, 2) * box)
        d = [np.empty(x0.shape[0]), np.empty(x0.shape[0])]
        for lib, out in zip((ref, fibres_lib), d):
            lib.dist_periodic(x0.shape[0], D(p), D(np.ascontiguousarray(x0)), D(box), D(out))
        assert np.array_equal(d[0], d[1])


def test_dist_periodic_minimum_image(fibres_lib):
    from jaxmaterials_b200 import _lib

    rng = np.random.default_rng(3)
    box = np.array([0.7, 0.3])
    q = np.ascontiguousarray(rng.uniform(size=(50, 2)) * box)
    p = np.ascontiguousarray(rng.uniform(size=2) * box)
    out = np.empty(50)
    fibres_lib.dist_periodic(50, p.ctypes.data_as(_lib.c_double_p), q.ctypes.data_as(_lib.c_double_p),
                             box.ctypes.data_as(_lib.c_double_p), out.ctypes.data_as(_lib.c_double_p))
    d = np.abs(p - q)
    d = np.minimum(d, box - d)
    assert np.allclose(out, np.hypot(d[:, 0], d[:, 1]), rtol=0, atol=1e-15)


def test_batch_equals_single_sets_on_any_thread_count(fibres_lib):
    from jaxmaterials_b200.data.distributions_fibres import (FibreDistribution2d,
                                                             initial_lattice, place_batch)

    rng = np.random.default_rng(8)
    boxes, radii, starts, single = [], [], [], []
    for i in range(7):
        box = np.array([rng.uniform(0.05, 0.2), rng.uniform(0.03, 0.06)])
        rd = radius_dist(40 + i)
        fd = FibreDistribution2d(box, volume_fraction=0.3, r_fibre_dist=rd)
        x, r = next(iter(fd))
        single.append(x)
        boxes.append(box)
        radii.append(r)
        starts.append(initial_lattice(box, 7.5e-3, 0.3))
    for threads in (1, 3, 0):
        moved = place_batch(boxes, radii, starts, threads=threads)
        assert all(np.array_equal(a, b) for a, b in zip(moved, single))


def test_batch_reports_sets_that_do_not_fit(fibres_lib):
    from jaxmaterials_b200.data.distributions_fibres import place_batch

    box = np.array([1.0, 1.0])
    x = np.array([[0.1, 0.1], [0.5, 0.5], [0.9, 0.2], [0.3, 0.8]])
    r = np.full(4, 0.4)  # four discs of radius 0.4 cannot fit a unit torus apart
    with pytest.raises(RuntimeError, match="still overlap"):
        place_batch([box], [r], [x], it_max_ovlap=20, max_sweeps=3)
    with pytest.raises(ValueError):
        place_batch([box], [r[:2]], [x[:2]])
