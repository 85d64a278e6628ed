"""Batched solves: instances grouped by microstructure (lsb_set_lame_group) and the
dataset entry point lsb_c_eff_batch over structures of uneven grid sizes.

Every instance of a grouped launch computes exactly what it computes alone (same kernels,
its own reference medium and stop decision), so grouped and separate solves agree bit
for bit; C_eff is checked against the FP64 oracle at 1e-5 relative (Frobenius).
"""

import numpy as np
import pytest

from oracle import ls_oracle as O

pytestmark = pytest.mark.gpu


def fibre_set(sizes, seed=11):
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.data import fibres as F

    rng = np.random.default_rng(seed)
    out = []
    for i, n in enumerate(sizes):
        st = F.generate_layered_fibres(n, int(rng.integers(2, 5)), float(rng.uniform(2.0, 3.5)),
                                       float(rng.uniform(0.3, 0.45)), int(rng.integers(1 << 30)))
        lm, mu = F.lame_fields(st)
        out.append((lm, mu, GridSpec(n, n, n, float(n), float(n), float(n))))
    return out


@pytest.mark.parametrize("n,depth", [(32, 5), (48, 0), (24, 5)])
def test_grouped_equals_separate(n, depth):
    import torch
    from jaxmaterials_b200.solver import Solver

    structs = fibre_set([n, n, n], seed=n + depth)
    g = structs[0][2]
    eye = np.eye(6, dtype=np.float32)
    single = Solver(g, batch=6, depth=depth)
    sep = [single.solve(lm, mu, eye, rtol=1e-6, maxiter=3000, want_sigma=False)
           for lm, mu, _ in structs]
    sep_eps = [r.epsilon.clone() for r in sep]
    grouped = Solver(g, batch=18, depth=depth)
    lms = np.stack([s[0] for s in structs])
    mus = np.stack([s[1] for s in structs])
    r = grouped.solve(lms, mus, np.tile(eye, (3, 1)), rtol=1e-6, maxiter=3000, want_sigma=False)
    for i in range(3):
        np.testing.assert_array_equal(r.iters[6 * i:6 * i + 6], sep[i].iters)
        np.testing.assert_array_equal(r.mean_sigma[6 * i:6 * i + 6], sep[i].mean_sigma)
        assert torch.equal(r.epsilon[6 * i:6 * i + 6], sep_eps[i])
    assert (r.status == 1).all()


def test_group_media_are_per_structure():
    """A homogeneous structure next to a heterogeneous one: its own reference medium is
    its material, so its instances stop at the first evaluation."""
    from jaxmaterials_b200.solver import Solver

    (lm, mu, g), = fibre_set([32])
    hom_l = np.full(g.shape, 2.0, np.float32)
    hom_m = np.full(g.shape, 1.5, np.float32)
    s = Solver(g, batch=12, depth=0)
    eye = np.eye(6, dtype=np.float32)
    r = s.solve(np.stack([lm, hom_l]), np.stack([mu, hom_m]), np.tile(eye, (2, 1)),
                rtol=1e-6, maxiter=3000, want_sigma=False)
    assert (r.iters[:6] > 10).all()
    assert (r.iters[6:] == 0).all()
    c_hom = np.diag([2.0 + 3.0, 5.0, 5.0, 3.0, 3.0, 3.0]).astype(np.float64)
    c_hom[:3, :3] += 2.0 - np.diag([2.0] * 3)
    np.testing.assert_allclose(r.mean_sigma[6:], c_hom, rtol=1e-6, atol=1e-6)


def test_c_eff_batch_uneven_sizes():
    from jaxmaterials_b200.solver import c_eff, c_eff_batch

    structs = fibre_set([16, 32, 24, 16, 48, 32, 20], seed=5)
    lms, mus, gs = zip(*structs)
    C, iters, status = c_eff_batch(lms, mus, list(gs), rtol=1e-6, maxiter=3000, depth=5)
    assert C.shape == (7, 6, 6) and (status == 1).all()
    # each structure exactly as the single-structure path computes it
    for i, (lm, mu, g) in enumerate(structs):
        c1, it1, _ = c_eff(lm, mu, g, rtol=1e-6, maxiter=3000, depth=5)
        np.testing.assert_array_equal(iters[i], it1)
        np.testing.assert_array_equal(C[i], c1)
    # and within 1e-5 of the FP64 oracle (two small ones)
    for i in (0, 6):
        lm, mu, g = structs[i]
        og = O.Grid(g.nx, g.ny, g.nz, g.Lx, g.Ly, g.Lz)
        c64, _ = O.c_eff(lm.astype(np.float64), mu.astype(np.float64), og, rtol=1e-9,
                         maxiter=5000, depth=5)
        assert np.linalg.norm(C[i] - c64) / np.linalg.norm(c64) < 1e-5


def test_c_eff_batch_memory_chunks():
    """A memory budget that holds one structure at a time gives the same answers."""
    from jaxmaterials_b200.solver import c_eff_batch

    structs = fibre_set([32, 32, 32, 16], seed=8)
    lms, mus, gs = zip(*structs)
    full = c_eff_batch(lms, mus, list(gs), depth=5, maxiter=3000)
    tight = c_eff_batch(lms, mus, list(gs), depth=5, maxiter=3000, memory_gb=0.05)
    np.testing.assert_array_equal(full[0], tight[0])
    np.testing.assert_array_equal(full[1], tight[1])


def test_c_eff_batch_graph_equals_threads(monkeypatch):
    """The whole dataset as one CUDA graph (the default schedule: every bucket a chain of
    its chunks' solves, each loop a device-stopped WHILE node) gives the threaded
    schedule's C_eff, iterations and status bit for bit, also for instances continued in
    FP64 after an FP32 stall (rtol 2e-7 lies below the FP32 floor at these sizes)."""
    from jaxmaterials_b200.solver import c_eff_batch

    structs = fibre_set([16, 32, 24, 16, 32, 48], seed=3)
    lms, mus, gs = zip(*structs)
    out = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("LSB_BATCH_GRAPH", mode)
        for rtol in (1e-6, 2e-7):
            out[mode, rtol] = c_eff_batch(lms, mus, list(gs), rtol=rtol, maxiter=3000, depth=5)
    for rtol in (1e-6, 2e-7):
        g, t = out["1", rtol], out["0", rtol]
        np.testing.assert_array_equal(g[0], t[0])
        np.testing.assert_array_equal(g[1], t[1])
        np.testing.assert_array_equal(g[2], t[2])
        assert (g[2] == 1).all()
    # FP64 solves (FP64 from the first update) in either mode, against the FP32-start ones
    f64 = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("LSB_BATCH_GRAPH", mode)
        f64[mode] = c_eff_batch(lms[:2], mus[:2], list(gs[:2]), rtol=1e-9, maxiter=3000, depth=5,
                                precision="fp64")
    np.testing.assert_array_equal(f64["1"][0], f64["0"][0])
    rel = np.linalg.norm(f64["1"][0] - out["1", 2e-7][0][:2]) / np.linalg.norm(f64["1"][0])
    assert rel < 1e-5


def test_c_eff_batch_graph_buckets_by_extents(monkeypatch):
    """Equal voxel counts with different extents are different buckets (their wave vectors
    differ); single-structure buckets and a one-structure dataset take the graph path too:
    the same results as the threaded schedule and as the single-structure path."""
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.solver import c_eff, c_eff_batch

    structs = fibre_set([16, 16, 24], seed=21)
    lms, mus, gs = zip(*structs)
    gs = [gs[0], GridSpec(16, 16, 16, 16.0, 24.0, 8.0), gs[2]]
    out = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("LSB_BATCH_GRAPH", mode)
        out[mode] = c_eff_batch(lms, mus, gs, rtol=1e-6, maxiter=3000, depth=5)
        one = c_eff_batch(lms[:1], mus[:1], gs[:1], rtol=1e-6, maxiter=3000, depth=5)
        np.testing.assert_array_equal(one[0][0], out[mode][0][0])
    for k in range(3):
        np.testing.assert_array_equal(out["1"][k], out["0"][k])
    for i in range(3):
        c1, it1, _ = c_eff(lms[i], mus[i], gs[i], rtol=1e-6, maxiter=3000, depth=5)
        np.testing.assert_array_equal(out["1"][0][i], c1)
        np.testing.assert_array_equal(out["1"][1][i], it1)
    assert not np.allclose(out["1"][0][0], out["1"][0][1])  # the extents matter


def test_c_eff_batch_rejects_bad_input():
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200._lib import LibraryError
    from jaxmaterials_b200.solver import c_eff_batch

    g = GridSpec(16, 16, 16, 16.0, 16.0, 16.0)
    a = np.ones(g.shape, np.float32)
    with pytest.raises(LibraryError):
        c_eff_batch([a], [a], [g], depth=9)
    with pytest.raises(ValueError):
        c_eff_batch([a], [a[:8]], [g])


def test_dataset_generation(tmp_path):
    """Generated dataset rows equal the FP64 oracle's C_eff of the stored fields ([mu, lambda]
    channel order; the reference's dataset loop, data.py:178-186) within 1e-5, equal the
    single-structure C_eff of the library, and survive a save/load round trip."""
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.data import dataset as D
    from jaxmaterials_b200.solver import c_eff
    from oracle import ls_oracle as O

    lame, sig, dom, iters = D.generate(3, n=16, seed=4)
    assert lame.shape == (3, 2, 16, 16, 16) and sig.shape == (3, 6, 6) and (iters > 0).all()
    g = GridSpec(16, 16, 16, 16.0, 16.0, 16.0)
    og = O.Grid(16, 16, 16, 16.0, 16.0, 16.0)
    for j in range(3):
        c, _, _ = c_eff(lame[j, 1], lame[j, 0], g, rtol=1e-6, depth=5)
        np.testing.assert_allclose(sig[j], c.astype(np.float32), rtol=1e-6, atol=1e-6)
        ref, _ = O.c_eff(lame[j, 1].astype(np.float64), lame[j, 0].astype(np.float64), og,
                         rtol=1e-6, atol=1e-20, depth=5, maxiter=2000, dtype=np.float64)
        assert np.linalg.norm(sig[j] - ref) / np.linalg.norm(ref) < 1e-5
    path = tmp_path / "d.npz"
    D.save(path, lame, sig, dom)
    ds = D.LayeredFibresDataset(path)
    np.testing.assert_array_equal(ds[2][1], sig[2])
