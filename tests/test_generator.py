"""Fibre microstructure generator: determinism and exact voxel indices against an
independent per-voxel evaluation of the inclusion predicate."""

import numpy as np

from jaxmaterials_b200.data import fibres


def brute_indicator(st):
    nx, ny, nz = st.n
    hx, hy, hz = (st.extents[d] / st.n[d] for d in range(3))
    out = np.zeros(st.n, dtype=bool)
    for layer in st.layers:
        r2 = layer.radius * layer.radius
        for k in range(layer.k_lo, layer.k_hi):
            z = (k + 0.5) * hz
            for i in range(nx):
                for j in range(ny):
                    if layer.orientation == 0:
                        u, lu = (j + 0.5) * hy, st.extents[1]
                    else:
                        u, lu = (i + 0.5) * hx, st.extents[0]
                    for uc, zc in layer.centres:
                        d = u - uc
                        if d > 0.5 * lu:
                            d -= lu
                        if d < -0.5 * lu:
                            d += lu
                        dz = z - zc
                        if d * d + dz * dz < r2:
                            out[i, j, k] = True
                            break
    return out


def test_deterministic():
    a = fibres.generate_layered_fibres(24, 3, 2.5, 0.4, seed=11)
    b = fibres.generate_layered_fibres(24, 3, 2.5, 0.4, seed=11)
    for la, lb in zip(a.layers, b.layers):
        assert np.array_equal(la.centres, lb.centres)
    assert np.array_equal(fibres.fibre_indicator(a), fibres.fibre_indicator(b))


def test_exact_voxels_against_brute_force():
    st = fibres.generate_layered_fibres((20, 16, 12), 2, 3.0, 0.4, seed=5)
    assert np.array_equal(fibres.fibre_indicator(st), brute_indicator(st))


def test_no_overlap_and_volume_fraction():
    st = fibres.config_structure("c1", seed=0)
    for layer in st.layers:
        c = layer.centres
        lu = st.extents[1] if layer.orientation == 0 else st.extents[0]
        for i in range(len(c)):
            d = c[i + 1:, 0] - c[i, 0]
            d = np.where(d > lu / 2, d - lu, d)
            d = np.where(d < -lu / 2, d + lu, d)
            assert np.all(d * d + (c[i + 1:, 1] - c[i, 1]) ** 2 >= 4 * layer.radius**2)
        assert layer.volume_fraction >= 0.40
    lm, mu = fibres.lame_fields(st)
    assert set(np.unique(lm)) == {np.float32(2.593), np.float32(19.44)}
    assert lm.shape == (32, 32, 32)
    assert np.array_equal(lm == np.float32(19.44), mu == np.float32(29.17))
