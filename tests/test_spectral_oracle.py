"""CPU checks of the warm-start network's oracle, including the torch restatement of the
inverse transform that the GPU tests' torch reference uses (no GPU)."""

import numpy as np

from oracle import spectral_net_oracle as SO


def test_inverse_half_spectrum_is_numpy_irfftn():
    import torch

    rng = np.random.default_rng(0)
    for n in [(8, 6, 10), (7, 9, 5)]:
        shape = (2, 3, n[0], n[1], n[2] // 2 + 1)
        yh = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        ref = np.fft.irfftn(yh, s=n, axes=(-3, -2, -1))
        got = SO.inverse_half_spectrum(torch.as_tensor(yh), n).numpy()
        assert np.abs(got - ref).max() < 1e-12


def test_retained_modes_are_distinct_and_low():
    kx, ky, kz = SO.retained_index((64, 64, 64), (12, 12, 12))
    assert len(set(zip(kx, ky, kz))) == 12 ** 3
    signed = np.where(kx >= 32, kx - 64, kx)
    assert signed.min() == -6 and signed.max() == 5 and kz.max() == 11


def test_spectral_layer_is_a_fourier_multiplier():
    """With every mode retained and each mode's weight the identity, the spectral branch
    reproduces its input (rfftn then irfftn)."""
    rng = np.random.default_rng(1)
    n = (6, 4, 6)
    h = rng.standard_normal((1, 3) + n)
    modes = (6, 4, 4)
    w = np.zeros((np.prod(modes), 3, 3, 2))
    w[:, np.arange(3), np.arange(3), 0] = 1.0
    np.testing.assert_allclose(SO.spectral(h, w, modes), h, atol=1e-12)


def test_oracle_gradient_is_consistent():
    """The oracle's central differences are linear in the loss weights (sanity of fd)."""
    rng = np.random.default_rng(2)
    n = (4, 4, 4)
    modes = (2, 2, 2)
    p = {"lift_w": rng.standard_normal((3, 2)), "lift_b": rng.standard_normal(3),
         "spec0": rng.standard_normal((8, 3, 3, 2)) * 0.1, "w0": rng.standard_normal((3, 3)),
         "b0": rng.standard_normal(3), "proj_w": rng.standard_normal((2, 3)),
         "proj_b": rng.standard_normal(2)}
    a = rng.standard_normal((1, 2) + n)
    w1 = rng.standard_normal((1, 2) + n)
    w2 = rng.standard_normal((1, 2) + n)
    g1 = SO.fd_gradient(p, a, 1, modes, w1, "w0", (1, 2))
    g2 = SO.fd_gradient(p, a, 1, modes, w2, "w0", (1, 2))
    g12 = SO.fd_gradient(p, a, 1, modes, w1 + w2, "w0", (1, 2))
    assert abs(g12 - g1 - g2) < 1e-8 * max(1.0, abs(g12))
