"""CPU oracle of the warm-start spectral network (test infrastructure only: tests import it
to check the CUDA kernels; the product never does).

The reference has no learned component (it generates C_eff datasets for a separately
trained model, src/jaxmaterials/data/data.py:148-186, and trains elsewhere), so this is
a NumPy FP64 restatement of the network the product defines, parity unpinned against
the reference: the pointwise layers, the per-mode complex channel mixing on the retained
modes and numpy.fft's rfftn/irfftn, with the parameters given as arrays (the product's
BF16-rounded weights are passed in already rounded). Gradients are checked against
central finite differences of this forward.
"""

import numpy as np


def gelu(x):
    from scipy.special import erf

    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def retained_index(n, modes):
    """Index arrays (kx, ky, kz) of the retained modes, in the kernels' mode order."""
    mx, my, mz = modes
    ix = np.arange(mx)
    iy = np.arange(my)
    kx = np.where(ix < mx // 2, ix, n[0] - mx + ix)
    ky = np.where(iy < my // 2, iy, n[1] - my + iy)
    kz = np.arange(mz)
    KX, KY, KZ = np.meshgrid(kx, ky, kz, indexing="ij")
    return KX.ravel(), KY.ravel(), KZ.ravel()


def pointwise(x, w, b, add=None, act=False):
    """x [B, cin, ...] -> [B, cout, ...]."""
    y = np.einsum("oi,bi...->bo...", w, x) + b.reshape((1, -1) + (1,) * (x.ndim - 2))
    if add is not None:
        y = y + add
    return gelu(y) if act else y


def spectral(h, w, modes):
    """irfftn(R . rfftn(h)) with R = w[..., 0] + i w[..., 1] on the retained modes."""
    n = h.shape[2:]
    xh = np.fft.rfftn(h, axes=(-3, -2, -1))
    kx, ky, kz = retained_index(n, modes)
    wc = w[..., 0] + 1j * w[..., 1]                  # [modes, cin, cout]
    sel = xh[:, :, kx, ky, kz]                       # [B, cin, modes]
    out = np.einsum("bim,mio->bom", sel, wc)
    yh = np.zeros((h.shape[0], wc.shape[2]) + xh.shape[2:], dtype=complex)
    yh[:, :, kx, ky, kz] = out
    return np.fft.irfftn(yh, s=n, axes=(-3, -2, -1))


def forward(params, a, layers, modes):
    """a [B, 2, nx, ny, nz] -> [B, out, nx, ny, nz] (FP64)."""
    h = pointwise(a, params["lift_w"], params["lift_b"])
    for l in range(layers):
        s = spectral(h, params[f"spec{l}"], modes)
        h = pointwise(h, params[f"w{l}"], params[f"b{l}"], add=s, act=True)
    return pointwise(h, params["proj_w"], params["proj_b"])


def fd_gradient(params, a, layers, modes, loss_weights, name, index, h=1e-3):
    """Central difference of L = sum(loss_weights * forward) w.r.t. params[name][index]."""
    p = {k: v.copy() for k, v in params.items()}
    base = p[name][index]
    p[name][index] = base + h
    lp = float(np.sum(loss_weights * forward(p, a, layers, modes)))
    p[name][index] = base - h
    lm = float(np.sum(loss_weights * forward(p, a, layers, modes)))
    return (lp - lm) / (2.0 * h)


def inverse_half_spectrum(yh, n):
    """(torch) Real field of a half spectrum [..., nx, ny, nz/2+1] that need not be Hermitian in
    its kz = 0 and kz = nz/2 planes: inverse DFT over x and y, then the C2R transform along
    z with the imaginary parts of those two planes dropped, i.e. the real part of the
    planes' contribution (numpy.fft.irfftn semantics, well defined for any input)."""
    import torch

    z = torch.fft.ifftn(yh, dim=(-3, -2))
    nzh = z.shape[-1]
    keep = torch.ones(nzh, device=z.device, dtype=z.real.dtype)
    keep[0] = 0.0
    if n[2] % 2 == 0:
        keep[nzh - 1] = 0.0
    z = torch.complex(z.real, z.imag * keep)
    return torch.fft.irfft(z, n=n[2], dim=-1)
