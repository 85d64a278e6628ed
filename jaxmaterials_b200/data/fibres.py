"""Seeded layered fibre microstructures and their voxelisation to Lame fields.

The reference generates layered cross-ply fibre composites
(``src/jaxmaterials/data/data.py:188-314``) with a fibre-shaking algorithm. The
workloads here use a simpler, fully seeded random-sequential-adsorption (RSA) layout:

* the periodic N^3 box is cut into ``nlayers`` layers along z; layer j covers the voxel
  planes ``[j*nz//nlayers, (j+1)*nz//nlayers)``;
* fibres in even layers run along x, in odd layers along y (0/90 cross-ply);
* in a layer, fibre centres (u, z) are drawn uniformly (u in-plane and periodic, z inside
  the layer) and rejected if closer than 2r to an accepted centre (periodic in u), until
  the fibre voxel fraction of the layer reaches the target or ``max_attempts`` is hit;
* fibres are clipped at their layer's z planes.

Voxel (i, j, k) has centre ((i+1/2) hx, (j+1/2) hy, (k+1/2) hz) and lies in a fibre of
radius r centred at (u_c, z_c) when du^2 + dz^2 < r^2 (strict, as in
``src/jaxmaterials/data/data.py:309-311``), where du is the periodic minimum image of
u - u_c computed as ``d = u - u_c; d -= L if d > L/2; d += L if d < -L/2`` in FP64.
Channel order of the returned fields is (lambda, mu).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

#: Lame parameters (GPa) of the matrix and of the fibres used by the workloads.
MATRIX_LAME = (2.593, 1.111)
FIBRE_LAME = (19.44, 29.17)


@dataclass
class FibreLayer:
    k_lo: int
    k_hi: int
    orientation: int  # 0: fibres along x; 1: along y
    centres: np.ndarray = field(default_factory=lambda: np.zeros((0, 2)))  # (n, 2): (u, z)
    radius: float = 0.0
    volume_fraction: float = 0.0


@dataclass
class FibreStructure:
    n: tuple
    extents: tuple
    layers: list

    @property
    def volume_fraction(self):
        nz = self.n[2]
        return sum(l.volume_fraction * (l.k_hi - l.k_lo) for l in self.layers) / nz


def _periodic(d, length):
    d = np.where(d > 0.5 * length, d - length, d)
    return np.where(d < -0.5 * length, d + length, d)


def _layer_mask(layer, n, extents):
    """Boolean (n_u, n_layer_z) cross-section of the fibres in ``layer``."""
    ax = 1 if layer.orientation == 0 else 0  # in-plane periodic axis u
    nu, lu = n[ax], extents[ax]
    hu, hz = lu / nu, extents[2] / n[2]
    u = (np.arange(nu) + 0.5) * hu
    z = (np.arange(layer.k_lo, layer.k_hi) + 0.5) * hz
    mask = np.zeros((nu, layer.k_hi - layer.k_lo), dtype=bool)
    r2 = layer.radius * layer.radius
    for uc, zc in layer.centres:
        du = _periodic(u - uc, lu)
        dz = z - zc
        mask |= (du[:, None] * du[:, None] + dz[None, :] * dz[None, :]) < r2
    return mask


def generate_layered_fibres(n, nlayers, radius, volume_fraction, seed, extents=None,
                            max_attempts=20000):
    """RSA layout of a layered cross-ply composite on an n^3 (or n=(nx,ny,nz)) grid.

    ``radius`` is in length units (voxels when ``extents`` defaults to the voxel counts).
    The same ``seed`` always gives the same layout."""
    n = (n, n, n) if np.isscalar(n) else tuple(int(v) for v in n)
    extents = tuple(float(v) for v in n) if extents is None else tuple(extents)
    rng = np.random.default_rng(seed)
    layers = []
    for j in range(nlayers):
        k_lo, k_hi = (j * n[2]) // nlayers, ((j + 1) * n[2]) // nlayers
        layer = FibreLayer(k_lo, k_hi, j % 2, radius=float(radius))
        ax = 1 if layer.orientation == 0 else 0
        lu, nu = extents[ax], n[ax]
        hu, hz = lu / nu, extents[2] / n[2]
        z_lo, z_hi = k_lo * hz, k_hi * hz
        u = (np.arange(nu) + 0.5) * hu
        z = (np.arange(k_lo, k_hi) + 0.5) * hz
        mask = np.zeros((nu, k_hi - k_lo), dtype=bool)
        total = mask.size
        centres = []
        r2 = float(radius) * float(radius)
        attempts = 0
        while mask.sum() < volume_fraction * total and attempts < max_attempts:
            attempts += 1
            uc = rng.uniform(0.0, lu)
            zc = rng.uniform(z_lo, z_hi)
            if centres:
                c = np.asarray(centres)
                du = _periodic(c[:, 0] - uc, lu)
                dz = c[:, 1] - zc
                if np.any(du * du + dz * dz < 4.0 * r2):
                    continue
            centres.append((uc, zc))
            du = _periodic(u - uc, lu)
            dz = z - zc
            mask |= (du[:, None] * du[:, None] + dz[None, :] * dz[None, :]) < r2
        layer.centres = np.asarray(centres).reshape(-1, 2)
        layer.volume_fraction = float(mask.sum()) / total
        layers.append(layer)
    return FibreStructure(n, extents, layers)


def fibre_indicator(structure):
    """Boolean (nx, ny, nz) array, True in fibre voxels."""
    nx, ny, nz = structure.n
    ind = np.zeros((nx, ny, nz), dtype=bool)
    for layer in structure.layers:
        mask = _layer_mask(layer, structure.n, structure.extents)
        if layer.orientation == 0:  # along x: cross-section (y, z)
            ind[:, :, layer.k_lo:layer.k_hi] |= mask[None, :, :]
        else:  # along y: cross-section (x, z)
            ind[:, :, layer.k_lo:layer.k_hi] |= mask[:, None, :]
    return ind


def lame_fields(structure, matrix=MATRIX_LAME, fibre=FIBRE_LAME, dtype=np.float32):
    """(lambda, mu) fields of shape (nx, ny, nz) for a fibre structure."""
    ind = fibre_indicator(structure)
    lmbda = np.where(ind, fibre[0], matrix[0]).astype(dtype)
    mu = np.where(ind, fibre[1], matrix[1]).astype(dtype)
    return lmbda, mu


def config_structure(name, seed=0):
    """Named workloads: ``"c1"`` 32^3, 2 layers, r=3, vf 0.40; ``"c2_128"`` / ``"c2_256"``
    128^3 / 256^3, 4 layers, r=4, vf 0.45; ``"c4"`` 64^3, 4 layers, r=3, vf 0.40."""
    table = {
        "c1": (32, 2, 3.0, 0.40),
        "c2_128": (128, 4, 4.0, 0.45),
        "c2_256": (256, 4, 4.0, 0.45),
        "c4": (64, 4, 3.0, 0.40),
    }
    n, nl, r, vf = table[name]
    return generate_layered_fibres(n, nl, r, vf, seed)


def batch_structure_params(count, seed):
    """Per-structure parameters of the batched workload: N in {32,48,64,96,128},
    2-6 layers, radius 2-5 voxels, volume fraction 0.30-0.55, one seed each."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        out.append(
            dict(
                n=int(rng.choice([32, 48, 64, 96, 128])),
                nlayers=int(rng.integers(2, 7)),
                radius=float(rng.uniform(2.0, 5.0)),
                volume_fraction=float(rng.uniform(0.30, 0.55)),
                seed=int(rng.integers(0, 2**31 - 1)),
            )
        )
    return out
