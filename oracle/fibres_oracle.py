"""CPU oracle of the voxelisation of layered fibre composites (TEST INFRASTRUCTURE ONLY:
the product never imports this module).

Restates ``LayeredFibresDatasetGenerator.material_properties``
(src/jaxmaterials/data/data.py:267-314) in NumPy with the reference's evaluation order:
voxel centres ``L/N (1/2 + i)``, every field set to the matrix value, the void layers
(``z < d_void`` or ``z > L_z - d_void``) adding ``void - matrix`` once, then every fibre
adding ``fibre - matrix`` where ``(u - u0)**2 + (z - z0)**2 < r**2`` (u = x for orientation
0, y for 1), each in-place addition rounded to the field's dtype. Pinned against the
reference's own outputs in tests/golden/reference_fibres.npz.
"""

import numpy as np


def material_properties(grid, d_void, values, fibre_positions, fibre_radii, fibre_orientations,
                        dtype=np.float64):
    """(mu, lambda) at the voxel centres, shape (2, nx, ny, nz).

    grid: (nx, ny, nz, Lx, Ly, Lz); values = (mu_void, lambda_void, mu_fibre, lambda_fibre,
    mu_material, lambda_material)."""
    nx, ny, nz, Lx, Ly, Lz = grid
    nx, ny, nz = int(nx), int(ny), int(nz)
    X, Y, Z = np.meshgrid(Lx / nx * (1 / 2 + np.arange(nx)), Ly / ny * (1 / 2 + np.arange(ny)),
                          Lz / nz * (1 / 2 + np.arange(nz)), indexing="ij")
    void = (Z < d_void) + (Z > Lz - d_void)
    out = np.zeros((2, nx, ny, nz), dtype=dtype)
    for c in range(2):
        v_void, v_fibre, v_mat = values[c], values[2 + c], values[4 + c]
        out[c] = v_mat
        out[c] += void * (v_void - v_mat)
        for pos, rad, orientation in zip(fibre_positions, fibre_radii, fibre_orientations):
            u = Y if orientation else X
            for p, r in zip(pos, rad):
                out[c] += ((u - p[0]) ** 2 + (Z - p[1]) ** 2 < r ** 2) * (v_fibre - v_mat)
    return out
