"""CPU oracle of the voxelisation of layered fibre composites (TEST INFRASTRUCTURE ONLY:
the product never imports this module).

Restates ``LayeredFibresDatasetGenerator.material_properties``
(src/jaxmaterials/data/data.py:267-314) in NumPy with the reference's evaluation order:
voxel centres ``L/N (1/2 + i)``, every field set to the matrix value, the void layers
(``z < d_void`` or ``z > L_z - d_void``) adding ``void - matrix`` once, then every fibre
adding ``fibre - matrix`` where ``(u - u0)**2 + (z - z0)**2 < r**2`` (u = x for orientation
0, y for 1), each in-place addition rounded to the field's dtype. Pinned against the
reference's own outputs in tests/golden/reference_fibres.npz.

Also restates the reference's NumPy fibre-shaking path (``FibreDistribution2d`` with
``fast_code=False``, src/jaxmaterials/data/distributions_fibres.py:205-295), which the
product does not provide: the same algorithm as the C++ library, driven by a NumPy
generator, pinned to the reference's output in the same fixture.
"""

import itertools

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


def dist_periodic(p, q, domain_size):
    """Minimum-image distances from point p to every row of q, as the reference's NumPy
    ``_dist_periodic`` (distributions_fibres.py:268-295): the smallest of the nine
    periodic images' Euclidean distances."""
    domain_size = np.asarray(domain_size, dtype=np.float64)
    n = q.shape[0]
    d = np.empty(shape=(9, n))
    for j, off in enumerate(itertools.product([-domain_size[0], 0, +domain_size[0]],
                                              [-domain_size[1], 0, +domain_size[1]])):
        d[j, :] = np.sqrt(np.sum((p + np.asarray(off) - q) ** 2, axis=1))
    return np.min(d, axis=0)


def move_fibres(rng, x, r, domain_size, num_repeats=30, it_max_ovlap=5000, eps_fibres=3.0e-4):
    """The reference's NumPy shaking path (distributions_fibres.py:205-266) with generator
    ``rng`` (the instance's ``default_rng(seed)``): fibres visited in a random order, each
    moved to a random point within the mean distance to its three nearest neighbours until
    its gap to every other fibre is at least ``eps_fibres``; after ``it_max_ovlap`` trials
    the trial with the fewest overlaps is kept and another sweep is forced. At least
    ``num_repeats`` sweeps. Moves x (n, 2) in place and returns it."""
    domain_size = np.asarray(domain_size, dtype=np.float64)
    n = r.shape[0]
    order = rng.permutation(range(n))
    overlap = True
    sweep = 0
    while overlap or sweep < num_repeats:
        overlap = False
        for j in range(n):
            me = order[j]
            p = x[me, :]
            d = dist_periodic(p, x, domain_size)
            d[me] = np.inf
            reach = np.mean(sorted(d)[:3])
            gap, trials, fewest = 0, 0, np.inf
            while gap < eps_fibres:
                u_r = rng.uniform(low=0, high=reach)
                u_t = rng.uniform(low=0, high=2 * np.pi)
                trial = p + u_r * np.asarray([np.cos(u_t), np.sin(u_t)])
                for k in range(2):
                    while trial[k] < 0:
                        trial[k] += domain_size[k]
                    while trial[k] > domain_size[k]:
                        trial[k] -= domain_size[k]
                d = dist_periodic(trial, x, domain_size) - r[me] - r
                d[me] = np.inf
                gap = np.min(d)
                overlaps = np.count_nonzero(d < 0)
                if overlaps < fewest:
                    best, fewest = trial, overlaps
                trials += 1
                if trials > it_max_ovlap:
                    trial = best
                    overlap = True
                    break
            x[me, :] = trial[:]
        sweep += 1
    return x
