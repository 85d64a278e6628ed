"""Effective stiffness of many microstructures on one GPU (lsb_c_eff_batch).

The reference computes a dataset's C_eff one structure and one load case at a time
(src/jaxmaterials/data/data.py:148-186). Here the whole dataset goes to the library in
one call: structures of equal grid are solved together (six load cases each, every
instance with its own reference medium and convergence), grids of different sizes
concurrently on separate streams.
"""

import ctypes

import numpy as np

from .. import _lib
from .lippmann_schwinger import PRECISIONS


def c_eff_batch(lmbdas, mus, grid_specs, rtol=1e-6, atol=1e-20, maxiter=2000, depth=5,
                precision="mixed", memory_gb=0.0):
    """C_eff of every structure.

    lmbdas, mus: sequences of host arrays of shape grid_specs[i].shape (any float dtype;
    converted to float32 C order). grid_specs: one GridSpec per structure, or one for all.
    Returns ``(C, iters, status)`` with C of shape (n, 6, 6) (row k = mean stress for the
    unit strain e_k, tensor shear), iters and status of shape (n, 6).
    Raises if any solve did not converge.
    """
    n = len(lmbdas)
    if len(mus) != n:
        raise ValueError("lmbdas and mus differ in length")
    if not isinstance(grid_specs, (list, tuple)):
        grid_specs = [grid_specs] * n
    if len(grid_specs) != n:
        raise ValueError("one grid spec per structure expected")
    lib = _lib.load()
    voxels = np.zeros((max(n, 1), 3), dtype=np.int32)
    extents = np.zeros((max(n, 1), 3), dtype=np.float64)
    keep = []
    lp = (ctypes.c_void_p * max(n, 1))()
    mp = (ctypes.c_void_p * max(n, 1))()
    for i, (lm, mu, g) in enumerate(zip(lmbdas, mus, grid_specs)):
        voxels[i] = (g.nx, g.ny, g.nz)
        extents[i] = (g.Lx, g.Ly, g.Lz)
        a = np.ascontiguousarray(lm, dtype=np.float32)
        b = np.ascontiguousarray(mu, dtype=np.float32)
        if a.shape != g.shape or b.shape != g.shape:
            raise ValueError(f"structure {i}: expected fields of shape {g.shape}")
        keep += [a, b]
        lp[i] = a.ctypes.data
        mp[i] = b.ctypes.data
    c = np.zeros((max(n, 1), 6, 6), dtype=np.float64)
    iters = np.zeros((max(n, 1), 6), dtype=np.int32)
    status = np.zeros((max(n, 1), 6), dtype=np.int32)
    rc = lib.lsb_c_eff_batch(
        n, voxels.ctypes.data_as(_lib.c_int_p), extents.ctypes.data_as(_lib.c_double_p),
        ctypes.cast(lp, ctypes.POINTER(ctypes.c_void_p)),
        ctypes.cast(mp, ctypes.POINTER(ctypes.c_void_p)), int(depth), PRECISIONS[precision],
        float(rtol), float(atol), int(maxiter), float(memory_gb),
        c.ctypes.data_as(_lib.c_double_p), iters.ctypes.data_as(_lib.c_int_p),
        status.ctypes.data_as(_lib.c_int_p))
    _lib.check(rc, "lsb_c_eff_batch")
    c, iters, status = c[:n], iters[:n], status[:n]
    bad = np.argwhere(status != 1)
    if len(bad):
        i, k = bad[0]
        raise RuntimeError(f"structure {i}, load case {k} did not converge "
                           f"(status {status[i, k]}, {iters[i, k]} iterations)")
    return c, iters, status
