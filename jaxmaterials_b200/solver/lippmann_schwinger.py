"""Lippmann-Schwinger solver entry points (reference:
``src/jaxmaterials/solver/lippmann_schwinger.py``).

* ``lippmann_schwinger_cuda`` keeps the reference wrapper's signature and behaviour
  (``:268-329``): host NumPy arrays in, ``(epsilon, sigma, iter)`` out, ``RuntimeError``
  when ``iter == maxiter``. Unlike the reference wrapper it passes lambda FIRST, matching
  the C signature (the reference passes ``mu`` into the ``lambda`` slot, ``:310-312``).
* ``lippmann_schwinger`` (also exported as ``lippmann_schwinger_jax``) keeps the
  signature of ``lippmann_schwinger_jax`` (``:146-265``) and accepts NumPy arrays or
  CUDA torch tensors; torch tensors stay on the device.
* ``Solver`` is the reusable handle behind both (device buffers, batches of load
  cases sharing lambda and mu), and ``c_eff`` assembles the effective stiffness from the
  six unit loads (``src/jaxmaterials/data/data.py:178-186``).

All arithmetic happens in the CUDA library; this module only marshals arguments.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from .. import _lib
from ..common import GridSpec

__all__ = [
    "Solver",
    "SolveResult",
    "lippmann_schwinger",
    "lippmann_schwinger_jax",
    "lippmann_schwinger_cuda",
    "c_eff",
    "CONVERGED",
    "MAXITER",
    "NONFINITE",
    "STALLED",
    "TIMEOUT",
    "RULE_CUDA",
    "RULE_JAX",
]

# TIMEOUT: a kernel's bounded wait for its own copies ran out; recreate the Solver
CONVERGED, MAXITER, NONFINITE, STALLED, TIMEOUT = 1, 2, 3, 4, 5
RULE_CUDA, RULE_JAX = 0, 1
PRECISIONS = {"fp32": 0, "mixed": 1, "fp64": 2}


def _fptr(a):
    return a.ctypes.data_as(_lib.c_float_p)


def _grid_args(grid_spec):
    voxels = np.array([grid_spec.nx, grid_spec.ny, grid_spec.nz], dtype=np.int32)
    extents = np.array([grid_spec.Lx, grid_spec.Ly, grid_spec.Lz], dtype=np.float32)
    return voxels, extents


def lippmann_schwinger_cuda(lmbda, mu, epsilon_bar, grid_spec, rtol=1e-6, atol=1.0e-20,
                            maxiter=32, verbose=0):
    """Solve through the reference C signature ``lippmann_schwinger_solve``.

    :arg lmbda: Lame parameter lambda, shape (nx, ny, nz)
    :arg mu: Lame parameter mu, shape (nx, ny, nz)
    :arg epsilon_bar: macroscopic strain (6,), Voigt order, tensor shear entries
    :arg grid_spec: grid specification
    :arg rtol, atol: tolerances on the normalised divergence
    :arg maxiter: maximal number of iterations
    :arg verbose: 0 silent, 1 summary, 2 per-iteration table (printed by the library)
    Returns ``(epsilon, sigma, iter)`` as float32 arrays of shape (6, nx, ny, nz).
    """
    lib = _lib.load()
    voxels, extents = _grid_args(grid_spec)
    lm = np.ascontiguousarray(lmbda, dtype=np.float32)
    m = np.ascontiguousarray(mu, dtype=np.float32)
    eb = np.ascontiguousarray(epsilon_bar, dtype=np.float32)
    shape = (6, grid_spec.nx, grid_spec.ny, grid_spec.nz)
    if lm.shape != shape[1:] or m.shape != shape[1:] or eb.shape != (6,):
        raise ValueError("lmbda/mu must have shape (nx, ny, nz) and epsilon_bar shape (6,)")
    epsilon = np.empty(shape, dtype=np.float32)
    sigma = np.empty(shape, dtype=np.float32)
    it = lib.lippmann_schwinger_solve(
        _fptr(lm), _fptr(m), _fptr(eb), _fptr(epsilon), _fptr(sigma),
        voxels.ctypes.data_as(_lib.c_int_p), _fptr(extents), float(rtol), float(atol),
        int(maxiter), int(verbose))
    _lib.check(it, "lippmann_schwinger_solve")
    if it == maxiter:
        raise RuntimeError(f"Solver failed to converge after {maxiter} iterations")
    return epsilon, sigma, it


@dataclass
class SolveResult:
    epsilon: object        # (B, 6, nx, ny, nz) torch tensor on the device
    sigma: object          # same, or None
    iters: np.ndarray      # (B,) updates performed
    status: np.ndarray     # (B,) CONVERGED / MAXITER / NONFINITE
    residual: np.ndarray   # (B,) final criterion value
    mean_sigma: np.ndarray  # (B, 6) FP64 mean stress


class Solver:
    """Reusable solver for one grid: owns the device buffers of ``batch`` instances.

    Instances of one ``solve`` call share lambda and mu (shape (nx, ny, nz)) and differ
    in epsilon_bar (and optionally the warm start), or, with lambda and mu of shape
    (S, nx, ny, nz), instance b reads structure b // (B // S) (B a multiple of S; e.g.
    the six load cases of S structures). Uses the current CUDA device and torch's
    current stream.
    """

    def __init__(self, grid_spec, batch=1, depth=0, precision="mixed", stall_window=8):
        import torch

        if not torch.cuda.is_available():
            raise _lib.LibraryError("a CUDA device is required")
        self._lib = _lib.load()
        self.grid_spec = grid_spec
        self.batch = int(batch)
        self.depth = int(depth)
        self.device = torch.device("cuda", torch.cuda.current_device())
        voxels, _ = _grid_args(grid_spec)
        extents = np.array([grid_spec.Lx, grid_spec.Ly, grid_spec.Lz], dtype=np.float64)
        h = ctypes.c_void_p()
        _lib.check(self._lib.lsb_create(ctypes.byref(h), voxels.ctypes.data_as(_lib.c_int_p),
                                        extents.ctypes.data_as(_lib.c_double_p), self.batch,
                                        self.depth), "lsb_create")
        self._h = h
        self._last_batch = 0
        self._last_maxiter = 0
        self.set_precision(precision, stall_window)

    def set_precision(self, precision="mixed", stall_window=8):
        """Field precision: "fp32", "mixed" (FP32, FP64 once FP32 round-off stalls the
        criterion near the tolerance) or "fp64"."""
        _lib.check(self._lib.lsb_set_precision(self._h, PRECISIONS[precision], int(stall_window)),
                   "lsb_set_precision")
        self.precision = precision

    def tile_variant(self, variant=None):
        """x-pass tile variant in use (chosen by timing on the first FP32 solve); an
        argument 0 or 1 fixes it."""
        return _lib.check(self._lib.lsb_tile_variant(self._h, -1 if variant is None else int(variant)),
                          "lsb_tile_variant")

    def y_variant(self, variant=None):
        """y-pass variant in use (kz columns per block; chosen by timing on the first FP32
        solve); an argument 0 or 1 fixes it (bit-identical results either way)."""
        return _lib.check(self._lib.lsb_y_variant(self._h, -1 if variant is None else int(variant)),
                          "lsb_y_variant")

    def set_tiled(self, on=True):
        """Tiled spectrum layout between the y and x passes (the default where it applies;
        results are bit-identical either way). Returns whether it is in use."""
        return bool(_lib.check(self._lib.lsb_set_tiled(self._h, 1 if on else 0), "lsb_set_tiled"))

    def pass_config(self):
        """FP32 pass configuration: dict(tiled, xvariant, slab, yvariant, settled);
        settled once the autotuner ran (first FP32 solve) or the caller fixed it."""
        out = np.zeros(4, dtype=np.int32)
        _lib.check(self._lib.lsb_pass_config(self._h, out.ctypes.data_as(_lib.c_int_p)),
                   "lsb_pass_config")
        return {"tiled": bool(out[0]), "xvariant": int(out[1]), "slab": bool(out[2]),
                "yvariant": self.y_variant(), "settled": bool(out[3])}

    def set_device_loop(self, on=True):
        """Run each solve phase as one graph launch whose WHILE node stops on the device
        (default), or replay the iteration graph from the host in polled chunks."""
        _lib.check(self._lib.lsb_set_device_loop(self._h, 1 if on else 0), "lsb_set_device_loop")

    def set_slab(self, on=True):
        """Fused slab pass (inverse y + z + forward y per x-plane; opt-in, measured slower
        than the separate passes at 128^3; results are bit-identical either way). Returns
        whether it is in use."""
        return bool(_lib.check(self._lib.lsb_set_slab(self._h, 1 if on else 0), "lsb_set_slab"))

    def set_warm_history(self, on=True):
        """With on, a warm start (``epsilon0``) enters the Anderson history as the second
        iterate instead of starting the iteration (needs depth >= 1)."""
        _lib.check(self._lib.lsb_set_warm_history(self._h, 1 if on else 0), "lsb_set_warm_history")
        self._warm_history = bool(on)

    def set_damage(self, damage, k=1e-12, dtype=np.float32):
        """Stress law of the damage extension for the following solves (see
        ``jaxmaterials_b200.solver.damage``): damage field of shape (nx, ny, nz) or (S, nx,
        ny, nz) like lambda and mu (kept on the device by this solver), residual stiffness
        k; ``None`` restores the linear law."""
        import torch

        if damage is None:
            self._damage = None
            _lib.check(self._lib.lsb_set_damage(self._h, None, 4, 0.0), "lsb_set_damage")
            return
        tdt = torch.float64 if np.dtype(dtype) == np.float64 else torch.float32
        t = torch.as_tensor(damage, dtype=tdt, device=self.device).contiguous()
        g = self.grid_spec
        if tuple(t.shape[-3:]) != (g.nx, g.ny, g.nz) or t.dim() not in (3, 4):
            raise ValueError(f"damage must have shape {(g.nx, g.ny, g.nz)} or (S,) + that")
        self._damage = t
        _lib.check(self._lib.lsb_set_damage(self._h, ctypes.c_void_p(t.data_ptr()),
                                            t.element_size(), float(k)), "lsb_set_damage")

    def set_anisotropic(self, stiffness, c0=None, dtype=np.float32):
        """Anisotropic stiffness for the following solves (see
        ``jaxmaterials_b200.solver.anisotropic``): entries of shape (21, nx, ny, nz) or (S, 21,
        nx, ny, nz), kept on the device by this solver; c0 (21,) fixes the reference
        stiffness (default: mid-range of every entry); ``None`` restores the isotropic law."""
        import torch

        if stiffness is None:
            self._stiffness = None
            _lib.check(self._lib.lsb_set_anisotropic(self._h, None, 4, None), "lsb_set_anisotropic")
            return
        tdt = torch.float64 if np.dtype(dtype) == np.float64 else torch.float32
        t = torch.as_tensor(stiffness, dtype=tdt, device=self.device).contiguous()
        g = self.grid_spec
        if tuple(t.shape[-4:]) != (21, g.nx, g.ny, g.nz) or t.dim() not in (4, 5):
            raise ValueError(f"stiffness must have shape (21, {g.nx}, {g.ny}, {g.nz}) or (S,) + that")
        self._stiffness = t
        c0p = None
        if c0 is not None:
            self._c0 = np.ascontiguousarray(np.asarray(c0, dtype=np.float64).reshape(21))
            c0p = self._c0.ctypes.data_as(_lib.c_double_p)
        _lib.check(self._lib.lsb_set_anisotropic(self._h, ctypes.c_void_p(t.data_ptr()),
                                                 t.element_size(), c0p), "lsb_set_anisotropic")

    def set_graphs(self, on=True):
        """Replay each iteration as a CUDA graph (default) or launch kernel by kernel."""
        _lib.check(self._lib.lsb_set_graphs(self._h, 1 if on else 0), "lsb_set_graphs")

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.lsb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _as_device(self, a, shape, dtype=None):
        import torch

        t = torch.as_tensor(a, dtype=dtype or torch.float32, device=self.device)
        t = t.contiguous()
        if tuple(t.shape) != tuple(shape):
            raise ValueError(f"expected shape {tuple(shape)}, got {tuple(t.shape)}")
        return t

    def solve(self, lmbda, mu, epsilon_bar, rtol=1e-6, atol=1e-20, maxiter=32,
              rule=RULE_CUDA, epsilon0=None, want_sigma=True, out=None, dtype=np.float32,
              e0_ref=None):
        """Run the fixed point for every row of ``epsilon_bar`` (shape (B, 6) or (6,)).

        ``dtype=np.float64`` runs FP64 fields end to end (inputs and outputs in FP64).
        ``e0_ref`` (B positive values): stop at rtol * e0_ref[b] instead of rtol times the
        instance's first criterion (for warm starts, the cold-start criterion)."""
        import torch

        f64 = np.dtype(dtype) == np.float64
        tdt = torch.float64 if f64 else torch.float32
        g = self.grid_spec
        nshape = (g.nx, g.ny, g.nz)
        eb = np.ascontiguousarray(np.atleast_2d(np.asarray(
            epsilon_bar.cpu() if isinstance(epsilon_bar, torch.Tensor) else epsilon_bar,
            dtype=np.float64 if f64 else np.float32)))
        b = eb.shape[0]
        if eb.shape[1] != 6 or b < 1 or b > self.batch:
            raise ValueError(f"epsilon_bar must have shape (B, 6) with 1 <= B <= {self.batch}")
        lshape = tuple(np.shape(lmbda))
        nstruct = 1 if lshape == nshape else (lshape[0] if len(lshape) == 4 else 0)
        if nstruct < 1 or b % nstruct != 0:
            raise ValueError(f"lambda must have shape {nshape} or (S,) + {nshape} with B = "
                             f"{b} a multiple of S, got {lshape}")
        fshape = nshape if lshape == nshape else (nstruct,) + nshape
        lm = self._as_device(lmbda, fshape, tdt)
        m = self._as_device(mu, fshape, tdt)
        _lib.check(self._lib.lsb_set_lame_group(self._h, 0 if lshape == nshape else b // nstruct),
                   "lsb_set_lame_group")
        e0 = None
        if epsilon0 is not None:
            e0 = self._as_device(epsilon0, (b, 6) + nshape, tdt)
        eps = out if out is not None else torch.empty((b, 6) + nshape, dtype=tdt,
                                                      device=self.device)
        sig = torch.empty_like(eps) if want_sigma else None
        iters = np.zeros(b, dtype=np.int32)
        status = np.zeros(b, dtype=np.int32)
        resid = np.zeros(b, dtype=np.float64)
        mean = np.zeros((b, 6), dtype=np.float64)
        stream = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._lib.lsb_set_stream(self._h, ctypes.c_void_p(stream)), "lsb_set_stream")
        if e0_ref is None:
            _lib.check(self._lib.lsb_set_reference_e0(self._h, b, None), "lsb_set_reference_e0")
        else:
            ref = np.ascontiguousarray(np.broadcast_to(np.asarray(e0_ref, np.float64), (b,)))
            _lib.check(self._lib.lsb_set_reference_e0(self._h, b, ref.ctypes.data_as(_lib.c_double_p)),
                       "lsb_set_reference_e0")
        fn = self._lib.lsb_solve_f64 if f64 else self._lib.lsb_solve
        ebp = eb.ctypes.data_as(_lib.c_double_p) if f64 else _fptr(eb)
        rc = fn(
            self._h, b, ctypes.c_void_p(lm.data_ptr()), ctypes.c_void_p(m.data_ptr()),
            ebp, ctypes.c_void_p(e0.data_ptr() if e0 is not None else 0),
            ctypes.c_void_p(eps.data_ptr()),
            ctypes.c_void_p(sig.data_ptr() if sig is not None else 0),
            mean.ctypes.data_as(_lib.c_double_p), float(rtol), float(atol), int(maxiter),
            int(rule), iters.ctypes.data_as(_lib.c_int_p), status.ctypes.data_as(_lib.c_int_p),
            resid.ctypes.data_as(_lib.c_double_p))
        _lib.check(rc, "lsb_solve_f64" if f64 else "lsb_solve")
        self._last_batch = b
        self._last_maxiter = int(maxiter)
        return SolveResult(eps, sig, iters, status, resid, mean)

    def project_compatible(self, epsilon, epsilon_bar):
        """Compatible part of strain fields, for use as a warm start:
        eps_bar + P(eps - eps_bar), P = Gamma^0 C^0 the projection onto zero-mean compatible
        fields of this solver's discretisation (modified wave vectors). Computed as one
        update of the homogeneous medium lambda = 0, mu = 1/2 started from eps, which gives
        eps_bar + (I - P)(eps - eps_bar). epsilon: (B, 6, nx, ny, nz) float32 CUDA tensor,
        epsilon_bar: (B, 6). Returns a new tensor."""
        import torch

        g = self.grid_spec
        eb = np.ascontiguousarray(np.atleast_2d(np.asarray(
            epsilon_bar.cpu() if isinstance(epsilon_bar, torch.Tensor) else epsilon_bar,
            dtype=np.float32)))
        lam0 = torch.zeros(g.shape, device=self.device, dtype=torch.float32)
        mu0 = torch.full(g.shape, 0.5, device=self.device, dtype=torch.float32)
        prec = self.precision
        hist = getattr(self, "_warm_history", False)
        self.set_precision("fp32", 0)
        if hist:
            self.set_warm_history(False)   # the update must start from epsilon
        try:
            r = self.solve(lam0, mu0, eb, rtol=0.0, atol=0.0, maxiter=1, epsilon0=epsilon,
                           want_sigma=False)
        finally:
            self.set_precision(prec)
            if hist:
                self.set_warm_history(True)
        ebt = torch.as_tensor(eb, device=self.device).view(eb.shape[0], 6, 1, 1, 1)
        return epsilon + ebt - r.epsilon

    def kernel_launches(self):
        """Kernels enqueued by this solver so far."""
        return int(self._lib.lsb_kernel_launches(self._h))

    def fp64_iters(self):
        """Updates of each instance of the last solve that ran with FP64 fields."""
        out = np.zeros(self._last_batch, dtype=np.int32)
        _lib.check(self._lib.lsb_fp64_iters(self._h, out.ctypes.data_as(_lib.c_int_p)),
                   "lsb_fp64_iters")
        return out

    def profile_step(self, lmbda, mu, batch=None, reps=5):
        """Average CUDA-event time (ms) of every launch of one FP32 iteration as the solve
        runs it (Anderson when depth > 0, plain otherwise): list of (kernel name, ms) in
        launch order."""
        import torch

        g = self.grid_spec
        b = self.batch if batch is None else int(batch)
        lm = self._as_device(lmbda, g.shape)
        m = self._as_device(mu, g.shape)
        _lib.check(self._lib.lsb_set_lame_group(self._h, 0), "lsb_set_lame_group")
        work = torch.empty((b, 6) + g.shape, dtype=torch.float32, device=self.device)
        ms = np.zeros(32, dtype=np.float32)
        names = ctypes.create_string_buffer(1024)
        stream = torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(self._lib.lsb_set_stream(self._h, ctypes.c_void_p(stream)), "lsb_set_stream")
        n = self._lib.lsb_profile_step(
            self._h, b, ctypes.c_void_p(lm.data_ptr()), ctypes.c_void_p(m.data_ptr()),
            ctypes.c_void_p(work.data_ptr()), int(reps), _fptr(ms), ms.shape[0], names,
            len(names))
        _lib.check(n if n < 0 else 0, "lsb_profile_step")
        return list(zip(names.value.decode().split(","), [float(v) for v in ms[:n]]))

    def history(self):
        """Criterion after every evaluation of the last solve, shape (B, maxiter + 1)."""
        n = self._last_maxiter + 1
        out = np.zeros((self._last_batch, n), dtype=np.float64)
        _lib.check(self._lib.lsb_history(self._h, out.ctypes.data_as(_lib.c_double_p), n),
                   "lsb_history")
        return out


_solver_cache = {}


def _cached_solver(grid_spec, batch, depth):
    import torch

    key = (grid_spec.nx, grid_spec.ny, grid_spec.nz, grid_spec.Lx, grid_spec.Ly,
           grid_spec.Lz, batch, depth, torch.cuda.current_device())
    s = _solver_cache.get(key)
    if s is None:
        if len(_solver_cache) > 8:
            _solver_cache.clear()
        s = Solver(grid_spec, batch=batch, depth=depth)
        _solver_cache[key] = s
    return s


def lippmann_schwinger(lmbda, mu, epsilon_bar, grid_spec, rtol=1e-6, atol=1e-20, depth=0,
                       maxiter=32, dtype=np.float32, epsilon0=None, precision=None):
    """Signature of the reference ``lippmann_schwinger_jax`` (``:146-265``).

    Returns ``(epsilon, sigma, iter)`` with fields of shape (6, nx, ny, nz): NumPy arrays
    for NumPy input, CUDA tensors for torch input. Stops when
    e <= max(rtol e0, atol) or after ``maxiter`` updates, without raising (as the
    reference). ``dtype`` float32 runs FP32 fields (mixed precision: FP64 fields take
    over if FP32 round-off stalls the criterion near the tolerance; ``precision="fp32"``
    disables that); float64 runs FP64 fields. Norms and the stop decision are FP64.
    """
    import torch

    f64 = np.dtype(dtype) == np.float64
    as_torch = isinstance(lmbda, torch.Tensor)
    s = _cached_solver(grid_spec, 1, depth)
    s.set_precision(precision or ("fp64" if f64 else "mixed"))
    e0 = None if epsilon0 is None else (
        epsilon0.reshape((1, 6) + grid_spec.shape) if as_torch
        else np.asarray(epsilon0).reshape((1, 6) + grid_spec.shape))
    eb = np.asarray(epsilon_bar.cpu() if isinstance(epsilon_bar, torch.Tensor) else epsilon_bar,
                    dtype=np.float64).reshape(1, 6)
    r = s.solve(lmbda, mu, eb, rtol=rtol, atol=atol, maxiter=maxiter, rule=RULE_JAX,
                epsilon0=e0, dtype=np.float64 if f64 else np.float32)
    eps, sig = r.epsilon[0], r.sigma[0]
    if not as_torch:
        eps, sig = eps.cpu().numpy(), sig.cpu().numpy()
    return eps, sig, int(r.iters[0])


lippmann_schwinger_jax = lippmann_schwinger


def c_eff(lmbda, mu, grid_spec, rtol=1e-6, atol=1e-20, maxiter=1000, depth=0, solver=None,
          precision="mixed"):
    """Effective stiffness: row k = mean stress for the unit strain e_k (tensor shear).

    Solves the six load cases as one batch. Returns ``(C, iters, result)``."""
    s = solver if solver is not None else _cached_solver(grid_spec, 6, depth)
    if solver is None:
        s.set_precision(precision)
    r = s.solve(lmbda, mu, np.eye(6, dtype=np.float32), rtol=rtol, atol=atol,
                maxiter=maxiter, rule=RULE_CUDA, want_sigma=False)
    return r.mean_sigma.copy(), r.iters.copy(), r
