"""Damage extension: the reference's degraded stress law, tensile energy, damaged
elasticity solve and phase-field solve (``src/jaxmaterials/solver/lippmann_schwinger.py``
:36-100 and :330-547), with the same signatures, on the GPU through
``liblippmannschwinger.so`` (``lsb_damage_stress``, ``lsb_strain_energy``,
``lsb_set_damage``, ``lsb_phase_field_solve``).

Fields are device tensors or host arrays; results come back as torch tensors on the device
when any field argument was a torch tensor, else as NumPy arrays. Voigt components (v0..v5)
enter the 3 x 3 strain tensor as [[v0, v5, v4], [v5, v1, v3], [v4, v3, v2]], as in the
reference (src/jaxmaterials/utilities.py:65-85).

Differences from the reference: ``elasticity_solve`` in float32 continues in FP64 where
FP32 round-off stalls the criterion above the tolerance (the linear solver's mixed
precision); the phase-field solve's norms are accumulated in FP64.
"""

import ctypes

import numpy as np

from .. import _lib
from .lippmann_schwinger import RULE_JAX, Solver

__all__ = ["compute_sigma_damaged", "compute_strain_energy", "update_history",
           "elasticity_solve", "phase_field_solve"]


def _torch_in(*xs):
    import torch

    return any(isinstance(x, torch.Tensor) for x in xs)


def _dtype_of(x, dtype):
    """The requested dtype, else the field's own (float64 stays float64, all else float32)."""
    import torch

    if dtype is not None:
        return np.dtype(dtype)
    if isinstance(x, torch.Tensor):
        return np.dtype(np.float64 if x.dtype == torch.float64 else np.float32)
    return np.dtype(np.float64 if np.asarray(x).dtype == np.float64 else np.float32)


def _dev(a, dtype):
    import torch

    tdt = torch.float64 if np.dtype(dtype) == np.float64 else torch.float32
    return torch.as_tensor(a, dtype=tdt, device="cuda").contiguous()


def _out(t, as_torch):
    return t if as_torch else t.cpu().numpy()


def _stream():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def compute_sigma_damaged(lmbda, mu, epsilon, d=None, k=1e-12, dtype=None):
    """sigma = ((1 - d)^2 + k) sigma+ + sigma- (sigma+ + sigma- without d); epsilon of shape
    (6, nx, ny, nz) or (B, 6, nx, ny, nz); lambda, mu, d of shape (nx, ny, nz)."""
    as_t = _torch_in(lmbda, mu, epsilon, d)
    dt = _dtype_of(epsilon, dtype)
    e = _dev(epsilon, dt)
    squeeze = e.dim() == 4
    if squeeze:
        e = e.unsqueeze(0)
    nv = int(np.prod(e.shape[-3:]))
    lm, m = _dev(lmbda, dt), _dev(mu, dt)
    dd = _dev(d, dt) if d is not None else None
    s = e.new_empty(e.shape)
    lib = _lib.load()
    _lib.check(lib.lsb_damage_stress(nv, e.shape[0], ctypes.c_void_p(e.data_ptr()),
                                     ctypes.c_void_p(lm.data_ptr()), ctypes.c_void_p(m.data_ptr()),
                                     ctypes.c_void_p(dd.data_ptr() if dd is not None else 0),
                                     float(k), ctypes.c_void_p(s.data_ptr()), e.element_size(),
                                     _stream()), "lsb_damage_stress")
    return _out(s[0] if squeeze else s, as_t)


def compute_strain_energy(lmbda, mu, epsilon, dtype=None):
    """Tensile energy psi+ = 1/2 lambda <tr eps>+^2 + mu sum <eig>+^2, shape (nx, ny, nz)."""
    as_t = _torch_in(lmbda, mu, epsilon)
    dt = _dtype_of(epsilon, dtype)
    e = _dev(epsilon, dt)
    lm, m = _dev(lmbda, dt), _dev(mu, dt)
    psi = e.new_empty(e.shape[1:])
    lib = _lib.load()
    _lib.check(lib.lsb_strain_energy(psi.numel(), ctypes.c_void_p(e.data_ptr()),
                                     ctypes.c_void_p(lm.data_ptr()), ctypes.c_void_p(m.data_ptr()),
                                     ctypes.c_void_p(psi.data_ptr()), None, e.element_size(),
                                     _stream()), "lsb_strain_energy")
    return _out(psi, as_t)


def update_history(history, lmbda, mu, epsilon):
    """history = max(history, psi+) in place (a device tensor; the staggered scheme's
    history field, tests/phasefield.py)."""
    import torch

    if not isinstance(history, torch.Tensor) or not history.is_cuda or not history.is_contiguous():
        raise ValueError("history must be a contiguous CUDA tensor")
    dt = np.float64 if history.dtype == torch.float64 else np.float32
    e = _dev(epsilon, dt)
    lm, m = _dev(lmbda, dt), _dev(mu, dt)
    lib = _lib.load()
    _lib.check(lib.lsb_strain_energy(history.numel(), ctypes.c_void_p(e.data_ptr()),
                                     ctypes.c_void_p(lm.data_ptr()), ctypes.c_void_p(m.data_ptr()),
                                     None, ctypes.c_void_p(history.data_ptr()),
                                     history.element_size(), _stream()), "lsb_strain_energy")
    return history


_solvers = {}


def _solver(grid_spec, depth):
    key = (grid_spec.nx, grid_spec.ny, grid_spec.nz, grid_spec.Lx, grid_spec.Ly, grid_spec.Lz,
           depth)
    s = _solvers.get(key)
    if s is None:
        s = _solvers[key] = Solver(grid_spec, batch=1, depth=depth)
    return s


def elasticity_solve(lmbda, mu, epsilon_bar, dvar, kk, grid_spec, rtol=1e-6, atol=1e-20,
                     depth=0, maxiter=32, dtype=np.float32, solver=None):
    """The damaged Lippmann-Schwinger solve (lippmann_schwinger.py:330-455): returns
    ``(epsilon (6, nx, ny, nz), sigma, iterations)``; stops when e <= max(atol, rtol e0)."""
    as_t = _torch_in(lmbda, mu, epsilon_bar, dvar)
    f64 = np.dtype(dtype) == np.float64
    s = solver or _solver(grid_spec, depth)
    s.set_damage(dvar, kk, np.float64 if f64 else np.float32)
    try:
        r = s.solve(lmbda, mu, np.asarray(epsilon_bar.cpu() if hasattr(epsilon_bar, "cpu")
                                          else epsilon_bar, dtype=np.float64),
                    rtol=rtol, atol=atol, maxiter=maxiter, rule=RULE_JAX, want_sigma=True,
                    dtype=np.float64 if f64 else np.float32)
    finally:
        s.set_damage(None)
    return _out(r.epsilon[0], as_t), _out(r.sigma[0], as_t), int(r.iters[0])


def phase_field_solve(HH, d_old, gc, lc, grid_spec, tolerance=1e-6, maxiter=1000,
                      dtype=np.float32, solver=None):
    """The phase-field fixed point (lippmann_schwinger.py:457-547): returns ``(d,
    iterations)`` for the history field HH and the previous damage d_old (nx, ny, nz)."""
    as_t = _torch_in(HH, d_old)
    dt = np.dtype(dtype)
    s = solver or _solver(grid_spec, 0)
    h = _dev(HH, dt).reshape(grid_spec.nx, grid_spec.ny, grid_spec.nz)
    d = _dev(d_old, dt).reshape(grid_spec.nx, grid_spec.ny, grid_spec.nz).clone()
    iters = ctypes.c_int()
    res = ctypes.c_double()
    import torch

    with torch.cuda.device(s.device):
        _lib.check(s._lib.lsb_set_stream(s._h, _stream()), "lsb_set_stream")
        _lib.check(s._lib.lsb_phase_field_solve(
            s._h, ctypes.c_void_p(h.data_ptr()), ctypes.c_void_p(d.data_ptr()), float(gc),
            float(lc), float(tolerance), int(maxiter), d.element_size(), ctypes.byref(iters),
            ctypes.byref(res)), "lsb_phase_field_solve")
    return _out(d, as_t), int(iters.value)


def benchmark(n=128, seed=0, depth=3):
    """One staggered step of the reference's phase-field fracture driver
    (tests/phasefield.py:165-214) on an n^3 cross-ply composite: phase-field solve from a
    history field, damaged elasticity solve (Anderson depth ``depth``, rtol 1e-6, tension
    along y), history update; the damaged solve is also timed against the linear solve of the
    same problem. CUDA events on the current stream."""
    import torch

    from .. import GridSpec
    from ..data import fibres

    st = fibres.generate_layered_fibres(n, 4, 4.0, 0.45, seed=seed)
    lm, mu = fibres.lame_fields(st)
    g = GridSpec(n, n, n, float(n), float(n), float(n))
    lm_d = torch.as_tensor(lm, device="cuda")
    mu_d = torch.as_tensor(mu, device="cuda")
    eb = np.array([0.0, 1e-3, 0.0, 0.0, 0.0, 0.0])
    rng = np.random.default_rng(seed)
    # a damage field concentrated in a band across the fibres
    x = (np.arange(n) + 0.5) / n
    band = np.exp(-((x - 0.5) / 0.05) ** 2)
    d0 = torch.as_tensor((0.5 * band[None, :, None] * np.ones((n, n, n))).astype(np.float32),
                         device="cuda")
    hist = torch.as_tensor(rng.uniform(0.0, 1e-3, (n, n, n)).astype(np.float32), device="cuda")
    s_lin = Solver(g, batch=1, depth=depth)
    s_dmg = Solver(g, batch=1, depth=depth)
    stream = torch.cuda.current_stream()

    def timed(fn):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1)

    def lin():
        return s_lin.solve(lm_d, mu_d, eb, rtol=1e-6, atol=1e-20, maxiter=2000, rule=RULE_JAX,
                           want_sigma=False)

    def dmg():
        return elasticity_solve(lm_d, mu_d, eb, d0, 1e-6, g, rtol=1e-6, depth=depth,
                                maxiter=2000, solver=s_dmg)

    def pf():
        return phase_field_solve(hist, d0, 2.7e-3, 1.5, g, tolerance=1e-6, maxiter=10000)

    for _ in range(2):  # warm-up (plans, graphs, x-pass tile choice, work buffers)
        for f in (lin, dmg, pf):
            f()
    r_lin, ms_lin = timed(lin)
    (eps, _, it_dmg), ms_dmg = timed(dmg)
    (_, it_pf), ms_pf = timed(pf)
    h2 = hist.clone()
    _, ms_hist = timed(lambda: update_history(h2, lm_d, mu_d, eps))
    s_lin.close()
    s_dmg.close()
    return {"grid": [n, n, n], "anderson_depth": depth, "load": "unit tension along y (1e-3)",
            "linear_solve_ms": ms_lin, "linear_iters": int(r_lin.iters[0]),
            "damaged_solve_ms": ms_dmg, "damaged_iters": it_dmg,
            "damaged_ms_per_iter": ms_dmg / max(it_dmg, 1),
            "linear_ms_per_iter": ms_lin / max(int(r_lin.iters[0]), 1),
            "phase_field_ms": ms_pf, "phase_field_iters": it_pf,
            "phase_field_ms_per_iter": ms_pf / max(it_pf, 1),
            "history_update_ms": ms_hist}


def main(argv=None):
    """``python -m jaxmaterials_b200.solver.damage [--n 128]``: timings of one staggered
    phase-field fracture step as one JSON line."""
    import argparse
    import json

    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, default=128)
    p.add_argument("--depth", type=int, default=3)
    a = p.parse_args(argv)
    print(json.dumps(benchmark(a.n, depth=a.depth)))


if __name__ == "__main__":
    main()
