"""Warm-start network kernels (include/spectral_net.h): forward against the FP64 CPU
oracle, backward against central finite differences of the oracle and against torch
autograd of a plain torch FP32 restatement, the Adam kernel against its formula; the
reference-criterion stop rule; the data/training/evaluation pipeline on a small grid.

Tolerances: forward 1e-5 relative to the output's max-abs (FP32 accumulation, BF16
weights passed rounded to both sides); gradients 2e-3 relative to the gradient's
max-abs against FD (h = 1e-3 in FP64) and 1e-4 against torch autograd.
"""

import ctypes

import numpy as np
import pytest

from oracle import spectral_net_oracle as SO

pytestmark = pytest.mark.gpu


def is_weight(name):
    return name.startswith("spec") or name.endswith("_w") or (name[0] == "w" and name[1:].isdigit())


def rounded_params(net):
    import torch

    return {k: (v.detach().to(torch.bfloat16) if is_weight(k) else v.detach()).double().cpu().numpy()
            for k, v in net.params.items()}


def torch_reference(net, a):
    """Plain torch FP32 forward with the BF16-rounded weights (differentiable); layers with
    a multiple of 16 input channels take their activations rounded to BF16 as well, as the
    tensor-core kernels do."""
    import torch
    import torch.nn.functional as F

    p = net.params

    def rw(w):
        return w + (w.to(torch.bfloat16).float() - w).detach()

    def pw(x, w, b):
        if x.shape[1] % 16 == 0 and x[0, 0].numel() % 16 == 0:
            x = rw(x)
        return torch.einsum("oi,bi...->bo...", rw(w), x) + b.view(1, -1, 1, 1, 1)

    n = tuple(a.shape[2:])
    kx, ky, kz = (torch.as_tensor(v, device=a.device) for v in SO.retained_index(n, net.modes))
    h = pw(a, p["lift_w"], p["lift_b"])
    for l in range(net.layers):
        xh = torch.fft.rfftn(h, dim=(-3, -2, -1))
        w = rw(p[f"spec{l}"])
        wc = torch.complex(w[..., 0], w[..., 1])
        out = torch.einsum("bim,mio->bom", xh[:, :, kx, ky, kz], wc)
        yh = torch.zeros((h.shape[0], wc.shape[2]) + tuple(xh.shape[2:]), dtype=xh.dtype,
                         device=a.device)
        yh[:, :, kx, ky, kz] = out
        h = F.gelu(pw(h, p[f"w{l}"], p[f"b{l}"]) + SO.inverse_half_spectrum(yh, n))
    return pw(h, p["proj_w"], p["proj_b"])


def tiny(n, seed=3):
    import torch
    from jaxmaterials_b200.learned.network import SpectralNet

    net = SpectralNet(width=4, layers=2, modes=(4, 4, 3), out_channels=6, seed=seed)
    g = torch.Generator().manual_seed(seed + 1)
    for v in net.params.values():  # nonzero biases, so that they are tested too
        if v.dim() == 1:
            v.data.copy_((torch.rand(v.shape, generator=g) - 0.5).to(v.device))
    a = torch.randn((2, 2) + n, generator=g).cuda()
    return net, a


@pytest.mark.parametrize("n", [(8, 8, 8), (8, 6, 10), (10, 8, 7)])
def test_forward_matches_oracle(n):
    net, a = tiny(n)
    y = net(a).detach().cpu().numpy()
    ref = SO.forward(rounded_params(net), a.double().cpu().numpy(), net.layers, net.modes)
    assert np.abs(y - ref).max() / np.abs(ref).max() < 1e-5


@pytest.mark.parametrize("n", [(8, 8, 8), (10, 8, 7)])
def test_gradients_match_oracle_fd(n):
    import torch

    net, a = tiny(n)
    rng = np.random.default_rng(7)
    wts = rng.standard_normal((2, 6) + n)
    out = net(a)
    (out * torch.as_tensor(wts, device="cuda", dtype=torch.float32)).sum().backward()
    params = rounded_params(net)
    a64 = a.double().cpu().numpy()
    for name, p in net.params.items():
        g = p.grad.detach().double().cpu().numpy()
        scale = np.abs(g).max()
        for _ in range(3):
            idx = tuple(int(rng.integers(s)) for s in g.shape)
            fd = SO.fd_gradient(params, a64, net.layers, net.modes, wts, name, idx)
            assert abs(g[idx] - fd) <= 2e-3 * scale, (name, idx, g[idx], fd)


def test_gradients_match_torch_autograd():
    import torch

    net, a = tiny((8, 8, 8))
    wts = torch.randn((2, 6, 8, 8, 8), device="cuda")
    (net(a) * wts).sum().backward()
    mine = {k: v.grad.clone() for k, v in net.params.items()}
    for v in net.params.values():
        v.grad = None
    (torch_reference(net, a) * wts).sum().backward()
    for k, v in net.params.items():
        err = (mine[k] - v.grad).abs().max() / v.grad.abs().max()
        assert err < 1e-4, (k, float(err))


def test_full_width_forward_matches_torch():
    """The 32-channel, 12-mode configuration (kernel pairs (2,32), (32,32), (32,36)) at
    32^3 against the torch restatement (torch.fft, activations of the 32-channel layers
    rounded to BF16 as the tensor-core kernels round them). The two sides compute the
    pre-rounding activations in a different order, so an activation within FP32 round-off
    of a BF16 rounding boundary can round to neighbouring BF16 values: one BF16 step
    (2^-8 relative) in single activations, hence 5e-3 of the output's max-abs here; the
    layers themselves are checked to 1e-5 with identical inputs
    (test_tensor_core_pointwise_layers, test_truncated_transforms_match_numpy)."""
    import torch
    from jaxmaterials_b200.learned.network import SpectralNet

    net = SpectralNet(seed=5)
    a = torch.randn((2, 2, 32, 32, 32), device="cuda")
    with torch.no_grad():
        y = net(a)
        ref = torch_reference(net, a)
    assert ((y - ref).abs().max() / ref.abs().max()) < 5e-3


@pytest.mark.parametrize("n,modes", [((8, 6, 10), (4, 4, 3)), ((10, 8, 7), (4, 6, 4)),
                                     ((16, 16, 16), (8, 8, 9)), ((64, 64, 64), (12, 12, 12))])
def test_truncated_transforms_match_numpy(n, modes):
    """The network's truncated transforms against numpy: forward = rfftn at the retained
    modes, inverse(1/N, 2) = irfftn of the zero-padded half spectrum (also with the z
    Nyquist plane retained and imaginary parts on the kz = 0 and Nyquist planes), and each
    transform's transpose as a real-linear map is the other (the backward passes)."""
    import torch
    from jaxmaterials_b200 import _lib
    from jaxmaterials_b200.learned.network import _ptr, _stream

    lib = _lib.load()
    rng = np.random.default_rng(3)
    bc = 5
    nn = (ctypes.c_int * 3)(*n)
    mm = (ctypes.c_int * 3)(*modes)
    kx, ky, kz = SO.retained_index(n, modes)
    f = rng.standard_normal((bc,) + n).astype(np.float32)
    y = (rng.standard_normal((bc,) + modes) + 1j * rng.standard_normal((bc,) + modes)).astype(np.complex64)
    fd = torch.as_tensor(f).cuda()
    yd = torch.as_tensor(y).cuda()
    work = torch.empty((bc, n[0], modes[1], modes[2]), dtype=torch.complex64, device="cuda")

    def fwd(x, scale=1.0, w=1.0):
        out = torch.empty((bc,) + modes, dtype=torch.complex64, device="cuda")
        _lib.check_net(lib.lsn_truncated_forward(bc, nn, mm, _ptr(x), _ptr(work), _ptr(out), scale, w,
                                                 _stream(x)), "forward")
        return out

    def inv(x, scale=1.0, w=1.0):
        out = torch.empty((bc,) + n, dtype=torch.float32, device="cuda")
        _lib.check_net(lib.lsn_truncated_inverse(bc, nn, mm, _ptr(x), _ptr(work), _ptr(out), scale, w,
                                                 _stream(x)), "inverse")
        return out

    full = np.fft.rfftn(f.astype(np.float64), axes=(1, 2, 3))
    ref = full[:, kx, ky, kz].reshape((bc,) + modes)
    got = fwd(fd).cpu().numpy()
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-5
    yh = np.zeros((bc, n[0], n[1], n[2] // 2 + 1), complex)
    yh[:, kx, ky, kz] = y.reshape(bc, -1).astype(complex)
    ref = np.fft.irfftn(yh, s=n, axes=(1, 2, 3))
    got = inv(yd, 1.0 / np.prod(n), 2.0).cpu().numpy()
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-5
    # transposes: <fwd(f), y>_R = <f, inv(y)> for (1, 1) and (1/N, 2)
    for scale, w in ((1.0, 1.0), (1.0 / np.prod(n), 2.0)):
        lhs = float((fwd(fd, scale, w).cpu().numpy().astype(np.complex128).conj() * y).real.sum())
        rhs = float((f.astype(np.float64) * inv(yd, scale, w).cpu().numpy()).sum())
        assert abs(lhs - rhs) < 1e-5 * max(abs(lhs), abs(rhs), 1.0), (scale, lhs, rhs)


@pytest.mark.parametrize("cout,act", [(32, 1), (36, 0)])
def test_tensor_core_pointwise_layers(cout, act):
    """The tensor-core pointwise layers (32 input channels) against an FP32 torch
    computation with the kernels' BF16 roundings: forward y = act(W x + b + add) with x and
    W rounded; backward dpre = dy act'(pre), dW = sum_v bf16(dpre) bf16(x), dx = W^T bf16(dpre),
    db = sum_v dpre. Products of BF16 values are exact in FP32, so only the order of the
    FP32 sums differs: 1e-5 relative to each output's max-abs."""
    import torch
    import torch.nn.functional as F
    from jaxmaterials_b200 import _lib
    from jaxmaterials_b200.learned.network import _ptr, _stream

    lib = _lib.load()
    g = torch.Generator(device="cuda").manual_seed(7)
    bsz, cin, shape = 3, 32, (16, 12, 8)
    nv = int(np.prod(shape))
    x = torch.randn((bsz, cin) + shape, device="cuda", generator=g)
    w = (torch.randn((cout, cin), device="cuda", generator=g) / 6).to(torch.bfloat16)
    b = torch.randn((cout,), device="cuda", generator=g)
    add = torch.randn((bsz, cout) + shape, device="cuda", generator=g) if act else None
    y = torch.empty((bsz, cout) + shape, device="cuda")
    pre = torch.empty_like(y) if act else None
    _lib.check_net(lib.lsn_pointwise_forward(bsz, cin, cout, nv, _ptr(x), _ptr(w), _ptr(b), _ptr(add),
                                             _ptr(pre), _ptr(y), act, _stream(x)), "forward")
    xb, wf = x.to(torch.bfloat16).float(), w.float()
    z = torch.einsum("oi,bi...->bo...", wf, xb) + b.view(1, -1, 1, 1, 1)
    if act:
        z = z + add
        assert (pre - z).abs().max() / z.abs().max() < 1e-5
    ref = F.gelu(z) if act else z
    assert (y - ref).abs().max() / ref.abs().max() < 1e-5

    dy = torch.randn_like(y)
    dx = torch.empty_like(x)
    dpre = torch.empty_like(y) if act else None
    dw = torch.zeros((cout, cin), device="cuda")
    db = torch.zeros((cout,), device="cuda")
    _lib.check_net(lib.lsn_pointwise_backward(bsz, cin, cout, nv, _ptr(x), _ptr(w), _ptr(pre), _ptr(dy),
                                              act, _ptr(dx), _ptr(dpre), _ptr(dw), _ptr(db), _stream(x)),
                   "backward")
    torch.cuda.synchronize()
    if act:
        zz = z.detach().requires_grad_(True)
        (gr,) = torch.autograd.grad(F.gelu(zz), zz, dy)
        assert (dpre - gr).abs().max() / gr.abs().max() < 1e-5
        # the products below take the kernel's own dpre (rounding the reference's instead
        # could land on the other side of a BF16 rounding boundary)
        dp = dpre
    else:
        dp = dy
    dpb = dp.to(torch.bfloat16).float()
    dw_ref = torch.einsum("bo...,bi...->oi", dpb, xb)
    dx_ref = torch.einsum("oi,bo...->bi...", wf, dpb)
    db_ref = dp.sum(dim=(0, 2, 3, 4))
    assert (dw - dw_ref).abs().max() / dw_ref.abs().max() < 1e-5
    assert (dx - dx_ref).abs().max() / dx_ref.abs().max() < 1e-5
    assert (db - db_ref).abs().max() / db_ref.abs().max() < 1e-5


def test_adam_kernel():
    import torch
    from jaxmaterials_b200.learned.network import Adam

    p = torch.randn(1000, device="cuda", requires_grad=True)
    opt = Adam([p], lr=1e-2)
    ref = p.detach().clone()
    m = torch.zeros_like(ref)
    v = torch.zeros_like(ref)
    for t in range(1, 4):
        g = torch.randn(1000, device="cuda")
        p.grad = g.clone()
        opt.step()
        m = 0.9 * m + 0.1 * g
        v = 0.999 * v + 0.001 * g * g
        ref = ref - 1e-2 * (m / (1 - 0.9 ** t)) / (torch.sqrt(v / (1 - 0.999 ** t)) + 1e-8)
    assert torch.allclose(p.detach(), ref, rtol=1e-5, atol=1e-6)


def test_warm_start_from_solution_needs_no_iterations():
    """With the cold start's criterion as the reference, a solve started from the cold
    solution stops at once, or after the few updates that the FP32 rounding of an iterate
    finished in FP64 needs (mixed precision); without it the stricter relative threshold
    makes every instance iterate."""
    import torch
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.learned import warm_start as W
    from jaxmaterials_b200.solver import Solver

    ind = torch.as_tensor(W.indicators(W.structure_params(2, 32, 9), workers=1)).cuda()
    lm, mu = W.lame_from_indicator(ind)
    g = GridSpec(32, 32, 32, 32.0, 32.0, 32.0)
    s = Solver(g, batch=12, depth=5)
    eb = np.tile(np.eye(6, dtype=np.float32), (2, 1))
    cold = s.solve(lm, mu, eb, rtol=1e-6, maxiter=3000, want_sigma=False)
    e0 = s.solve(lm, mu, eb, maxiter=0, want_sigma=False).residual
    cold_again = s.solve(lm, mu, eb, rtol=1e-6, maxiter=3000, want_sigma=False)
    np.testing.assert_allclose(e0, s.history()[:, 0], rtol=1e-12)
    np.testing.assert_array_equal(cold_again.iters, cold.iters)
    warm = s.solve(lm, mu, eb, rtol=1e-6, maxiter=3000, want_sigma=False,
                   epsilon0=cold.epsilon, e0_ref=e0)
    assert (warm.iters <= 2).all() and (warm.iters == 0).sum() >= 6
    again = s.solve(lm, mu, eb, rtol=1e-6, maxiter=3000, want_sigma=False,
                    epsilon0=cold.epsilon)
    assert (again.iters > 2).all()


def test_training_pipeline_small():
    """Data from the solver, a few training epochs, cold vs warm evaluation (16^3)."""
    import torch
    from jaxmaterials_b200.learned import warm_start as W
    from jaxmaterials_b200.learned.network import SpectralNet

    ind = torch.as_tensor(W.indicators(W.structure_params(8, 16, 1), workers=1)).cuda()
    targets, it = W.solve_dataset(ind, chunk=4)
    assert targets.shape == (8, 36, 16, 16, 16) and (it > 0).all()
    net = SpectralNet(modes=(8, 8, 8), seed=2)
    losses = W.train(net, ind, targets, epochs=3, batch=4, lr=3e-3)
    assert losses[-1] < losses[0]
    summ = W.summarise(W.evaluate(net, ind[:4], chunk=4), 16)
    assert summ["c_eff_warm_vs_cold_rel_max"] < 1e-5
    assert summ["warm_iters_per_solve"] > 0


def test_project_compatible():
    """The projection keeps compatible fields, is idempotent, and a warm start projected
    from an arbitrary field converges to the cold solution."""
    import torch
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.learned import warm_start as W
    from jaxmaterials_b200.solver import Solver

    ind = torch.as_tensor(W.indicators(W.structure_params(1, 32, 4), workers=1)).cuda()
    lm, mu = W.lame_from_indicator(ind)
    g = GridSpec(32, 32, 32, 32.0, 32.0, 32.0)
    s = Solver(g, batch=6, depth=5)
    eb = np.eye(6, dtype=np.float32)
    cold = s.solve(lm, mu, eb, rtol=1e-6, maxiter=3000, want_sigma=False)
    p = s.project_compatible(cold.epsilon, eb)
    assert (p - cold.epsilon).abs().max() < 1e-5 * cold.epsilon.abs().max()
    noise = cold.epsilon + 0.3 * torch.randn_like(cold.epsilon)
    q = s.project_compatible(noise, eb)
    q2 = s.project_compatible(q, eb)
    assert (q2 - q).abs().max() < 1e-5 * q.abs().max()
    e0 = s.solve(lm, mu, eb, maxiter=0, want_sigma=False).residual
    warm = s.solve(lm, mu, eb, rtol=1e-6, maxiter=3000, want_sigma=False, epsilon0=q, e0_ref=e0)
    assert (warm.status == 1).all()
    rel = np.linalg.norm(warm.mean_sigma - cold.mean_sigma) / np.linalg.norm(cold.mean_sigma)
    assert rel < 1e-5


def test_warm_start_in_anderson_history():
    """A warm start placed in the Anderson history: the exact solution cuts the solve to a
    few updates, a poor compatible field still converges to the cold C_eff."""
    import torch
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.learned import warm_start as W
    from jaxmaterials_b200.solver import Solver

    ind = torch.as_tensor(W.indicators(W.structure_params(1, 32, 12), workers=1)).cuda()
    lm, mu = W.lame_from_indicator(ind)
    g = GridSpec(32, 32, 32, 32.0, 32.0, 32.0)
    s = Solver(g, batch=6, depth=5)
    eb = np.eye(6, dtype=np.float32)
    cold = s.solve(lm, mu, eb, rtol=1e-6, maxiter=3000, want_sigma=False)
    s.set_warm_history(True)
    exact = s.solve(lm, mu, eb, rtol=1e-6, maxiter=3000, want_sigma=False, epsilon0=cold.epsilon)
    assert (exact.status == 1).all() and (exact.iters <= 4).all()
    # (the projection switches the history mode off for its own update)
    poor = s.project_compatible(cold.epsilon + 0.5 * torch.randn_like(cold.epsilon), eb)
    assert (poor - cold.epsilon).abs().max() > 0.1
    r = s.solve(lm, mu, eb, rtol=1e-6, maxiter=3000, want_sigma=False, epsilon0=poor)
    s.set_warm_history(False)
    assert (r.status == 1).all()
    for x in (exact, r):
        rel = np.linalg.norm(x.mean_sigma - cold.mean_sigma) / np.linalg.norm(cold.mean_sigma)
        assert rel < 1e-5
