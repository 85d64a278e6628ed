"""Spectral-convolution network (Fourier neural operator) that maps the Lame fields of a
microstructure to the strain fields of its six unit load cases, used as a warm start.

Architecture, for a grid of nv voxels:
    a  = ((lambda - c_l) / s_l, (mu - c_m) / s_m)                  2 channels
    h0 = W_lift a + b_lift                                          width channels
    h_{l+1} = GELU(W_l h_l + b_l + irfftn(R_l . rfftn(h_l)))        l = 0 .. layers-1
    out = W_proj h_L + b_proj                                       36 channels
R_l mixes channels per retained Fourier mode (modes[0] x modes[1] x modes[2]: the lowest
|kx|, |ky| and kz >= 0); out[6 k + c] is component c of the strain fluctuation for the
unit load e_k. Weights are BF16 in the kernels (FP32 master copies here), accumulation
FP32; the 32-channel pointwise layers run on the tensor cores with their activations
rounded to BF16. Every operation of the network, forward and backward, runs in the kernels
of include/spectral_net.h: the pointwise layers, the per-mode mixing and the truncated
transforms between the fields and their retained modes (direct sums over those modes
instead of full 3-D FFTs).
"""

import ctypes
import math

import numpy as np

from .. import _lib
from ..data.fibres import FIBRE_LAME, MATRIX_LAME

# input normalisation: the two phases map to -1 / +1
LAMBDA_CENTRE = 0.5 * (MATRIX_LAME[0] + FIBRE_LAME[0])
LAMBDA_SCALE = 0.5 * (FIBRE_LAME[0] - MATRIX_LAME[0])
MU_CENTRE = 0.5 * (MATRIX_LAME[1] + FIBRE_LAME[1])
MU_SCALE = 0.5 * (FIBRE_LAME[1] - MATRIX_LAME[1])


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def _stream(t):
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _functions():
    import torch

    lib = _lib.load()

    class Pointwise(torch.autograd.Function):
        """y = act(W x + b + add) over [B][cin][nv] -> [B][cout][nv]."""

        @staticmethod
        def forward(ctx, x, w, b, add, act):
            x = x.contiguous()
            bsz, cin = x.shape[0], x.shape[1]
            nv = x[0, 0].numel()
            cout = w.shape[0]
            w16 = w.detach().to(torch.bfloat16).contiguous()
            y = torch.empty((bsz, cout) + tuple(x.shape[2:]), device=x.device, dtype=torch.float32)
            pre = torch.empty_like(y) if act else None
            addc = add.contiguous() if add is not None else None
            _lib.check_net(lib.lsn_pointwise_forward(bsz, cin, cout, nv, _ptr(x), _ptr(w16),
                                                     _ptr(b.detach()), _ptr(addc), _ptr(pre),
                                                     _ptr(y), int(act), _stream(x)),
                           "lsn_pointwise_forward")
            ctx.save_for_backward(x, w16, pre)
            ctx.act = int(act)
            ctx.has_add = add is not None
            return y

        @staticmethod
        def backward(ctx, dy):
            x, w16, pre = ctx.saved_tensors
            dy = dy.contiguous()
            bsz, cin = x.shape[0], x.shape[1]
            nv = x[0, 0].numel()
            cout = w16.shape[0]
            dx = torch.empty_like(x) if ctx.needs_input_grad[0] else None
            want_add = ctx.has_add and ctx.needs_input_grad[3]
            dpre = torch.empty_like(dy) if (want_add and ctx.act) else None
            dw = torch.zeros((cout, cin), device=x.device, dtype=torch.float32)
            db = torch.zeros((cout,), device=x.device, dtype=torch.float32)
            _lib.check_net(lib.lsn_pointwise_backward(bsz, cin, cout, nv, _ptr(x), _ptr(w16),
                                                      _ptr(pre), _ptr(dy), ctx.act, _ptr(dx),
                                                      _ptr(dpre), _ptr(dw), _ptr(db),
                                                      _stream(x)),
                           "lsn_pointwise_backward")
            dadd = (dpre if ctx.act else dy) if want_add else None
            return dx, dw, db, dadd, None

    class Spectral(torch.autograd.Function):
        """yh[b, o, k] = sum_i xh[b, i, k] W[k, i, o] on the retained modes (zero elsewhere)."""

        @staticmethod
        def forward(ctx, xh, w, n, modes):
            xh = xh.contiguous()
            bsz, cin = xh.shape[0], xh.shape[1]
            cout = w.shape[2]
            w16 = w.detach().to(torch.bfloat16).contiguous()
            yh = torch.zeros((bsz, cout) + tuple(xh.shape[2:]), device=xh.device,
                             dtype=torch.complex64)
            nn = (ctypes.c_int * 3)(*n)
            mm = (ctypes.c_int * 3)(*modes)
            _lib.check_net(lib.lsn_spectral_forward(bsz, cin, cout, nn, mm, _ptr(xh), _ptr(w16),
                                                    _ptr(yh), _stream(xh)),
                           "lsn_spectral_forward")
            ctx.save_for_backward(xh, w16)
            ctx.n, ctx.modes = n, modes
            return yh

        @staticmethod
        def backward(ctx, dyh):
            xh, w16 = ctx.saved_tensors
            dyh = dyh.contiguous()
            bsz, cin = xh.shape[0], xh.shape[1]
            cout = w16.shape[2]
            dxh = torch.zeros_like(xh) if ctx.needs_input_grad[0] else None
            dw = torch.empty(tuple(w16.shape), device=xh.device, dtype=torch.float32)
            nn = (ctypes.c_int * 3)(*ctx.n)
            mm = (ctypes.c_int * 3)(*ctx.modes)
            _lib.check_net(lib.lsn_spectral_backward(bsz, cin, cout, nn, mm, _ptr(xh), _ptr(w16),
                                                     _ptr(dyh), _ptr(dxh), _ptr(dw),
                                                     _stream(xh)),
                           "lsn_spectral_backward")
            return dxh, dw, None, None

    def _trunc(kind, f_or_x, n, modes, scale, w_int, out):
        bc = out.shape[0] * out.shape[1]
        work = torch.empty((bc, n[0], modes[1], modes[2]), device=out.device, dtype=torch.complex64)
        nn = (ctypes.c_int * 3)(*n)
        mm = (ctypes.c_int * 3)(*modes)
        fn = lib.lsn_truncated_forward if kind == "fwd" else lib.lsn_truncated_inverse
        _lib.check_net(fn(bc, nn, mm, _ptr(f_or_x), _ptr(work), _ptr(out), float(scale), float(w_int),
                          _stream(out)), "lsn_truncated_" + kind)
        return out

    class TruncatedForward(torch.autograd.Function):
        """h [B, C, nx, ny, nz] -> its retained modes [B, C, mx, my, mz] (numpy rfftn
        restricted to them); backward: the transposed map (truncated inverse, no weights)."""

        @staticmethod
        def forward(ctx, h, n, modes):
            h = h.contiguous()
            out = torch.empty(tuple(h.shape[:2]) + tuple(modes), device=h.device, dtype=torch.complex64)
            ctx.n, ctx.modes = n, modes
            return _trunc("fwd", h, n, modes, 1.0, 1.0, out)

        @staticmethod
        def backward(ctx, dx):
            dx = dx.contiguous()
            dh = torch.empty(tuple(dx.shape[:2]) + tuple(ctx.n), device=dx.device, dtype=torch.float32)
            return _trunc("inv", dx, ctx.n, ctx.modes, 1.0, 1.0, dh), None, None

    class TruncatedInverse(torch.autograd.Function):
        """Retained modes [B, C, mx, my, mz] -> real field (numpy irfftn of the zero-padded
        half spectrum); backward: the transposed map (truncated forward, same weights)."""

        @staticmethod
        def forward(ctx, y, n, modes):
            y = y.contiguous()
            out = torch.empty(tuple(y.shape[:2]) + tuple(n), device=y.device, dtype=torch.float32)
            ctx.n, ctx.modes = n, modes
            return _trunc("inv", y, n, modes, 1.0 / (n[0] * n[1] * n[2]), 2.0, out)

        @staticmethod
        def backward(ctx, ds):
            ds = ds.contiguous()
            dy = torch.empty(tuple(ds.shape[:2]) + tuple(ctx.modes), device=ds.device, dtype=torch.complex64)
            n = ctx.n
            return _trunc("fwd", ds, n, ctx.modes, 1.0 / (n[0] * n[1] * n[2]), 2.0, dy), None, None

    return Pointwise, Spectral, TruncatedForward, TruncatedInverse


_FN = None


def functions():
    global _FN
    if _FN is None:
        _FN = _functions()
    return _FN


class SpectralNet:
    """The warm-start network. Parameters are FP32 torch tensors (``params``, a dict);
    the kernels read BF16 copies made at every call."""

    def __init__(self, width=32, layers=4, modes=(12, 12, 12), out_channels=36, seed=0,
                 device="cuda"):
        import torch

        self.width, self.layers, self.modes = int(width), int(layers), tuple(int(m) for m in modes)
        self.out_channels = int(out_channels)
        g = torch.Generator().manual_seed(seed)
        nm = self.modes[0] * self.modes[1] * self.modes[2]

        def uni(shape, bound):
            return (torch.rand(shape, generator=g) * 2.0 - 1.0) * bound

        p = {"lift_w": uni((width, 2), 1.0 / math.sqrt(2)), "lift_b": torch.zeros(width)}
        for l in range(layers):
            p[f"spec{l}"] = uni((nm, width, width, 2), 1.0 / width)
            p[f"w{l}"] = uni((width, width), 1.0 / math.sqrt(width))
            p[f"b{l}"] = torch.zeros(width)
        p["proj_w"] = uni((out_channels, width), 1.0 / math.sqrt(width))
        p["proj_b"] = torch.zeros(out_channels)
        self.params = {k: v.to(device).requires_grad_(True) for k, v in p.items()}

    def parameter_count(self):
        return int(sum(v.numel() for v in self.params.values()))

    @staticmethod
    def encode(lmbda, mu):
        """Network input [B, 2, nx, ny, nz] from Lame fields [B, nx, ny, nz]."""
        import torch

        return torch.stack([(lmbda - LAMBDA_CENTRE) / LAMBDA_SCALE,
                            (mu - MU_CENTRE) / MU_SCALE], dim=1).float().contiguous()

    def forward(self, a):
        """a: [B, 2, nx, ny, nz] float32 CUDA tensor -> [B, out_channels, nx, ny, nz]."""
        import torch

        pointwise, spectral, tfwd, tinv = functions()
        p = self.params
        n = tuple(int(s) for s in a.shape[2:])
        # the mixing kernels read and write the dense retained-mode layout, which is the
        # half-spectrum layout of a (mx, my, 2 (mz - 1)) grid
        dense = (self.modes[0], self.modes[1], 2 * (self.modes[2] - 1))
        h = pointwise.apply(a, p["lift_w"], p["lift_b"], None, 0)
        for l in range(self.layers):
            xm = tfwd.apply(h, n, self.modes)
            ym = spectral.apply(xm, p[f"spec{l}"], dense, self.modes)
            s = tinv.apply(ym, n, self.modes)
            h = pointwise.apply(h, p[f"w{l}"], p[f"b{l}"], s, 1)
        return pointwise.apply(h, p["proj_w"], p["proj_b"], None, 0)

    __call__ = forward

    def warm_start(self, lmbda, mu, batch=4):
        """Strain fields of the six unit loads: [B, 6, 6, nx, ny, nz] with
        eps[b, k] = e_k + (predicted fluctuation with its mean removed). Runs the network
        on `batch` structures at a time."""
        import torch

        outs = []
        with torch.no_grad():
            for i in range(0, lmbda.shape[0], batch):
                outs.append(self.forward(self.encode(lmbda[i:i + batch], mu[i:i + batch])))
        out = torch.cat(outs)
        b = out.shape[0]
        out = out.view(b, 6, 6, *out.shape[2:])
        out = out - out.mean(dim=(-3, -2, -1), keepdim=True)
        eye = torch.eye(6, device=out.device, dtype=out.dtype).view(1, 6, 6, 1, 1, 1)
        return out + eye

    def state_dict(self):
        import torch

        sd = {k: v.detach().cpu() for k, v in self.params.items()}
        sd["_config"] = torch.tensor([self.width, self.layers, *self.modes, self.out_channels])
        return sd

    @classmethod
    def from_state_dict(cls, sd, device="cuda"):
        cfg = [int(v) for v in sd["_config"]]
        net = cls(width=cfg[0], layers=cfg[1], modes=tuple(cfg[2:5]), out_channels=cfg[5],
                  device=device)
        for k in net.params:
            net.params[k].data.copy_(sd[k].to(net.params[k].dtype))
        return net


class Adam:
    """Adam over the network's FP32 parameters with the library's kernel."""

    def __init__(self, params, lr=1e-3, betas=(0.9, 0.999), eps=1e-8):
        import torch

        self.params = list(params)
        self.lr, self.betas, self.eps = lr, betas, eps
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.t = 0

    def step(self, lr=None):
        lib = _lib.load()
        self.t += 1
        for p, m, v in zip(self.params, self.m, self.v):
            if p.grad is None:
                continue
            g = p.grad.contiguous()
            _lib.check_net(lib.lsn_adam(p.numel(), _ptr(p.data), _ptr(g), _ptr(m), _ptr(v),
                                        float(self.lr if lr is None else lr), self.betas[0],
                                        self.betas[1], self.eps, self.t, _stream(p)),
                           "lsn_adam")

    def zero_grad(self):
        for p in self.params:
            p.grad = None
