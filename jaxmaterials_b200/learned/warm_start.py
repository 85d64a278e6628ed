"""Training data, training loop and warm-start evaluation of the spectral network.

Data: seeded structures of the batched workload's distribution (2-6 cross-ply layers,
fibre radius 2-5 voxels, volume fraction 0.30-0.55) at one grid size, solved by the
library for the six unit loads (Anderson, tol 1e-6). Inputs are kept on the device as
phase indicators (uint8), targets as BF16 strain fluctuations eps - e_k [36][nv].

Evaluation: for held-out structures, the cold solve starts from eps = e_k; the warm
solve starts from the compatible part of the network's prediction (the iteration keeps
any incompatible part of its start, see Solver.project_compatible), the scaled warm solve
from e_k + theta (prediction - e_k) with theta minimising the start's residual, and the
history solve from e_k with the prediction as the second Anderson iterate
(Solver.set_warm_history). The warm and scaled solves stop at the same absolute residual as
the cold one (its threshold is rtol times the cold start's first criterion, obtained
from a maxiter = 0 solve and passed as the reference criterion). Reported: iterations of
both, wall time of both (the warm time includes inference and the extra criterion
evaluation), and the network's own C_eff (mean stress of the predicted strains) against
the solved C_eff.

    python -m jaxmaterials_b200.learned.warm_start --train 4096 --test 512 --n 64
"""

import json
import math
import multiprocessing as mp
import os
import time

import numpy as np

from ..data import fibres
from ..data.fibres import FIBRE_LAME, MATRIX_LAME


def structure_params(count, n, seed):
    rng = np.random.default_rng(seed)
    return [dict(n=n, nlayers=int(rng.integers(2, 7)), radius=float(rng.uniform(2.0, 5.0)),
                 volume_fraction=float(rng.uniform(0.30, 0.55)),
                 seed=int(rng.integers(0, 2**31 - 1))) for _ in range(count)]


def _indicator(p):
    st = fibres.generate_layered_fibres(p["n"], p["nlayers"], p["radius"], p["volume_fraction"],
                                        p["seed"])
    return fibres.fibre_indicator(st).astype(np.uint8)


def indicators(params, workers=None):
    """Phase indicators (1 = fibre) of the structures, built on host cores (spawned pool)."""
    workers = workers or min(16, os.cpu_count() or 1)
    if workers <= 1 or len(params) < 8:
        return np.stack([_indicator(p) for p in params])
    with mp.get_context("spawn").Pool(workers) as pool:
        return np.stack(pool.map(_indicator, params, chunksize=8))


def lame_from_indicator(ind):
    """(lambda, mu) float32 device tensors from a uint8 indicator tensor."""
    import torch

    f = ind.bool()
    one = torch.ones((), device=ind.device, dtype=torch.float32)
    lm = torch.where(f, one * FIBRE_LAME[0], one * MATRIX_LAME[0])
    mu = torch.where(f, one * FIBRE_LAME[1], one * MATRIX_LAME[1])
    return lm.contiguous(), mu.contiguous()


def solve_dataset(ind, depth=5, rtol=1e-6, chunk=32, maxiter=5000):
    """Strain fields of the six unit loads for every structure: BF16 fluctuation targets
    [count, 36, n, n, n] on the device, plus iterations [count, 6]."""
    import torch
    from .. import GridSpec
    from ..solver import Solver

    count, n = ind.shape[0], ind.shape[1]
    g = GridSpec(n, n, n, float(n), float(n), float(n))
    chunk = min(chunk, count)
    s = Solver(g, batch=6 * chunk, depth=depth)
    targets = torch.empty((count, 36, n, n, n), device="cuda", dtype=torch.bfloat16)
    iters = np.zeros((count, 6), dtype=np.int32)
    eye = torch.eye(6, device="cuda").view(1, 6, 6, 1, 1, 1)
    for c0 in range(0, count, chunk):
        c = min(chunk, count - c0)
        lm, mu = lame_from_indicator(ind[c0:c0 + c])
        r = s.solve(lm, mu, np.tile(np.eye(6, dtype=np.float32), (c, 1)), rtol=rtol,
                    maxiter=maxiter, want_sigma=False)
        if not (r.status == 1).all():
            raise RuntimeError("training solve did not converge")
        eps = r.epsilon.view(c, 6, 6, n, n, n)
        targets[c0:c0 + c] = (eps - eye).view(c, 36, n, n, n).to(torch.bfloat16)
        iters[c0:c0 + c] = r.iters.reshape(c, 6)
    s.close()
    return targets, iters


def train(net, ind, targets, epochs=20, batch=8, lr=2e-3, seed=0, log=None):
    """Adam on the mean squared error of the predicted fluctuations, cosine learning rate.
    Returns the per-epoch mean losses."""
    import torch
    from .network import Adam, SpectralNet

    count = ind.shape[0]
    opt = Adam(net.params.values(), lr=lr)
    steps_per_epoch = max(1, count // batch)
    total = epochs * steps_per_epoch
    g = torch.Generator(device="cpu").manual_seed(seed)
    losses = []
    step = 0
    for ep in range(epochs):
        perm = torch.randperm(count, generator=g)
        acc = torch.zeros((), device="cuda")
        for i in range(steps_per_epoch):
            idx = perm[i * batch:(i + 1) * batch].cuda()
            lm, mu = lame_from_indicator(ind[idx])
            out = net(SpectralNet.encode(lm, mu))
            loss = torch.mean((out - targets[idx].float()) ** 2)
            opt.zero_grad()
            loss.backward()
            opt.step(lr=lr * 0.5 * (1.0 + math.cos(math.pi * step / total)))
            acc += loss.detach()
            step += 1
        losses.append(float(acc) / steps_per_epoch)
        if log:
            log(f"epoch {ep}: loss {losses[-1]:.4e}")
    return losses


def residual_norm(result):
    """Unnormalised equilibrium residual of a maxiter = 0 solve: the criterion times the
    Voigt-weighted norm of the mean stress (the criterion's denominator up to N)."""
    w = np.array([1.0, 1.0, 1.0, 2.0, 2.0, 2.0])
    return result.residual * np.sqrt((w * result.mean_sigma ** 2).sum(axis=1))


def scaled_start(s, lm, mu, eb, eps):
    """eps_bar + theta (eps - eps_bar) with theta per instance minimising the residual of
    the start. eps must be compatible (Solver.project_compatible). The residual is affine
    in theta, so its square is a quadratic fixed by three criterion evaluations (theta =
    0, 1, -1), each a maxiter = 0 solve. Returns (start, theta, e0 of the cold start)."""
    import torch

    b = eps.shape[0]
    ebt = torch.as_tensor(eb, device=eps.device).view(b, 6, 1, 1, 1)
    d = eps - ebt
    r0 = s.solve(lm, mu, eb, maxiter=0, want_sigma=False)
    rp = s.solve(lm, mu, eb, maxiter=0, want_sigma=False, epsilon0=ebt + d)
    rm = s.solve(lm, mu, eb, maxiter=0, want_sigma=False, epsilon0=ebt - d)
    a, p2, m2 = residual_norm(r0) ** 2, residual_norm(rp) ** 2, residual_norm(rm) ** 2
    curv = 0.5 * (p2 + m2) - a
    slope = 0.25 * (p2 - m2)
    theta = np.where(curv > 0, np.clip(-slope / np.where(curv > 0, curv, 1.0), 0.0, 2.0), 0.0)
    th = torch.as_tensor(theta, device=eps.device, dtype=eps.dtype).view(b, 1, 1, 1, 1)
    return ebt + th * d, theta, r0.residual


def evaluate(net, ind, depth=5, rtol=1e-6, chunk=16, maxiter=5000):
    """Cold against warm-started solves of the structures in `ind` (uint8 [count, n, n, n]
    on the device). Returns a dict of totals and per-structure arrays."""
    import torch
    from .. import GridSpec
    from ..solver import Solver

    count, n = ind.shape[0], ind.shape[1]
    g = GridSpec(n, n, n, float(n), float(n), float(n))
    chunk = min(chunk, count)
    s = Solver(g, batch=6 * chunk, depth=depth)
    eye6 = np.eye(6, dtype=np.float32)
    out = {"cold_iters": [], "warm_iters": [], "scaled_iters": [], "hist_iters": [], "theta": [],
           "c_eff": [], "c_eff_warm": [], "c_eff_scaled": [], "c_eff_hist": [], "c_eff_net": [],
           "cold_s": 0.0, "warm_s": 0.0, "scaled_s": 0.0, "hist_s": 0.0, "inference_s": 0.0}
    for c0 in range(0, count, chunk):
        c = min(chunk, count - c0)
        lm, mu = lame_from_indicator(ind[c0:c0 + c])
        eb = np.tile(eye6, (c, 1))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cold = s.solve(lm, mu, eb, rtol=rtol, maxiter=maxiter, want_sigma=False)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        eps0 = net.warm_start(lm, mu)                      # [c, 6, 6, n, n, n]
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        eps0 = s.project_compatible(eps0.reshape(6 * c, 6, n, n, n), eb)
        torch.cuda.synchronize()
        t2b = time.perf_counter()
        e0 = s.solve(lm, mu, eb, maxiter=0, want_sigma=False).residual
        warm = s.solve(lm, mu, eb, rtol=rtol, maxiter=maxiter, want_sigma=False,
                       epsilon0=eps0, e0_ref=e0)
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        start, theta, e0s = scaled_start(s, lm, mu, eb, eps0)
        scaled = s.solve(lm, mu, eb, rtol=rtol, maxiter=maxiter, want_sigma=False,
                         epsilon0=start, e0_ref=e0s)
        torch.cuda.synchronize()
        t4 = time.perf_counter()
        # the prediction as the second entry of the Anderson history (after the cold start)
        s.set_warm_history(True)
        hist = s.solve(lm, mu, eb, rtol=rtol, maxiter=maxiter, want_sigma=False, epsilon0=eps0)
        s.set_warm_history(False)
        torch.cuda.synchronize()
        t5 = time.perf_counter()
        out["hist_s"] += (t2b - t1) + (t5 - t4)
        out["hist_iters"].append(hist.iters.reshape(c, 6))
        out["c_eff_hist"].append(hist.mean_sigma.reshape(c, 6, 6))
        out["cold_s"] += t1 - t0
        out["warm_s"] += t3 - t1
        out["scaled_s"] += (t2b - t1) + (t4 - t3)
        out["inference_s"] += t2 - t1
        if not ((cold.status == 1).all() and (warm.status == 1).all() and (scaled.status == 1).all()):
            raise RuntimeError("evaluation solve did not converge")
        out["cold_iters"].append(cold.iters.reshape(c, 6))
        out["warm_iters"].append(warm.iters.reshape(c, 6))
        out["scaled_iters"].append(scaled.iters.reshape(c, 6))
        out["theta"].append(theta.reshape(c, 6))
        out["c_eff_scaled"].append(scaled.mean_sigma.reshape(c, 6, 6))
        out["c_eff"].append(cold.mean_sigma.reshape(c, 6, 6))
        out["c_eff_warm"].append(warm.mean_sigma.reshape(c, 6, 6))
        # network C_eff: mean stress of the (projected) predicted strain fields
        e = eps0.view(c, 6, 6, n, n, n).double()
        tr = e[:, :, 0] + e[:, :, 1] + e[:, :, 2]
        lmd, mud = lm.double().unsqueeze(1), mu.double().unsqueeze(1)
        sig = 2.0 * mud.unsqueeze(2) * e
        sig[:, :, :3] += (lmd * tr).unsqueeze(2)
        out["c_eff_net"].append(sig.mean(dim=(-3, -2, -1)).cpu().numpy())
        del eps0, e, sig
    s.close()
    for k in ("cold_iters", "warm_iters", "scaled_iters", "hist_iters", "theta", "c_eff",
              "c_eff_warm", "c_eff_scaled", "c_eff_hist", "c_eff_net"):
        out[k] = np.concatenate(out[k])
    return out


def summarise(ev, n):
    """JSON-ready summary of evaluate()."""
    c, cw, cn = ev["c_eff"], ev["c_eff_warm"], ev["c_eff_net"]

    def rel(a, b):
        return np.linalg.norm(a - b, axis=(1, 2)) / np.linalg.norm(b, axis=(1, 2))

    solves = 6 * c.shape[0]
    return {
        "grid": n,
        "structures": int(c.shape[0]),
        "cold_iters_per_solve": float(ev["cold_iters"].mean()),
        "warm_iters_per_solve": float(ev["warm_iters"].mean()),
        "iterations_saved": float(1.0 - ev["warm_iters"].mean() / ev["cold_iters"].mean()),
        "cold_solves_per_s": solves / ev["cold_s"],
        "warm_solves_per_s": solves / ev["warm_s"],
        "inference_s_per_structure": ev["inference_s"] / c.shape[0],
        "scaled_iters_per_solve": float(ev["scaled_iters"].mean()),
        "scaled_iterations_saved": float(1.0 - ev["scaled_iters"].mean() / ev["cold_iters"].mean()),
        "scaled_solves_per_s": solves / ev["scaled_s"],
        "theta_mean": float(ev["theta"].mean()),
        "history_iters_per_solve": float(ev["hist_iters"].mean()),
        "history_iterations_saved": float(1.0 - ev["hist_iters"].mean() / ev["cold_iters"].mean()),
        "history_solves_per_s": solves / ev["hist_s"],
        "c_eff_history_vs_cold_rel_max": float(rel(ev["c_eff_hist"], c).max()),
        "c_eff_warm_vs_cold_rel_max": float(max(rel(cw, c).max(), rel(ev["c_eff_scaled"], c).max())),
        "c_eff_network_rel_mean": float(rel(cn, c).mean()),
        "c_eff_network_rel_max": float(rel(cn, c).max()),
    }


def main():
    import argparse

    import torch
    from .network import SpectralNet

    ap = argparse.ArgumentParser(description="train and evaluate the warm-start network")
    ap.add_argument("--train", type=int, default=4096)
    ap.add_argument("--test", type=int, default=512)
    ap.add_argument("--test-large", type=int, default=32, help="held-out structures at 2n")
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--depth", type=int, default=5)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default="spectral_net.pt")
    ap.add_argument("--report", default=None)
    ap.add_argument("--load", default=None, help="evaluate a saved network instead of training")
    args = ap.parse_args()

    def log(msg):
        print(msg, flush=True)

    report = {"config": vars(args)}
    t = time.perf_counter()
    test_np = indicators(structure_params(args.test, args.n, args.seed + 1))
    big_np = (indicators(structure_params(args.test_large, 2 * args.n, args.seed + 2))
              if args.test_large > 0 else None)
    if args.load:
        net = SpectralNet.from_state_dict(torch.load(args.load))
    else:
        ind = torch.as_tensor(indicators(structure_params(args.train, args.n, args.seed))).cuda()
        log(f"structures: {time.perf_counter() - t:.1f} s")
        t = time.perf_counter()
        targets, it = solve_dataset(ind, depth=args.depth)
        torch.cuda.synchronize()
        report["data_s"] = time.perf_counter() - t
        report["data_iters_per_solve"] = float(it.mean())
        log(f"solver data: {report['data_s']:.1f} s, {it.mean():.1f} iterations per solve")
        net = SpectralNet(seed=args.seed)
        report["parameters"] = net.parameter_count()
        t = time.perf_counter()
        report["losses"] = train(net, ind, targets, epochs=args.epochs, batch=args.batch,
                                 lr=args.lr, seed=args.seed, log=log)
        torch.cuda.synchronize()
        report["train_s"] = time.perf_counter() - t
        log(f"training: {report['train_s']:.1f} s")
        del targets, ind
        torch.cuda.empty_cache()
        torch.save(net.state_dict(), args.out)
    report["eval"] = summarise(evaluate(net, torch.as_tensor(test_np).cuda(), depth=args.depth),
                               args.n)
    log(json.dumps(report["eval"]))
    if big_np is not None:
        report["eval_large"] = summarise(evaluate(net, torch.as_tensor(big_np).cuda(),
                                                  depth=args.depth, chunk=4), 2 * args.n)
        log(json.dumps(report["eval_large"]))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
