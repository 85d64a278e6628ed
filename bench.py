"""Benchmark: effective-stiffness solves of a 128^3 cross-ply fibre composite on B200.

Workload (one "step"): the six unit-load Lippmann-Schwinger solves (tol 1e-6, rtol on the
normalised equilibrium residual) of one seeded 128^3 microstructure with 4 alternating
0/90 layers, fibre radius 4 voxels, 45% fibre volume fraction, phase contrast ~26
(matrix lambda, mu = 2.593, 1.111; fibres 19.44, 29.17), solved as one batch of six
instances; outputs the 6x6 effective stiffness. Each rank solves its own microstructure
(seed = rank): weak scaling, no collective on the data path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Rank 0 prints one JSON line. `value` = solves/s over all ranks with inputs resident in
HBM; `e2e` = the same through the public API from pinned host buffers (lambda, mu in,
C_eff out) per step.
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s & voxel-iter/s at 1e-6 resid: learned+batched vs plain (1 B200)"
WORKLOAD = "c2_128"
FALLBACK_HBM_GBS = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--depth", type=int, default=5)
    p.add_argument("--no-plain", action="store_true", help="skip the plain-iteration comparison")
    p.add_argument("--cpu-sample-s", type=float, default=12.0)
    p.add_argument("--batched", type=int, default=512,
                   help="structures of the batched uneven-size workload (0: skip)")
    p.add_argument("--batched-plain", action="store_true",
                   help="also time the batched workload with the plain iteration")
    p.add_argument("--generator", type=int, default=16,
                   help="samples of the layered-fibre dataset generator leg (0: skip)")
    p.add_argument("--damage", type=int, default=128,
                   help="grid of the phase-field fracture step leg (0: skip)")
    p.add_argument("--aniso", type=int, default=128,
                   help="grid of the anisotropic C_eff leg (0: skip)")
    p.add_argument("--c2-256", type=int, default=1, dest="c2_256",
                   help="steps of the 256^3 config-2 leg (0: skip)")
    p.add_argument("--learned", type=int, default=32,
                   help="grid of the bounded learned warm-start leg (0: skip)")
    p.add_argument("--comparators", type=int, default=1,
                   help="time the cuFFT loop and the reference's CUDA library (0: skip)")
    # fixed-iteration runs for profilers (no JSON line): every pass of every iteration does
    # its full work (tolerances 0), on the seeded n^3 benchmark composite
    p.add_argument("--profile-case", action="store_true",
                   help="run --iters iterations of --batch load cases at --n^3 and exit")
    p.add_argument("--profile-net", type=int, default=0, metavar="N",
                   help="per-kernel device times of one training step of the warm-start "
                        "network at N^3 (batch --batch) and exit")
    p.add_argument("--layout", default="tuned", choices=["tuned", "tiled", "strided"],
                   help="--profile-case: spectrum layout between the y and x passes "
                        "(default: the autotuner's choice)")
    p.add_argument("--n", type=int, default=128)
    p.add_argument("--batch", type=int, default=2)
    p.add_argument("--iters", type=int, default=3)
    p.add_argument("--precision", default="fp32", choices=["fp32", "mixed", "fp64"])
    return p.parse_args()


def profile_case(args):
    """A fixed number of iterations (tolerances 0) of `--batch` unit loads on the seeded
    n^3 cross-ply composite (4 layers, r = 4, vf 0.45), for ncu launch lists and captures."""
    import torch

    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.data import fibres
    from jaxmaterials_b200.solver import Solver

    n = args.n
    st = fibres.generate_layered_fibres(n, 4, 4.0, 0.45, seed=0)
    lm, mu = fibres.lame_fields(st)
    g = GridSpec(n, n, n, float(n), float(n), float(n))
    s = Solver(g, batch=args.batch, depth=args.depth, precision=args.precision)
    s.set_device_loop(False)  # profilers do not see kernels inside conditional graphs
    if args.layout != "tuned":
        s.set_tiled(args.layout == "tiled")
        s.tile_variant(0)
    eb = np.eye(6, dtype=np.float32)[np.arange(args.batch) % 6]
    r = s.solve(lm, mu, eb, rtol=0.0, atol=0.0, maxiter=args.iters, want_sigma=False)
    torch.cuda.synchronize()
    print(f"n={n} batch={args.batch} depth={args.depth} iters={list(r.iters)} "
          f"launches={s.kernel_launches()}")
    s.close()


def profile_net(args):
    """Device time of every kernel of one training step of the warm-start network
    (forward, MSE loss, backward, Adam) on random inputs of its shape at n^3, batch
    `--batch`: torch.profiler (CUPTI) over three steps after three warm-up steps."""
    import torch
    from torch.profiler import ProfilerActivity, profile

    from jaxmaterials_b200.learned.network import Adam, SpectralNet

    n, bsz = args.profile_net, args.batch
    g = torch.Generator(device="cuda").manual_seed(0)
    net = SpectralNet(seed=0)
    opt = Adam(net.params.values(), lr=1e-3)
    lm = torch.rand((bsz, n, n, n), device="cuda", generator=g) * 17 + 2.5
    mu = torch.rand((bsz, n, n, n), device="cuda", generator=g) * 28 + 1.1
    tgt = torch.randn((bsz, 36, n, n, n), device="cuda", generator=g) * 0.1

    def step():
        out = net(SpectralNet.encode(lm, mu))
        loss = torch.mean((out - tgt) ** 2)
        opt.zero_grad()
        loss.backward()
        opt.step()

    for _ in range(3):
        step()
    torch.cuda.synchronize()
    t = time.perf_counter()
    for _ in range(3):
        step()
    torch.cuda.synchronize()
    print(f"n={n} batch={bsz} ms per step {(time.perf_counter() - t) / 3 * 1e3:.2f}")
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        for _ in range(3):
            step()
        torch.cuda.synchronize()
    print(prof.key_averages().table(sort_by="cuda_time_total", row_limit=25, max_name_column_width=60))


def generator_run(count, seed):
    """The reference's dataset generator in its own script's configuration
    (src/generate_data.py:14-56) for `count` samples, through
    jaxmaterials_b200.data.layered.benchmark (placement on the host cores, GPU voxelisation,
    whole pipeline with the six C_eff solves per sample), beside the oracle's NumPy
    voxelisation of the first sample (the reference's CPU code path, restated) as the CPU
    baseline and the check that both fields are equal."""
    from jaxmaterials_b200.data.layered import benchmark, reference_config_generator
    from oracle import fibres_oracle

    res, (sample, field) = benchmark(count, seed, keep_first=True)
    gen = reference_config_generator(1, seed)
    g = gen.grid_spec
    t = time.perf_counter()
    ref = fibres_oracle.material_properties((g.nx, g.ny, g.nz, g.Lx, g.Ly, g.Lz), gen.d_void,
                                            gen._values, *sample, dtype=np.float32)
    t_cpu = time.perf_counter() - t
    peak, peak_kind = measured_peak()
    gbs = res["voxelise_bytes_per_sample"] / (res["voxelise_ms_per_sample"] / 1000.0) / 1e9
    res.update({
        "placement_threads": os.cpu_count(),
        "voxelise_write_GBs": gbs, "voxelise_frac_of_peak": gbs / peak, "peak_source": peak_kind,
        "cpu_baseline": {"value": t_cpu, "unit": "s/sample", "cores": 1, "kind": "port",
                         "sample": "voxelisation of the first sample by the oracle's NumPy "
                                   "restatement of data.py:267-314"},
        "voxelise_matches_oracle": bool(np.array_equal(field, ref)),
        "pipeline": "placement + voxelisation + 6 plain solves per sample (rtol = atol = "
                    "1e-4, maxiter 100) + host copies",
    })
    return res


def damage_run(n):
    """One staggered step of the reference's phase-field fracture driver (tests/phasefield.py)
    on the n^3 benchmark composite through jaxmaterials_b200.solver.damage.benchmark, beside
    the oracle's NumPy damaged iteration (the reference's JAX code path, restated) timed on a
    bounded sample as the CPU baseline."""
    from jaxmaterials_b200.solver.damage import benchmark
    from oracle import damage_oracle as D
    from oracle import ls_oracle as O

    res = benchmark(n)
    m = 48
    rng = np.random.default_rng(0)
    lm = rng.uniform(1.0, 20.0, (m, m, m))
    mu = rng.uniform(1.0, 20.0, (m, m, m))
    dd = rng.uniform(0.0, 1.0, (m, m, m))
    t = time.perf_counter()
    D.elasticity_solve(lm, mu, np.array([0.0, 1e-3, 0, 0, 0, 0]), dd, 1e-6,
                       O.Grid(m, m, m, float(m), float(m), float(m)), rtol=0.0, atol=0.0, depth=3,
                       maxiter=3, dtype=np.float32, spectrum="half")
    per_vi = (time.perf_counter() - t) / (4 * m ** 3)  # 4 stress evaluations / transforms
    nv = n ** 3
    gpu_vips = res["damaged_iters"] * nv / (res["damaged_solve_ms"] / 1000.0)
    res.update({
        "damaged_voxel_iter_per_s": gpu_vips,
        "cpu_baseline": {"value": 1.0 / per_vi, "unit": "voxel-iterations/s", "cores": os.cpu_count(),
                         "kind": "port", "sample": f"3 damaged Anderson updates at {m}^3 "
                         "(oracle, FP32 fields, SciPy FFT on all cores)"},
    })
    return res


def aniso_run(n):
    """C_eff of a two-phase anisotropic n^3 field through
    jaxmaterials_b200.solver.anisotropic.benchmark, beside the oracle's NumPy iteration of
    the same law (the derivation restated; the reference has no solver for it) on a bounded
    sample as the CPU baseline."""
    from jaxmaterials_b200.solver.anisotropic import benchmark, two_phase_stiffness
    from oracle import aniso_oracle as A
    from oracle import ls_oracle as O

    res = benchmark(n)
    m = 48
    c = two_phase_stiffness(m, 1)
    t = time.perf_counter()
    A.lippmann_schwinger(c, np.eye(6)[0], O.Grid(m, m, m, float(m), float(m), float(m)),
                         rtol=0.0, atol=0.0, depth=5, maxiter=3, dtype=np.float32)
    per_vi = (time.perf_counter() - t) / (4 * m ** 3)
    res["cpu_baseline"] = {"value": 1.0 / per_vi, "unit": "voxel-iterations/s",
                           "cores": os.cpu_count(), "kind": "port",
                           "sample": f"3 anisotropic Anderson updates of one load at {m}^3 "
                                     "(oracle, FP32 fields, SciPy FFT on all cores)"}
    return res


def learned_run(n, train_count, test_count, epochs, depth):
    """The learned warm start (config 5) at a bounded size, so that the line carries it:
    `train_count` structures of the batched distribution at n^3 solved by the library
    (training data), the spectral network trained on them by the library's kernels
    (`epochs` epochs), then `test_count` held-out structures solved as batches cold,
    warm-started (compatible part of the prediction, the same absolute stop), with the
    scaled start and with the prediction in the Anderson history, and with the plain
    iteration (depth 0, cold). The full configuration (4096 structures at 64^3, 20 epochs)
    is `python -m jaxmaterials_b200.learned.warm_start`."""
    import torch
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.learned import warm_start as W
    from jaxmaterials_b200.learned.network import SpectralNet
    from jaxmaterials_b200.solver import Solver

    t0 = time.perf_counter()
    ind = torch.as_tensor(W.indicators(W.structure_params(train_count, n, 11))).cuda()
    targets, it = W.solve_dataset(ind, depth=depth)
    torch.cuda.synchronize()
    data_s = time.perf_counter() - t0
    net = SpectralNet(seed=0)
    t0 = time.perf_counter()
    losses = W.train(net, ind, targets, epochs=epochs)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    del targets, ind
    torch.cuda.empty_cache()
    test = torch.as_tensor(W.indicators(W.structure_params(test_count, n, 12))).cuda()
    chunk = min(16, test_count)
    res = W.summarise(W.evaluate(net, test, depth=depth, chunk=chunk), n)
    # the plain iteration on the same held-out structures, same batches
    g = GridSpec(n, n, n, float(n), float(n), float(n))
    s = Solver(g, batch=6 * chunk, depth=0)
    eye = np.eye(6, dtype=np.float32)
    plain_s, plain_it = 0.0, []
    for c0 in range(0, test_count, chunk):
        c = min(chunk, test_count - c0)
        lm, mu = W.lame_from_indicator(test[c0:c0 + c])
        s.solve(lm, mu, np.tile(eye, (c, 1)), rtol=1e-6, maxiter=5000, want_sigma=False)  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = s.solve(lm, mu, np.tile(eye, (c, 1)), rtol=1e-6, maxiter=5000, want_sigma=False)
        torch.cuda.synchronize()
        plain_s += time.perf_counter() - t0
        plain_it.append(r.iters)
    s.close()
    plain = 6 * test_count / plain_s
    best = max(("warm", res["warm_solves_per_s"]), ("scaled", res["scaled_solves_per_s"]),
               ("history", res["history_solves_per_s"]), key=lambda kv: kv[1])
    res.update({
        "train_structures": train_count, "epochs": epochs, "data_s": data_s, "train_s": train_s,
        "final_loss": losses[-1], "plain_iters_per_solve": float(np.concatenate(plain_it).mean()),
        "plain_solves_per_s": plain,
        "learned_batched_solves_per_s": best[1], "learned_mode": best[0],
        "learned_batched_vs_plain": best[1] / plain,
        "cold_anderson_batched_vs_plain": res["cold_solves_per_s"] / plain,
        "timing": "wall clock per batch of 16 structures x 6 loads after the network's inference "
                  "(included in the warm figures)",
    })
    return res


def batched_workload(count, seed):
    """Seeded structures with N in {32,48,64,96,128}, 2-6 layers, radius 2-5 voxels,
    volume fraction 0.30-0.55; cubic voxels of unit size."""
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.data import fibres

    lms, mus, gs = [], [], []
    for p in fibres.batch_structure_params(count, seed):
        st = fibres.generate_layered_fibres(p["n"], p["nlayers"], p["radius"],
                                            p["volume_fraction"], p["seed"])
        lm, mu = fibres.lame_fields(st)
        lms.append(lm)
        mus.append(mu)
        gs.append(GridSpec(*st.n, *st.extents))
    return lms, mus, gs


def batched_run(count, seed, depth):
    """One pass of lsb_c_eff_batch over `count` structures x 6 load cases, host inputs
    (lambda, mu) in and C_eff out; wall-clock around the blocking call. A warm-up pass
    over one structure per grid size runs first."""
    import torch
    from jaxmaterials_b200.solver import c_eff_batch

    lms, mus, gs = batched_workload(count, seed)
    seen = {}
    for i, g in enumerate(gs):
        seen.setdefault(g.shape, i)
    w = list(seen.values())
    c_eff_batch([lms[i] for i in w], [mus[i] for i in w], [gs[i] for i in w], depth=depth,
                maxiter=5000)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    C, iters, status = c_eff_batch(lms, mus, gs, depth=depth, maxiter=5000)
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    nv = np.array([g.number_of_voxels for g in gs], dtype=np.float64)
    by_n = {}
    for g, it in zip(gs, iters):
        by_n.setdefault(g.nx, []).append(float(it.mean()))
    # each grid size alone (same call, its structures only): where the time goes
    per_size = {}
    for n in sorted(by_n):
        idx = [i for i, g in enumerate(gs) if g.nx == n]
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        _, it_n, _ = c_eff_batch([lms[i] for i in idx], [mus[i] for i in idx], [gs[i] for i in idx],
                                 depth=depth, maxiter=5000)
        torch.cuda.synchronize()
        sec_n = time.perf_counter() - t1
        per_size[str(n)] = {"structures": len(idx), "seconds": sec_n,
                            "solves_per_s": 6 * len(idx) / sec_n,
                            "voxel_iter_per_s": float((nv[idx][:, None] * it_n).sum()) / sec_n}
    return {
        "per_size_alone": per_size,
        "seconds": sec,
        "solves": 6 * count,
        "value": 6 * count / sec,
        "unit": "solves/s",
        "voxel_iter_per_s": float((nv[:, None] * iters).sum()) / sec,
        "iters_per_solve": float(iters.mean()),
        "iters_per_solve_by_n": {str(k): float(np.mean(v)) for k, v in sorted(by_n.items())},
        "voxels_total": float(nv.sum()),
        "all_converged": bool((status == 1).all()),
        "h2d_bytes": float(8 * nv.sum()),
    }


def workload(seed):
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.data import fibres

    st = fibres.config_structure(WORKLOAD, seed=seed)
    lm, mu = fibres.lame_fields(st)
    g = GridSpec(*st.n, *st.extents)
    return st, g, lm, mu


def config_dict(st, depth):
    n = st.n
    return {
        "workload": f"{WORKLOAD}: {n[0]}^3 cross-ply, 4 layers 0/90, fibre radius 4 vox, "
                    f"vf {st.volume_fraction:.3f}, contrast ~26, 6 unit loads per step, "
                    f"tol rtol=1e-6 on the equilibrium residual, "
                    f"{'plain Moulinec-Suquet' if depth == 0 else f'Anderson m={depth}'}",
        "grid": list(n),
        "loads_per_step": 6,
        "anderson_depth": depth,
        "fields": "FP32 fields and FFTs, FP64 residual norms",
        "l2": "inputs larger than L2: 6 instances x (strain 50 MB + spectrum 51 MB) + Lame 17 MB",
    }


def fixture_iters(depth):
    path = os.path.join(ROOT, "tests", "golden", f"bench_{WORKLOAD}.npz")
    if os.path.exists(path):
        d = np.load(path)
        key = f"iters_d{depth}"
        if key in d:
            return [int(v) for v in d[key]]
    return None


def fixture_c_eff(depth):
    """FP64 oracle C_eff of the seed-0 benchmark structure (tests/golden/bench_c2_128.npz,
    made by tests/golden/make_bench_fixture.py), or None."""
    path = os.path.join(ROOT, "tests", "golden", f"bench_{WORKLOAD}.npz")
    if os.path.exists(path):
        d = np.load(path)
        key = f"ceff_d{depth}"
        if key in d:
            return np.asarray(d[key], dtype=np.float64)
    return None


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.idx)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def mark(self, which):
        """Record the wall time of the start/end of the timed region."""
        setattr(self, which, time.time())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        t0, t1 = getattr(self, "start", None), getattr(self, "end", None)
        lines = [l for ts, l in self.lines if t0 is None or t1 is None or t0 - 0.25 <= ts <= t1 + 0.25]
        if not lines:
            lines = [l for _, l in self.lines]
        for line in lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_sample(lm, mu, g, depth, budget_s, threads):
    """Oracle (NumPy/SciPy port of the reference JAX solver) on the host cores: time whole
    iterations of one load case until `budget_s` is spent. Returns (s per voxel-iter,
    iterations timed)."""
    from oracle import ls_oracle as O

    og = O.Grid(g.nx, g.ny, g.nz, g.Lx, g.Ly, g.Lz)
    eb = np.zeros(6)
    eb[0] = 1.0
    total_t, total_it = 0.0, 0
    chunk = 1
    while total_t < budget_s:
        t0 = time.perf_counter()
        _, _, it = O.lippmann_schwinger(lm, mu, eb, og, rtol=0.0, atol=0.0, depth=depth,
                                        maxiter=chunk, dtype=np.float32, workers=threads)
        total_t += time.perf_counter() - t0
        total_it += it
        chunk = min(chunk * 2, 4)
    return total_t / (total_it * g.number_of_voxels), total_it


def kernel_bytes(name, nv, nm, batch, depth):
    """Algorithmic bytes of one launch of the named kernel over `batch` instances of one
    structure (FP32 fields: real field 6 Nv 4 B, half spectrum 6 Nm 8 B, Lame pair 2 Nv 4 B;
    residual ring slots in FP16, 6 Nv 2 B; every Anderson ring slot filled)."""
    real, spec, lame = 6 * nv * 4, 6 * nm * 8, 2 * nv * 4
    res = 6 * nv * 2
    m1 = depth + 1
    table = {
        "x pass": batch * 2 * spec,                          # spectrum read + write
        "finalize": 0,
        "y pass inverse": batch * 2 * spec,
        "y pass forward": batch * 2 * spec,
        "z pass update": batch * (2 * spec + 2 * real) + lame,  # spectrum r/w, eps r/w
        "z pass residual rings": batch * (spec + real + res + real),  # spectrum, eps in; r, g out
        "anderson gram": batch * m1 * res,                   # every r slot
        "anderson solve": 0,
        "anderson combine": batch * (m1 * real + real),      # every g slot in, eps out
        "z pass stress": batch * (real + spec) + lame,        # eps in, spectrum out
        # fused slab pass: the z pass's bytes (the y transforms stay on chip)
        "slab update": batch * (2 * spec + 2 * real) + lame,
        "slab residual rings": batch * (spec + real + res + real),
        "slab stress": batch * (real + spec) + lame,
    }
    if name not in table:
        raise KeyError(f"no algorithmic byte count for kernel {name!r}")
    return table[name]


def step_roofline(solver, lm_d, mu_d, g, batch, depth, workload):
    """Every launch of one iteration of the timed step (CUDA events on the solver's stream,
    full workload), its algorithmic bytes and fraction of the measured HBM peak; the
    dominant launch is the line's roofline kernel."""
    prof = solver.profile_step(lm_d, mu_d, batch=batch, reps=5)
    nv, nm = g.number_of_voxels, g.number_of_modes
    peak, peak_kind = measured_peak()
    traffic_tab = {}
    tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            traffic_tab = json.load(f)
    kernels = []
    for name, ms in prof:
        b = kernel_bytes(name, nv, nm, batch, depth)
        gbs = b / (ms / 1000.0) / 1e9 if ms > 0 else 0.0
        kernels.append({"kernel": name, "ms": ms, "algorithmic_bytes": b, "GBs": gbs,
                        "frac": gbs / peak, "traffic": traffic_tab.get(f"{workload}:{name}")})
    top = max(kernels, key=lambda k: k["ms"])
    step_ms = sum(k["ms"] for k in kernels)
    step_bytes = sum(k["algorithmic_bytes"] for k in kernels)
    survey_b = 152.0 if depth == 0 else 200.0 + 72.0 * depth
    return {
        "pass_config": solver.pass_config(),
        "bound": "hbm",
        "kernel": top["kernel"],
        "achieved": top["GBs"],
        "peak": peak,
        "peak_source": peak_kind,
        "unit": "GB/s",
        "frac": top["frac"],
        "traffic": top["traffic"],
        "algorithmic_bytes_per_launch": top["algorithmic_bytes"],
        "ms_per_launch": top["ms"],
        "step": {"ms": step_ms, "algorithmic_bytes": step_bytes,
                 "bytes_per_voxel_iter": step_bytes / (nv * batch),
                 "GBs": step_bytes / (step_ms / 1000.0) / 1e9,
                 "frac": step_bytes / (step_ms / 1000.0) / 1e9 / peak,
                 "survey_bytes_per_voxel_iter": survey_b,
                 "frac_at_survey_bytes": survey_b * nv * batch / (step_ms / 1000.0) / 1e9 / peak},
        "kernels": kernels,
    }


def ceff_run(g, lm_d, mu_d, depth, steps, warmup, maxiter=5000, precision="mixed"):
    """`steps` timed six-load C_eff solves (CUDA events on the current stream) after
    `warmup` untimed ones; returns the figures and the last result."""
    import torch
    from jaxmaterials_b200.solver import CONVERGED, Solver

    eye = np.eye(6, dtype=np.float32)
    s = Solver(g, batch=6, depth=depth, precision=precision)
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        r = s.solve(lm_d, mu_d, eye, rtol=1e-6, atol=1e-20, maxiter=maxiter, want_sigma=False)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    its, f64 = 0, 0
    t0.record(stream)
    for _ in range(steps):
        r = s.solve(lm_d, mu_d, eye, rtol=1e-6, atol=1e-20, maxiter=maxiter, want_sigma=False)
        its += int(r.iters.sum())
        f64 += int(s.fp64_iters().sum())
    t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    nv = g.number_of_voxels
    out = {"value": 6.0 * steps / (ms / 1000.0), "unit": "solves/s",
           "ms_per_step": ms / steps, "iters_per_solve": its / (6 * steps),
           "voxel_iter_per_s": its * nv / (ms / 1000.0),
           "fp64_iteration_share": f64 / its if its else 0.0,
           "all_converged": bool(np.all(r.status == CONVERGED))}
    return out, r, s


def c2_256_run(steps):
    """Config 2's 256^3 grid (4 layers, r = 4, vf 0.45, six unit loads, tol 1e-6):
    Anderson m = 5 and plain, each with its C_eff error against an FP64 Anderson solve of
    the same structure by the library's FP64 path (lsb_solve_f64), and against the FP64
    CPU oracle's C_eff where tests/golden/bench_c2_256.npz holds it."""
    import torch
    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.data import fibres
    from jaxmaterials_b200.solver import Solver

    st = fibres.config_structure("c2_256", seed=0)
    lm, mu = fibres.lame_fields(st)
    g = GridSpec(*st.n, *st.extents)
    lm_d = torch.as_tensor(lm, device="cuda")
    mu_d = torch.as_tensor(mu, device="cuda")
    res = {"workload": f"c2_256: 256^3 cross-ply, 4 layers, r = 4, vf {st.volume_fraction:.3f}, "
                       "6 unit loads, tol 1e-6, FP32 fields (mixed precision)",
           "timing": "CUDA events around the timed steps, inputs resident in HBM"}
    s64 = Solver(g, batch=6, depth=5, precision="fp64")
    lm64 = lm_d.double()
    mu64 = mu_d.double()
    r64 = s64.solve(lm64, mu64, np.eye(6), rtol=1e-6, atol=1e-20, maxiter=5000, want_sigma=False)
    c64 = np.asarray(r64.mean_sigma, np.float64)
    res["fp64_iters_per_solve"] = float(np.mean(r64.iters))
    s64.close()
    del lm64, mu64
    torch.cuda.empty_cache()
    ref_oracle = None
    path = os.path.join(ROOT, "tests", "golden", "bench_c2_256.npz")
    if os.path.exists(path):
        ref_oracle = np.load(path)["ceff_d5"]
    for depth, key in ((5, "anderson"), (0, "plain")):
        out, r, s = ceff_run(g, lm_d, mu_d, depth, steps, 1)
        c = np.asarray(r.mean_sigma, np.float64)
        out["c_eff_rel_err_vs_fp64_gpu"] = float(np.linalg.norm(c - c64) / np.linalg.norm(c64))
        if ref_oracle is not None:
            out["c_eff_rel_err_vs_fp64_oracle"] = float(
                np.linalg.norm(c - ref_oracle) / np.linalg.norm(ref_oracle))
        if depth == 5:
            out["roofline"] = step_roofline(s, lm_d, mu_d, g, 6, depth, "c2_256")
            out["roofline"].pop("kernels")
        s.close()
        torch.cuda.empty_cache()
        res[key] = out
    if ref_oracle is not None:
        res["fp64_gpu_vs_oracle"] = float(np.linalg.norm(c64 - ref_oracle) / np.linalg.norm(ref_oracle))
    return res


def comparators_run(g, lm, mu, lm_d, mu_d, plain_iters, plain_ms_per_iter):
    """The same 128^3 six-load workload on (a) this solver's plain loop with its FFT stages
    replaced by cuFFT R2C/C2R batch 6 (libcufft_comparator.so: the pointwise kernels are
    this project's), and (b) the reference's own CUDA library (cuFFT + its SIMT kernels,
    built from its sources into oracle/_ref, called through its C ABI with host buffers,
    lambda first), against this solver's plain iteration."""
    import ctypes

    import torch

    out = {"own_plain_ms_per_iter": plain_ms_per_iter}
    lib_path = os.path.join(ROOT, "jaxmaterials_b200", "libcufft_comparator.so")
    try:
        lib = ctypes.CDLL(lib_path)
        lib.cmp_cufft_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_int]
        lib.cmp_cufft_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_int, ctypes.c_void_p, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_void_p, ctypes.c_int,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.cmp_cufft_destroy.argtypes = [ctypes.c_void_p]
        lib.cmp_cufft_last_error.restype = ctypes.c_char_p
        h = ctypes.c_void_p()
        vox = np.array(g.shape, np.int32)
        ext = np.array([g.Lx, g.Ly, g.Lz], np.float64)
        if lib.cmp_cufft_create(ctypes.byref(h), vox.ctypes.data, ext.ctypes.data, 6) != 0:
            raise RuntimeError(lib.cmp_cufft_last_error().decode())
        eps = torch.empty((6, 6) + g.shape, dtype=torch.float32, device="cuda")
        eb = np.eye(6, dtype=np.float64)
        l0 = 0.5 * (float(lm.min()) + float(lm.max()))
        m0 = 0.5 * (float(mu.min()) + float(mu.max()))
        ms = np.zeros(1, np.float32)
        crit = np.zeros(6)
        mean = np.zeros((6, 6))
        iters = int(round(plain_iters))
        torch.cuda.synchronize()
        for rep in range(2):  # the first run warms up the plans
            rc = lib.cmp_cufft_run(h, ctypes.c_void_p(lm_d.data_ptr()), ctypes.c_void_p(mu_d.data_ptr()),
                                   6, eb.ctypes.data, l0, m0, ctypes.c_void_p(eps.data_ptr()),
                                   iters if rep else 4, ms.ctypes.data, crit.ctypes.data,
                                   mean.ctypes.data)
            if rc != 0:
                raise RuntimeError(lib.cmp_cufft_last_error().decode())
        lib.cmp_cufft_destroy(h)
        ref = fixture_c_eff(0)
        out["cufft_loop"] = {
            "ms_per_iter": float(ms[0]), "instances_per_iter": 6, "iterations": iters,
            "solves_per_s_at_own_plain_iters": 6.0 / (float(ms[0]) * plain_iters / 1000.0),
            "own_speedup_per_iter": float(ms[0]) / plain_ms_per_iter,
            "last_relative_criterion": [float(c) for c in crit],
            "c_eff_rel_err_vs_fp64_oracle": (float(np.linalg.norm(mean - ref) / np.linalg.norm(ref))
                                             if ref is not None else None),
            "what": "stress kernel, cufftExecR2C batch 36, Gamma^0 + FP64 criterion kernel, "
                    "cufftExecC2R batch 36, update kernel; fixed iteration count, CUDA events",
        }
    except Exception as exc:  # reported in the line; the solver figures stand
        out["cufft_loop"] = {"error": f"{type(exc).__name__}: {exc}"}
    ref_lib = os.path.join(ROOT, "oracle", "_ref", "liblippmannschwinger.so")
    if not os.path.exists(ref_lib):
        out["reference_cuda_library"] = {"unavailable": "oracle/_ref/liblippmannschwinger.so not built"}
        return out
    try:
        rl = ctypes.CDLL(ref_lib)
        F = ctypes.POINTER(ctypes.c_float)
        rl.lippmann_schwinger_solve.argtypes = [F, F, F, F, F, ctypes.POINTER(ctypes.c_int), F,
                                                ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                                ctypes.c_int]
        rl.lippmann_schwinger_solve.restype = ctypes.c_int
        lmc = np.ascontiguousarray(lm, np.float32)
        muc = np.ascontiguousarray(mu, np.float32)
        eps_h = np.empty((6,) + g.shape, np.float32)
        sig_h = np.empty_like(eps_h)
        vox = np.array(g.shape, np.int32)
        ext = np.array([g.Lx, g.Ly, g.Lz], np.float32)
        maxiter = int(round(plain_iters)) + 40
        p = lambda a: a.ctypes.data_as(F)
        times, its, means = [], [], []
        for k in range(6):
            eb = np.zeros(6, np.float32)
            eb[k] = 1.0
            t = time.perf_counter()
            it = rl.lippmann_schwinger_solve(p(lmc), p(muc), p(eb), p(eps_h), p(sig_h),
                                             vox.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                             p(ext), 1e-6, 1e-20, maxiter, 0)
            times.append(time.perf_counter() - t)
            its.append(int(it))
            means.append(sig_h.astype(np.float64).mean(axis=(1, 2, 3)))
        ref = fixture_c_eff(0)
        c = np.array(means)
        sec = float(np.sum(times))
        out["reference_cuda_library"] = {
            "solves_per_s": 6.0 / sec,
            "ms_per_iter": 1000.0 * sec / max(1, sum(its)),
            "instances_per_iter": 1,
            "iters": its,
            "converged": [i < maxiter for i in its],
            "maxiter": maxiter,
            # per instance-iteration: the reference iterates one load case per call, this
            # solver's plain figure is per iteration of all six
            "own_speedup_per_instance_iter": 1000.0 * sec / max(1, sum(its)) / (plain_ms_per_iter / 6.0),
            "c_eff_rel_err_vs_fp64_oracle": (float(np.linalg.norm(c - ref) / np.linalg.norm(ref))
                                             if ref is not None else None),
            "what": "reference lippmann_schwinger_solve (cuFFT + SIMT kernels, per-call plans "
                    "and allocations, host buffers), one call per load case, lambda first, "
                    "rtol 1e-6; wall clock per call; its FP32 iteration may stall above 1e-6 "
                    "and then runs to maxiter",
        }
    except Exception as exc:
        out["reference_cuda_library"] = {"error": f"{type(exc).__name__}: {exc}"}
    return out


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count()
    st, g, lm, mu = workload(0)
    iters = fixture_iters(args.depth)
    if iters is None:
        print(json.dumps({"impl": "reference", "unavailable": "iteration-count fixture missing"}))
        return
    mean_iters = float(np.mean(iters))
    nv = g.number_of_voxels
    budget = max(2.0, args.cpu_sample_s / 2)
    for _ in range(args.warmup):
        cpu_sample(lm, mu, g, args.depth, 0.5, threads)
    spv = []
    its = 0
    for _ in range(args.steps):
        s, n = cpu_sample(lm, mu, g, args.depth, budget, threads)
        spv.append(s)
        its += n
    s_per_vi = float(np.mean(spv))
    vips = 1.0 / s_per_vi
    solves = vips / (nv * mean_iters)
    sample = (f"{its} iterations of one load case at {g.nx}^3 over {args.steps} steps, "
              f"scaled by the FP64 oracle's iterations per solve ({mean_iters:.1f})")
    out = {
        "impl": "reference",
        "metric": METRIC,
        "value": solves,
        "unit": "solves/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 6.0 / solves * 1000.0,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": config_dict(st, args.depth),
        "voxel_iter_per_s": vips,
        "cpu_baseline": {"value": solves, "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": solves, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "reference JAX CPU path unavailable (jax not installed); timed the NumPy/SciPy "
                "port of lippmann_schwinger_jax (oracle/ls_oracle.py) with all host threads",
    }
    print(json.dumps(out))


def own_arm(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from jaxmaterials_b200.solver import CONVERGED, Solver

    st, g, lm, mu = workload(rank)
    dev = torch.device("cuda", local)
    lm_d = torch.as_tensor(lm, device=dev)
    mu_d = torch.as_tensor(mu, device=dev)
    eye = np.eye(6, dtype=np.float32)
    s = Solver(g, batch=6, depth=args.depth)
    stream = torch.cuda.current_stream(dev)
    maxiter = 5000

    def step(lm_t, mu_t):
        return s.solve(lm_t, mu_t, eye, rtol=1e-6, atol=1e-20, maxiter=maxiter, want_sigma=False)

    clocks = ClockSampler(local).__enter__()
    for _ in range(max(args.warmup, 3)):
        r = step(lm_d, mu_d)
    converged = bool(np.all(r.status == CONVERGED))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident timing
    launches0 = s.kernel_launches()
    iters_total = 0
    c_eff = None
    barrier()
    clocks.mark("start")
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    fp64_iters = 0
    for _ in range(args.steps):
        r = step(lm_d, mu_d)
        iters_total += int(r.iters.sum())
        fp64_iters += int(s.fp64_iters().sum())
        c_eff = r.mean_sigma
    t1.record(stream)
    barrier()
    clocks.mark("end")
    clocks.__exit__(None, None, None)
    launches = s.kernel_launches() - launches0
    ms = t0.elapsed_time(t1)

    # ---- the plain Moulinec-Suquet iteration on the same structure, same timing rules
    plain = None
    if args.depth > 0 and not args.no_plain:
        sp_ = Solver(g, batch=6, depth=0)
        for _ in range(3):
            sp_.solve(lm_d, mu_d, eye, rtol=1e-6, atol=1e-20, maxiter=maxiter, want_sigma=False)
        barrier()
        p0 = torch.cuda.Event(enable_timing=True)
        p1 = torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        pits = 0
        for _ in range(args.steps):
            rp = sp_.solve(lm_d, mu_d, eye, rtol=1e-6, atol=1e-20, maxiter=maxiter, want_sigma=False)
            pits += int(rp.iters.sum())
        p1.record(stream)
        barrier()
        pms = torch.tensor([p0.elapsed_time(p1)], device=dev, dtype=torch.float64)
        if world > 1:
            dist.all_reduce(pms, op=dist.ReduceOp.MAX)
        pms = float(pms.item())
        plain = {"value": 6.0 * args.steps * world / (pms / 1000.0), "unit": "solves/s",
                 "iters_per_solve": pits / (6 * args.steps),
                 "ms_per_iteration": pms / args.steps / (pits / (6 * args.steps)),
                 "voxel_iter_per_s": pits * world * g.number_of_voxels / (pms / 1000.0),
                 "all_converged": bool(np.all(rp.status == CONVERGED))}
        plain["roofline"] = step_roofline(sp_, lm_d, mu_d, g, 6, 0, WORKLOAD)
        sp_.close()
    ms_t = torch.tensor([ms], device=dev, dtype=torch.float64)
    it_t = torch.tensor([iters_total], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
        dist.all_reduce(it_t, op=dist.ReduceOp.SUM)
    ms_max = float(ms_t.item())
    solves = 6.0 * args.steps * world / (ms_max / 1000.0)
    vips = float(it_t.item()) * g.number_of_voxels / (ms_max / 1000.0)

    # ---- end to end through the public API from pinned host buffers
    lm_h = torch.from_numpy(lm).pin_memory()
    mu_h = torch.from_numpy(mu).pin_memory()
    lm_e = torch.empty_like(lm_d)
    mu_e = torch.empty_like(mu_d)
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        lm_e.copy_(lm_h, non_blocking=True)
        mu_e.copy_(mu_h, non_blocking=True)
        r = step(lm_e, mu_e)  # returns C_eff (6x6 FP64) on the host
    e1.record(stream)
    barrier()
    ems = torch.tensor([e0.elapsed_time(e1)], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(ems, op=dist.ReduceOp.MAX)
    e2e = 6.0 * args.steps * world / (float(ems.item()) / 1000.0)

    # ---- every launch of one iteration of the timed step, for the roofline (same stream,
    # CUDA events, full workload)
    roof = step_roofline(s, lm_d, mu_d, g, 6, args.depth, WORKLOAD)
    nv = g.number_of_voxels
    fp64_share = fp64_iters / max(1, iters_total)

    s.close()
    batched = None
    if args.batched > 0:
        torch.cuda.empty_cache()
        batched = {"structures": args.batched, "depth": args.depth, "precision": "mixed",
                   "sizes": [32, 48, 64, 96, 128], "layers": [2, 6], "radius": [2.0, 5.0],
                   "volume_fraction": [0.30, 0.55], "tol": 1e-6, "seed": 1000 + rank,
                   "timing": "wall clock around the blocking call; host lambda, mu in, "
                             "C_eff out; one warm-up pass over one structure per size"}
        batched["anderson"] = batched_run(args.batched, 1000 + rank, args.depth)
        if args.batched_plain:
            batched["plain"] = batched_run(args.batched, 1000 + rank, 0)
        if world > 1:
            # whole-job figures: all ranks' solves and voxel-iterations over the slowest rank
            for key in [k for k in ("anderson", "plain") if k in batched]:
                part = batched[key]
                sec = torch.tensor([part["seconds"]], device=dev, dtype=torch.float64)
                vit = torch.tensor([part["voxel_iter_per_s"] * part["seconds"]], device=dev,
                                   dtype=torch.float64)
                dist.all_reduce(sec, op=dist.ReduceOp.MAX)
                dist.all_reduce(vit, op=dist.ReduceOp.SUM)
                part["seconds"] = float(sec.item())
                part["value"] = 6 * args.batched * world / part["seconds"]
                part["voxel_iter_per_s"] = float(vit.item()) / part["seconds"]

    generator = None
    if args.generator > 0 and world == 1:
        torch.cuda.empty_cache()
        try:
            generator = generator_run(args.generator, 5713853)
        except Exception as exc:  # reported in the line; the solver figures stand
            generator = {"error": f"{type(exc).__name__}: {exc}"}

    damage = None
    if args.damage > 0 and world == 1:
        torch.cuda.empty_cache()
        try:
            damage = damage_run(args.damage)
        except Exception as exc:  # reported in the line; the solver figures stand
            damage = {"error": f"{type(exc).__name__}: {exc}"}

    aniso = None
    if args.aniso > 0 and world == 1:
        torch.cuda.empty_cache()
        try:
            aniso = aniso_run(args.aniso)
        except Exception as exc:  # reported in the line; the solver figures stand
            aniso = {"error": f"{type(exc).__name__}: {exc}"}

    comparators = None
    if args.comparators > 0 and world == 1 and plain is not None:
        torch.cuda.empty_cache()
        try:
            comparators = comparators_run(g, lm, mu, lm_d, mu_d, plain["iters_per_solve"],
                                          plain["ms_per_iteration"])
        except Exception as exc:  # reported in the line; the solver figures stand
            comparators = {"error": f"{type(exc).__name__}: {exc}"}

    learned = None
    if args.learned > 0 and world == 1:
        torch.cuda.empty_cache()
        try:
            learned = learned_run(args.learned, 256, 64, 6, args.depth)
        except Exception as exc:  # reported in the line; the solver figures stand
            learned = {"error": f"{type(exc).__name__}: {exc}"}

    c2_256 = None
    if args.c2_256 > 0 and world == 1:
        torch.cuda.empty_cache()
        try:
            c2_256 = c2_256_run(args.c2_256)
        except Exception as exc:  # reported in the line; the solver figures stand
            c2_256 = {"error": f"{type(exc).__name__}: {exc}"}

    ref = fixture_c_eff(args.depth if args.depth in (0, 5) else 5)
    c_eff_err = (float(np.linalg.norm(c_eff - ref) / np.linalg.norm(ref))
                 if ref is not None and rank == 0 else None)

    if rank == 0:
        out = {
            "metric": METRIC,
            "value": solves,
            "unit": "solves/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic",
            "config": config_dict(st, args.depth),
            "voxel_iter_per_s": vips,
            "iters_per_solve": float(iters_total) / (6 * args.steps),
            "all_converged": converged,
            "fp64_iteration_share": fp64_share,
            "plain": plain,
            "c2_256": c2_256,
            "learned": learned,
            "comparators": comparators,
            "batched": batched,
            "generator": generator,
            "damage": damage,
            "anisotropic": aniso,
            "c_eff_diag": [float(c_eff[k, k]) for k in range(6)],
            "c_eff_rel_err_vs_fp64": c_eff_err,
            "gpu_launches": int(launches),
            "roofline": roof,
            "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": 2 * nv * 4,
                    "d2h_bytes_per_step": 36 * 8},
            "clocks": clocks.summary(),
        }
        if world == 1:
            iters = fixture_iters(args.depth)
            threads = os.cpu_count()
            s_per_vi, n = cpu_sample(lm, mu, g, args.depth, args.cpu_sample_s, threads)
            mean_it = float(np.mean(iters)) if iters else out["iters_per_solve"]
            out["cpu_baseline"] = {
                "value": 1.0 / s_per_vi / (nv * mean_it),
                "unit": "solves/s",
                "cores": threads,
                "kind": "port",
                "sample": f"{n} iterations of one load case at {g.nx}^3 (NumPy/SciPy port, FP32), "
                          f"scaled by {mean_it:.1f} iterations per solve",
                "voxel_iter_per_s": 1.0 / s_per_vi,
            }
        print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.profile_net:
        profile_net(args)
        return
    if args.profile_case:
        profile_case(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        own_arm(args)


if __name__ == "__main__":
    main()
