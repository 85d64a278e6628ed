"""Run a fixed number of solver iterations on a seeded fibre composite, for profiling.

    python -m jaxmaterials_b200.profile_case --n 128 --batch 2 --iters 3 [--precision fp32]
        [--depth 5]

Every pass of every iteration does its full work (tolerances 0), so the kernels seen by a
profiler are those of the timed benchmark at the same grid size.
"""

import argparse

import numpy as np


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, default=128)
    p.add_argument("--batch", type=int, default=2)
    p.add_argument("--iters", type=int, default=3)
    p.add_argument("--precision", default="fp32", choices=["fp32", "mixed", "fp64"])
    p.add_argument("--depth", type=int, default=0, help="Anderson depth")
    a = p.parse_args()
    import torch

    from jaxmaterials_b200 import GridSpec
    from jaxmaterials_b200.data import fibres
    from jaxmaterials_b200.solver import Solver

    st = fibres.generate_layered_fibres(a.n, 4, 4.0, 0.45, seed=0)
    lm, mu = fibres.lame_fields(st)
    g = GridSpec(a.n, a.n, a.n, float(a.n), float(a.n), float(a.n))
    s = Solver(g, batch=a.batch, depth=a.depth, precision=a.precision)
    eb = np.eye(6, dtype=np.float32)[: a.batch]
    r = s.solve(lm, mu, eb, rtol=0.0, atol=0.0, maxiter=a.iters, want_sigma=False)
    torch.cuda.synchronize()
    print(f"n={a.n} batch={a.batch} iters={list(r.iters)} launches={s.kernel_launches()}")
    s.close()


if __name__ == "__main__":
    main()
