"""FP64 oracle results for the benchmark microstructures (effective stiffness and
iteration counts per load case), used by the parity tests at full size and to convert
the CPU baseline's bounded per-iteration sample into solves/s.

    python tests/golden/make_bench_fixture.py [name ...]

Writes tests/golden/bench_<name>.npz for each named structure (default: c1 c2_128); the
256^3 structure (c2_256) is run with Anderson depth 5 only (an FP64 CPU run of its plain
iteration would take hours).
"""

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from jaxmaterials_b200.data import fibres  # noqa: E402
from oracle import ls_oracle as O  # noqa: E402


def run(name, seed=0, depths=(0, 5)):
    st = fibres.config_structure(name, seed=seed)
    lm, mu = fibres.lame_fields(st)
    n = st.n
    g = O.Grid(*n, *st.extents)
    out = {"n": np.array(n), "seed": np.int64(seed), "volume_fraction": st.volume_fraction}
    for depth in depths:
        t = time.time()
        c, its = O.c_eff(lm.astype(np.float64), mu.astype(np.float64), g, rtol=1e-6,
                         atol=1e-20, depth=depth, maxiter=5000, dtype=np.float64)
        out[f"ceff_d{depth}"] = c
        out[f"iters_d{depth}"] = np.array(its)
        print(name, "depth", depth, "iters", its, f"{time.time() - t:.0f}s", flush=True)
    np.savez_compressed(os.path.join(HERE, f"bench_{name}.npz"), **out)


if __name__ == "__main__":
    for name in (sys.argv[1:] or ["c1", "c2_128"]):
        run(name, depths=(5,) if name == "c2_256" else (0, 5))
