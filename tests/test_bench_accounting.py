"""Host-side checks of the benchmark's roofline accounting (no GPU).

`bench.kernel_bytes` gives the algorithmic bytes of one launch of every kernel the solver's
per-launch profile (`lsb_profile_step`) names; the roofline's `achieved` figure and the
step's fraction of the HBM peak divide those bytes by CUDA-event durations. These tests pin
the per-voxel sums of one plain and one Anderson iteration, check that every label the
solver emits has an entry, and compare the committed ncu DRAM traffic
(`profiles/ncu_traffic.json`, 128^3 x 6 instances) with the same accounting.
"""

import json
import os
import re

import pytest

import bench
from tests.conftest import ROOT

N = 128
NV = N ** 3
NM = N * N * (N // 2 + 1)
BATCH = 6  # the benchmark's six load cases of one structure (one Lame pair)

PLAIN = ["x pass", "finalize", "y pass inverse", "z pass update", "y pass forward"]
ANDERSON = ["x pass", "finalize", "y pass inverse", "z pass residual rings", "anderson gram",
            "anderson solve", "anderson combine", "z pass stress", "y pass forward"]


def per_voxel(names, batch, depth):
    return sum(bench.kernel_bytes(k, NV, NM, batch, depth) for k in names) / (batch * NV)


def test_bytes_per_voxel_iteration():
    """Plain: four spectrum round trips, strain read and write, the Lame pair once per
    structure. Anderson depth m: the residual pass writes an FP16 residual (12 B) and an
    FP32 image (24 B) per voxel, the Gram row reads m + 1 FP16 slots, the combine m + 1 FP32
    slots and writes the strain, the stress pass reads it and writes the spectrum."""
    s = 6 * 8 * NM / NV  # one pass over the half spectrum, per voxel (24.375 B at 128)
    assert per_voxel(PLAIN, BATCH, 0) == pytest.approx(8 * s + 48 + 8 / BATCH)
    assert per_voxel(PLAIN, BATCH, 0) == pytest.approx(244 + 1 / 3)
    for m in range(1, 9):
        assert per_voxel(ANDERSON, BATCH, m) == pytest.approx(8 * s + 108 + 36 * (m + 1) + 8 / BATCH)
    assert per_voxel(ANDERSON, BATCH, 5) == pytest.approx(520 + 1 / 3)


def test_every_profile_label_has_bytes():
    """Every launch label of the solver's per-launch profile has an algorithmic byte count
    (a new kernel without one would make the bench line's roofline fail)."""
    with open(os.path.join(ROOT, "jaxmaterials_b200", "csrc", "ls_solver.cu")) as f:
        labels = set(re.findall(r'mark\("([^"]+)"\)', f.read()))
    assert {"x pass", "z pass residual rings", "anderson combine"} <= labels
    for name in labels:
        assert bench.kernel_bytes(name, NV, NM, BATCH, 5) >= 0
    with pytest.raises(KeyError):
        bench.kernel_bytes("no such kernel", NV, NM, BATCH, 5)


def test_committed_traffic_matches_accounting():
    """ncu's DRAM bytes per launch of the 128^3 x 6 workload (every Anderson slot filled)
    are within 15% below and 10% above the algorithmic bytes: no kernel re-reads its data
    (below 1 where the previous kernel's output is still in the 126 MB L2)."""
    with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
        traffic = json.load(f)
    checked = 0
    for key, measured in traffic.items():
        if not key.startswith("c2_128:"):
            continue
        name = key.split(":", 1)[1]
        algorithmic = bench.kernel_bytes(name, NV, NM, BATCH, 5)
        if algorithmic == 0:
            continue
        ratio = measured / algorithmic
        assert 0.85 <= ratio <= 1.10, (name, ratio)
        checked += 1
    assert checked >= 7


def _run_reference_arm(extra_env):
    import subprocess
    import sys

    env = dict(os.environ, **extra_env)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                           "--steps", "1", "--warmup", "0", "--cpu-sample-s", "1"],
                          capture_output=True, text=True, env=env, timeout=600, cwd=ROOT)


def test_reference_arm_line():
    """`bench.py --impl reference` (the CPU port timed on a bounded sample) prints one JSON
    line with the own arm's metric, unit and direction, a cpu_baseline describing the run and
    an e2e object with no host-device copies; under torchrun only rank 0 prints."""
    r = _run_reference_arm({"RANK": "0"})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC
    assert d["unit"] == "solves/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["config"]["workload"].startswith(bench.WORKLOAD)
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert cb["unit"] == d["unit"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
    r1 = _run_reference_arm({"RANK": "1", "WORLD_SIZE": "2"})
    assert r1.returncode == 0 and not [l for l in r1.stdout.splitlines() if l.startswith("{")]
