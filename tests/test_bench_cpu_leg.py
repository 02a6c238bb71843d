"""The bench's CPU legs (``cpu_baseline`` and the ``--impl reference`` arm): the oracle on the
host threads over a bounded sample of the seeded ensemble, with the step count taken from the
time budget when the whole sample fits it."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpu_baseline_whole_sample_takes_budgeted_steps(orc):
    import bench
    from summationbyparts_b200 import workloads

    insts = workloads.ensemble_instances(4, seed=1)
    v, d = bench.cpu_baseline(insts, 0.5, 2)
    assert d["instances"] == len(insts)
    assert d["points"] == sum(i.side ** 2 for i in insts)
    assert d["steps"] >= 1 and d["seconds"] > 0
    assert v == pytest.approx(d["points"] * d["steps"] / d["seconds"])
    # the systems stay built: a second call advances the same oracle systems further
    built = len(bench._CPU_SYSTEMS)
    bench.cpu_baseline(insts, 0.2, 2)
    assert len(bench._CPU_SYSTEMS) == built


def test_cpu_baseline_subset_is_one_step(orc):
    import bench
    from summationbyparts_b200 import workloads

    insts = workloads.ensemble_instances(64, seed=1)
    _, d = bench.cpu_baseline(insts, 1e-4, 1)  # far less than one step of the ensemble
    assert 1 <= d["instances"] < len(insts)
    assert d["steps"] == 1


def test_reference_arm_line(orc):
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1",
                          "--ninst", "4"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] == 2
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
