"""The reference arm of bench.py -- the reference's own CPU path
(tutorial/CPUlp.cuh, built from source into oracle/_ref) timed on the host --
prints one JSON line of the bench contract.  It needs no GPU, so it is
checked here at a small scale."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# Runs the reference arm in this process and then lists the shared objects the
# process mapped: the reference arm must not load the engine library.
_ARM = """
import json, sys
sys.argv = ["bench.py", "--impl", "reference", "--scale", "10", "--steps", "2", "--warmup", "1"]
import bench
bench.main()
maps = open("/proc/self/maps").read()
print("ENGINE_LOADED" if "libglp_b200" in maps else "ENGINE_NOT_LOADED")
"""


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, "-c", _ARM], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    if "unavailable" in line:  # the reference binary was not built in this tree
        assert not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_cpulp"))
        return
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["value"] > 0 and line["unit"] == "GTEPS" and line["higher_is_better"] is True
    assert "ENGINE_NOT_LOADED" in r.stdout  # the graph is built by the oracle, not by libglp_b200.so
    assert line["steps"] == 2 and line["warmup"] == 0
    assert line["config"]["n"] == 1024 and line["config"]["workload"] == "rmat10-ef16-seed2-classic-20it"
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"] == {"value": line["value"], "unit": "GTEPS", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_host_rmat_csr_equals_engine_sampler_csr():
    """The oracle's host R-MAT build (used by the CPU legs of the benchmark) is
    byte-identical to the engine's sampler + CSR construction."""
    import numpy as np

    from glp_b200 import graphs
    from oracle import oracle as O

    for scale, seed in ((9, 1), (12, 2)):
        off, cols = O.rmat_csr(scale, 16, seed=seed)
        o2, c2, _ = graphs.rmat(scale, 16, seed=seed, device="cpu").numpy()
        np.testing.assert_array_equal(off, o2)
        np.testing.assert_array_equal(cols, c2)


def test_full_count_roofline_counts_only_full_steps():
    """The full-count roofline averages a tier over the steps the engine runs
    in full mode: a step follows one that changed at least majority_permille
    labels per 1000 vertices (k_step_mode).  The changed counts below are
    those of R-MAT scale 24, 20 iterations: steps 1-3 are full, step 4 (after
    49.4 % changes) is a majority step."""
    from types import SimpleNamespace

    import numpy as np

    sys.path.insert(0, ROOT)
    import bench

    n = 16777216
    changed = np.array([8871861, 8871861, 8849431, 8286877, 3338088, 54466] + [9737] * 14)
    st = np.zeros((20, 8), dtype=np.float32)
    st[1:4, 4] = 2.5   # big tier in the full steps
    st[4, 4] = 0.04    # majority step: listed vertices only
    st[1:4, 3] = 1.0
    plan = {f"v_{k}": 1 for k in ("tiny", "group16", "group32", "mid", "big", "hub")}
    plan.update({f"e_{k}": 10 for k in ("tiny", "group16", "group32", "mid", "big", "hub")})
    run = SimpleNamespace(changed=changed, step_tier_ms=st)
    roof = bench.full_count_roofline(plan, [run], n, 6450.0)
    assert roof["full_count_launches"] == 3
    assert roof["kernel"] == "k_big"
    assert abs(roof["avg_launch_ms"] - 2.5) < 1e-6
    # with the old quarter-of-n rule the majority step would have been counted
    roof25 = bench.full_count_roofline(plan, [run], n, 6450.0, majority_permille=250)
    assert roof25["full_count_launches"] == 4
