"""The bench's reference arm (the CPU restatement on the host cores, on a
bounded sample) prints one JSON line with the contract's keys; runs without a
GPU (here on the 150k-edge model)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--config", "0",
                        "--steps", "1", "--warmup", "1", "--sample-steps", "4"], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["dtype"] == "f64"
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


def test_gpu_line_cpu_baseline_runs_in_a_fresh_process():
    """The cpu_baseline object of the GPU arm's line (a scaled sample of the
    reference arm, run as a subprocess): value, unit, cores, kind, sample."""
    sys.path.insert(0, ROOT)
    import bench
    cpu = bench.cpu_baseline(0, 3)
    assert cpu.get("value") and cpu["value"] > 0, cpu
    assert cpu["unit"] == "steps*RHS/s" and cpu["kind"] == "port" and cpu["cores"] >= 1
    assert "amortised" in cpu["sample"]


def test_model_batch_spans_100k_to_1m_edges():
    """The bench's 16 layered models have the uneven sizes of the multi-model
    batch they stand for (100k to 1M edges): the two coarsest hold 101 525
    and 105 367 edges, the finest 986 423."""
    sys.path.insert(0, ROOT)
    import bench
    from temf3dt_b200 import fetd
    sc = bench.layered_model_scales()
    assert len(sc) == 16 and 0.26 <= min(sc) and max(sc) <= 1.5
    order = sorted(range(16), key=lambda i: sc[i])

    def edges(i):
        return fetd.mesh_topology(bench.layered_model(i, sc[i]).mesh.tet_vex)[0].shape[0]

    assert sorted([edges(order[0]), edges(order[1])]) == [101525, 105367]
    assert edges(order[-1]) == 986423
