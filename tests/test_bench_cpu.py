"""The benchmark's CPU legs run on the host: the timed CPU baseline (the
oracle on a bounded sample of the workload) and the reference arm's JSON line.
Guards the host-side plumbing of bench.py that only the round-end benchmark
would otherwise exercise."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_cpu_baseline_sample_runs_for_each_scheme_family():
    import bench

    for scheme, recon in ((72, 2), (4, 2)):
        r = bench.cpu_baseline_sample(scheme, recon, target_s=0.2, n=13)
        assert r["value"] > 0 and r["steps"] >= 1 and r["kind"] == "port" and r["cores"] >= 1


def test_reference_arm_prints_one_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--n", "17"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["e2e"]["h2d_bytes_per_step"] == 0
