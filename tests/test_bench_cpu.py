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
        r = bench.cpu_baseline_sample(scheme, recon, steps=3, warm=0, n=13)
        assert r["value"] > 0 and r["steps"] == 3 and r["kind"] == "port" and r["cores"] >= 1
        assert r["spread"][0] <= r["value"] <= r["spread"][1] and "median of 3" in r["sample"]


def test_reference_arm_prints_one_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--n", "17"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["e2e"]["h2d_bytes_per_step"] == 0


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    """The timed region of a multi-GPU run is reported as the slowest rank's."""
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
    assert dict(out) == {0: 15.0, 1: 15.0}


def test_reference_arm_under_torchrun_prints_once():
    """Under torchrun with two ranks the reference arm runs on rank 0 only and
    the other rank exits 0 without output."""
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus",
           "2", "--steps", "1", "--warmup", "0", "--block-n", "17"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    assert json.loads(lines[0])["n_gpus"] == 2


def test_weno_traffic_comes_from_the_ncu_summary():
    """The roofline's traffic is the ncu DRAM figure of the committed 161^3
    summary, scaled by interior nodes to the benchmark block."""
    import bench

    t161, src = bench.weno_traffic_per_launch(161 ** 3)
    assert 6.9e8 < t161 < 7.3e8 and "161^3" in src
    t257, _ = bench.weno_traffic_per_launch(257 ** 3)
    assert abs(t257 / t161 - (257 / 161) ** 3) < 1e-12
