"""bench.py's JSON line contract: the reference arm (host cores only, so it
runs without a GPU) prints one JSON line with every required key."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _line(*args):
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], capture_output=True,
                       text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    return json.loads(lines[0])


def test_reference_arm_line_has_the_required_keys():
    d = _line("--impl", "reference", "--workload", "leaves", "--steps", "1", "--warmup", "0")
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["n_gpus"] == 1 and d["value"] > 0
    assert d["scaling"] in ("weak", "strong") and isinstance(d["higher_is_better"], bool)
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert "workload" in d["config"]


def test_unavailable_arms_say_why():
    d = _line("--impl", "reference", "--workload", "precision", "--steps", "1", "--warmup", "0")
    assert d["impl"] == "reference" and d["unavailable"]


def test_reference_arm_under_torchrun_prints_one_line():
    """Launched as an N > 1 run is (torchrun, one process per rank):
    rank 0 alone prints the line, and every rank exits 0."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
                        "--nproc-per-node", "2", "--master-addr", "127.0.0.1",
                        "--master-port", str(port), str(ROOT / "bench.py"), "--impl", "reference",
                        "--workload", "leaves", "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0


def test_plain_reference_arm_runs_full_steps_without_the_cuda_library():
    """The plain workload's reference arm at a reduced size: full iterations
    on the host cores, the same config dict as the GPU arm's, and
    libfluxion_b200.so never mapped into the process."""
    code = ("import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--gates', '20000', "
            "'--nets', '24000', '--die', '170', '--bins', '128', '--cong', '64', '--steps', '2', "
            "'--warmup', '1']; sys.path.insert(0, '.'); import bench; bench.main(); "
            "print('MAPPED', open('/proc/self/maps').read().count('libfluxion_b200'))")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert "MAPPED 0" in r.stdout
    assert d["impl"] == "reference" and d["steps"] == 2 and d["warmup"] == 1
    # every timed step is a whole iteration: steps x ms_per_step is the timed region
    lo, hi = d["step_seconds_min_max"]
    assert lo > 0 and d["ms_per_step"] / 1e3 >= lo * 0.99
    sys.path.insert(0, str(ROOT))
    import bench
    from oracle import oracle as orc
    s = orc.synth_plain(42, 20000, 24000, 170.0)
    adj = orc.build_adjacency(s.num_gates, s.net_ptr, s.net_gate)
    args = bench.parse(["--gates", "20000", "--nets", "24000", "--die", "170",
                                 "--bins", "128", "--cong", "64"])
    assert d["config"] == bench.plain_config(args, s.num_pins, len(adj[1]), 1)
