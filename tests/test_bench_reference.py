"""The bench's reference arm (the CPU restatement of the reference's step timed on the
host cores) on a small grid: it runs without a GPU and prints the JSON line the
measurement contract asks for."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_the_contract_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--maxx", "32", "--nz", "16",
                        "--steps", "1", "--warmup", "3", "--cpu-sample-xy", "32",
                        "--ref-sample-xy", "32"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
                "vs_baseline", "dtype", "data", "config", "e2e", "cpu_baseline"):
        assert key in line, key
    assert line["impl"] == "reference"
    assert line["value"] > 0 and line["unit"] == "Mcell-updates/s" and line["higher_is_better"] is True
    assert line["warmup"] >= 3
    assert line["e2e"]["value"] == line["value"] and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] in ("port", "reference") and line["cpu_baseline"]["cores"] >= 1
    assert "workload" in line["config"]
    # the timed region is the line's own steps x ms_per_step (the sample's time per step)
    assert line["sample"]["maxx"] == 32 and line["sample"]["cells"] == 32 * 32 * 16
    assert line["sample"]["reduced_size"] is False


def test_reference_arm_never_loads_the_cuda_library():
    """The reference arm builds its domain with the oracle's init routines: after a full run in
    one process, the product library is not mapped."""
    code = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--maxx', '64', '--nz', '16', "
            "'--steps', '2', '--warmup', '3', '--ref-sample-xy', '64', '--ref-seconds', '0.001']; "
            "runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('MAPPED' if 'libmimica_gpu' in maps else 'CLEAN'); "
            "print('ORACLE' if 'libmimica_oracle_omp' in maps else 'NO-ORACLE')")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    out = r.stdout.strip().splitlines()
    assert out[-2] == "CLEAN" and out[-1] == "ORACLE"
    line = json.loads(out[-3])
    # --ref-seconds is tiny, so the sample was halved down to the 32-cell floor
    assert line["sample"]["maxx"] == 32 and line["sample"]["reduced_size"] is True
    assert abs(line["ms_per_step"] * line["value"] * 1e3 - line["sample"]["cells"]) < 1e-6 * line["sample"]["cells"]


def test_reference_arm_under_torchrun_two_ranks():
    """Launched as for N GPUs: rank 0 alone prints the line, the other rank exits 0."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
                        "--impl", "reference", "--gpus", "2", "--maxx", "32", "--nz", "16", "--steps", "1", "--warmup", "3",
                        "--cpu-sample-xy", "32", "--ref-sample-xy", "32"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.strip().splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
