"""The benchmark's reference arm keeps its JSON contract on a machine without a
GPU: one line with the reference CPU backend's figures, and the reference CUDA
backend reported as unavailable rather than failing."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the no-GPU behaviour")
def test_reference_arm_prints_one_json_line_without_a_gpu(reflib):
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "3"],
                       cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "A-scans/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["e2e"]["value"] == d["value"]
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert cb["single_instance"]["cores"] == 1 and cb["single_instance"]["value"] > 0
    assert "unavailable" in d["cuda_backend"]


def test_reference_arm_loads_nothing_of_the_package(reflib):
    """The reference arm times the reference alone: after a full run of it, no
    module of octproengine_b200 is imported and libope_b200.so is not mapped,
    and its `config` object is the one the product arm prints."""
    code = ("import sys, runpy\n"
            "sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '3', '--no-cuda-reference']\n"
            "try:\n    runpy.run_path('bench.py', run_name='__main__')\nexcept SystemExit:\n    pass\n"
            "maps = open('/proc/self/maps').read()\n"
            "print('PKG', any(m == 'octproengine_b200' or m.startswith('octproengine_b200.') for m in sys.modules))\n"
            "print('SO', 'libope_b200' in maps, 'libope_host' in maps)\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "PKG False" in r.stdout and "SO False False" in r.stdout, r.stdout[-500:]
    line = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][0])
    sys.path.insert(0, ROOT)
    import bench
    assert line["config"] == json.loads(json.dumps(bench.bench_config(1)))


def test_kernel_counters_file_feeds_the_roofline_fields():
    """profiles/chain_kernel_n2048_cubic_u16.json (an ncu capture of one chain
    launch) holds what the bench line's roofline.traffic and fp32_pipe quote:
    the captured A-scan count, DRAM bytes near the algorithmic 4096 B read per
    A-scan, the pipe counters and the command that made it."""
    sys.path.insert(0, ROOT)
    import bench
    c = bench.kernel_counters()
    assert c is not None and c["ascans"] > 0 and c["command"].startswith("ncu ")
    read_per_ascan = c["dram_bytes_read"] / c["ascans"]
    assert 4096 <= read_per_ascan < 4096 * 1.05
    for k in ("fma_pipe_active_pct", "issue_active_pct", "warps_active_pct", "thread_inst_per_ascan"):
        assert c[k] > 0
