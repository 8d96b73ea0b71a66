"""The benchmark's reference arm (bench.py --impl reference) is the CPU decoder of the path on
the host cores: it builds its inputs with the format library (libcodag_fmt.so) and decodes with
the oracle, so the CUDA library (libcodag_b200.so) is never mapped into that process."""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_maps_no_cuda_library():
    code = ("import runpy, sys; "
            "sys.argv = ['bench.py', '--impl', 'reference', '--n-files', '120', '--steps', '1', '--warmup', '3']; "
            "runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('MAPS', 'libcodag_b200.so' in maps, 'libcodag_fmt.so' in maps)")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(next(x for x in r.stdout.splitlines() if x.startswith("{")))
    assert line["impl"] == "reference" and line["bit_exact"]
    assert line["config"]["workload"].startswith("batched")
    assert "MAPS False True" in r.stdout
