"""bench.py's reference arm (CPU): the reference's own routine, fed by the
reference's own parser, mesh builder output and init_RNG, never loads the
product library."""
import json
import os
import subprocess
import sys

import pytest

from conftest import ROOT

PROBE = """
import runpy, sys
sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '1', '--batch', '2',
            '--ref-packets', '1200']
try:
    runpy.run_path('bench.py', run_name='__main__')
finally:
    maps = open('/proc/self/maps').read()
    print('PRODUCT_LIBRARY_LOADED' if 'liboctmps_b200' in maps else 'PRODUCT_LIBRARY_ABSENT',
          file=sys.stderr)
"""


def test_reference_arm_runs_without_the_product_library():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "bscan_ref_mesh.npz")) or \
            not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libocref_fast.so")):
        pytest.skip("reference host build or its mesh cache not built here")
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "PRODUCT_LIBRARY_ABSENT" in r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
