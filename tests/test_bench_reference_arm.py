"""The benchmark's reference arm times the oracle's restatement of the
reference step loop on a model from the checker's numpy builder: it never
maps the engine library, and it times exactly the requested steps."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_does_not_load_the_engine_library():
    code = ("import sys; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '2', '--warmup', '3']; "
            "import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); "
            "print('ENGINE_MAPPED', 'libcrush_b200' in maps, 'ORACLE_MAPPED', 'liboracle' in maps)")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["steps"] == 2 and line["warmup"] == 3
    assert line["config"]["elements"] == 278640
    assert lines[-1] == "ENGINE_MAPPED False ORACLE_MAPPED True"
