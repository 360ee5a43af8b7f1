"""The reference arm of the benchmark (`bench.py --impl reference`) times the
reference's own integrator compiled for the host and must not map this
back end's library: checked in a fresh process on a tiny workload through
/proc/self/maps. Also: the checker's copy of the render-setting defaults
equals the library's."""
import ctypes as C
import json
import subprocess
import sys
from pathlib import Path

import pytest

import bench
import oracle
from nectarrender_b200 import capi, scenes

ROOT = Path(__file__).resolve().parents[1]

PROBE = r"""
import json, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "2", "--warmup", "1",
            "--levels", "1", "--res", "16x16", "--spp-per-step", "1"]
sys.path.insert(0, {root!r})
import bench
bench.main()
maps = open("/proc/self/maps").read()
libs = sorted({{l.split()[-1] for l in maps.splitlines() if l.endswith(".so") or ".so." in l}})
print("MAPS " + json.dumps([p for p in libs if {root!r} in p]), file=sys.stderr)
"""


def test_reference_arm_does_not_map_the_product_library():
    if not (oracle.REF_CPU_SO.exists() or oracle.ORACLE_SO.exists()):
        pytest.skip("no checker library built")
    r = subprocess.run([sys.executable, "-c", PROBE.format(root=str(ROOT))], capture_output=True,
                       text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    mapped = json.loads(next(l for l in r.stderr.splitlines() if l.startswith("MAPS "))[5:])
    assert mapped, "the checker library should be mapped"
    assert all("/oracle/" in p for p in mapped), mapped
    assert not any("libnectar_b200" in p or "_pathtracer" in p for p in mapped), mapped


def test_checker_defaults_equal_the_library_defaults():
    spec = scenes.cornell(res=8, spp=2, depth=5, seed=9)
    a = oracle.render_config(spec)
    b = capi.render_config(spec)
    for name, _ in capi.RenderConfig._fields_:
        assert getattr(a, name) == pytest.approx(getattr(b, name)), name
