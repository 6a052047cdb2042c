"""The bench's reference arm times the oracle without the umapcu library:
it must load neither the package nor its CUDA library (CPU only, a
subprocess on the 10k-point workload with a private kNN cache directory)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_SNIPPET = r"""
import json, os, sys
sys.argv = ["bench.py", "--impl", "reference", "--workload", "c1", "--steps", "1", "--warmup", "1"]
sys.path.insert(0, os.getcwd())
import bench
bench.main()
maps = open("/proc/self/maps").read()
print(json.dumps({"umapcu_imported": "umapcu" in sys.modules, "libumapcu_mapped": "libumapcu" in maps,
                  "liboracle_mapped": "liboracle" in maps}))
"""


def test_reference_arm_loads_no_umapcu(tmp_path):
    env = dict(os.environ, UMAPCU_KNN_CACHE=str(tmp_path), CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "-c", _SNIPPET], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    bench_line, probe = lines[0], lines[-1]
    assert bench_line["impl"] == "reference" and bench_line["value"] > 0
    assert bench_line["cpu_baseline"]["kind"] == "port"
    assert not probe["umapcu_imported"] and not probe["libumapcu_mapped"] and probe["liboracle_mapped"]
    # the same workload description as the umapcu arm prints
    sys.path.insert(0, ROOT)
    import bench
    args = type("A", (), {"workload": "c1", "optimiser": "adam"})()
    assert bench_line["config"] == bench.config_of(args, bench.WORKLOADS["c1"])
