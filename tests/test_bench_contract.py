"""The benchmark's reference arm on the host: the JSON line's keys and units, and the rank rule of
a multi-process launch (rank 0 alone measures and prints)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SMALL = ["--impl", "reference", "--steps", "1", "--warmup", "0", "--width", "96", "--height", "64",
         "--instances", "2", "--subdiv", "2", "--tex", "64", "--cpu-seconds", "0.3", "--depth", "4"]


def run(args, env_extra=None):
    env = dict(os.environ)
    env.update(env_extra or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, cwd=ROOT, env=env,
                          capture_output=True, text=True, timeout=600)


def test_reference_arm_json_line():
    r = run(SMALL)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "Mrays/s" and d["higher_is_better"] is True
    assert d["value"] > 0.0 and d["steps"] == 1 and d["warmup"] == 0
    assert "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    r = run(SMALL, {"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


def test_cpu_legs_never_load_the_product_library():
    """The reference arm and the cpu_baseline leg pack their scene with the oracle's own Material::new
    and Camera::from_proj_view, so liblambent_b200.so is never mapped into that process."""
    code = (
        "import sys, types; sys.argv = ['bench.py'] + %r\n"
        "import bench\n"
        "a = bench.parse()\n"
        "bench.run_reference(a)\n"
        "bench.cpu_reference(a, 0.2)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print('PRODUCT_LOADED' if 'liblambent_b200' in maps else 'PRODUCT_ABSENT')\n"
        "print('ORACLE_LOADED' if 'liblambent_oracle' in maps else 'ORACLE_ABSENT')\n" % (SMALL,))
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "PRODUCT_ABSENT" in r.stdout and "ORACLE_LOADED" in r.stdout, r.stdout[-2000:]


def test_oracle_packer_matches_library_packer():
    """The oracle-packed scene equals the library-packed one: material records byte for byte, camera
    matrices value for value (the two inversions may differ in the sign of a zero)."""
    import numpy as np
    from lambent_b200 import scenes
    from oracle import oracle_py as O
    import ctypes as C
    a = scenes.icosphere_field(96, 64, instances=3, subdiv=1, tex_size=16, tex_layers=2)
    b = scenes.icosphere_field(96, 64, instances=3, subdiv=1, tex_size=16, tex_layers=2, packer=O.OraclePacker)
    assert [bytes(m) for m in a.materials] == [bytes(m) for m in b.materials]
    cam = lambda c: np.frombuffer(bytes(c), np.float32)
    assert np.array_equal(cam(a.camera.c), cam(b.camera.c))
    c1, c2 = scenes.cornell_box(64, 64), scenes.cornell_box(64, 64, packer=O.OraclePacker)
    assert [bytes(m) for m in c1.materials] == [bytes(m) for m in c2.materials]
    assert C.sizeof(c2.camera.c) == 128 and np.array_equal(cam(c1.camera.c), cam(c2.camera.c))
