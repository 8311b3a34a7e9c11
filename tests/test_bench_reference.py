"""The reference arm of bench.py on a small graph (CPU only): it prints one JSON line with the
keys the benchmark contract asks for, measured with the host's cores on the reference's own
engine (oracle/_ref/libwkref.so) where it was built, else on the oracle (its restatement)."""
import json
import os
import subprocess
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "refpin"))
import refengine  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line(built):
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--orgs", "20", "--light", "256", "--steps", "2", "--warmup", "1"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [x for x in out.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config"):
        assert key in d, key
    assert d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1
    assert d["higher_is_better"] is True and d["unit"] == "light queries/s"
    assert d["config"]["workload"] and d["config"]["orgs"] == 20
    cb = d["cpu_baseline"]
    want = "reference" if refengine.available() else "port"
    assert cb["kind"] == want and cb["cores"] >= 1 and cb["value"] == d["value"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_does_not_load_the_product(built):
    """The reference arm generates its graph with the generator's own library and reads the
    type instances from the oracle's store: the product library is never mapped, and the
    reference engine is, where it was built."""
    code = ("import runpy, sys; sys.argv = ['bench.py', '--impl', 'reference', '--orgs', '5', "
            "'--light', '64', '--steps', '1', '--warmup', '1']; "
            "runpy.run_path('bench.py', run_name='__main__'); "
            "maps = open('/proc/self/maps').read(); "
            "print('PRODUCT_MAPPED' if 'libwukong_b200' in maps else 'PRODUCT_NOT_MAPPED'); "
            "print('ORACLE_MAPPED' if 'liboracle' in maps else 'ORACLE_NOT_MAPPED'); "
            "print('REF_MAPPED' if 'libwkref' in maps else 'REF_NOT_MAPPED')")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600,
                         cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    assert "PRODUCT_NOT_MAPPED" in out.stdout and "ORACLE_MAPPED" in out.stdout
    assert ("REF_MAPPED" if refengine.available() else "REF_NOT_MAPPED") in out.stdout
