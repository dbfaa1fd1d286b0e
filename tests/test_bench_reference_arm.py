"""The benchmark's reference arm on the host cores (no GPU): `bench.py --impl
reference` times whole steps of the reference's algorithm through the oracle
(the C restatement of its kernels) on a state from the host overlap search.

It must load none of this repository's CUDA code, print one JSON line in the
benchmark's format with the repository arm's workload string, and report an
end-to-end figure that moves no bytes between host and device.
"""

from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent

PROBE = r"""
import contextlib, io, runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--n", "2000", "--steps", "1", "--warmup", "0"]
buf = io.StringIO()
with contextlib.redirect_stdout(buf):
    try:
        runpy.run_path("bench.py", run_name="__main__")
    except SystemExit as e:
        assert not e.code, e.code
line = buf.getvalue().strip().splitlines()[-1]
maps = open("/proc/self/maps").read()
print(line)
print("LIBDEM_MAPPED" if "libdem_b200" in maps else "LIBDEM_NOT_MAPPED")
"""


def test_reference_arm_runs_on_the_host_only():
    p = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    line, mapped = p.stdout.strip().splitlines()[-2:]
    assert mapped == "LIBDEM_NOT_MAPPED"
    d = json.loads(line)
    assert d["impl"] == "reference" and d["unit"] == "steps/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 1 and d["warmup"] == 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["e2e"]["value"] == d["value"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["cores"] >= 1 and cb["kind"] in ("reference", "port")
    sys.path.insert(0, str(ROOT))
    import bench

    assert d["config"]["workload"] == bench.direct_workload(2000)
