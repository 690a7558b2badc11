"""bench.py --impl reference: the reference arm runs the reference's own
build on the bench's seeded graph without importing this engine's package
(the graph comes from oracle/libgrgen.so), and always prints one JSON line:
the measurement, or an `unavailable` line saying why the reference build
could not run (not built, or no usable GPU here)."""

import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_prints_one_line_without_the_engine():
    r = subprocess.run([sys.executable, "-X", "importtime", str(ROOT / "bench.py"), "--impl", "reference",
                        "--workload", "bfs-grid-256", "--steps", "3", "--warmup", "3"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, r.stdout
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert "unavailable" in line or (line["metric"] == "GTEPS per query" and line["value"] > 0)
    imported = [ln for ln in r.stderr.splitlines() if "import time:" in ln and "galoisgpu_b200" in ln]
    assert not imported, imported[:3]
