"""The command-line programs against the golden output files.

galoisgpu_b200/bin/{bfs,sssp} take the reference apps' command line
(skelapp/skel.cu:95-125, apps/bfs/support.cu, apps/sssp/support.cu) and must
write byte-identical -o output.  oracle/_ref/{bfs,sssp}_gft are the
reference's own driver (skel.cu + support.cu) linked with the drop-in
kernel.cu replacements over libgft: the link-level drop-in, held to the same
hashes.  Each program runs as a child process on the GPU."""

import hashlib
import subprocess
from pathlib import Path

import pytest

from test_golden import MANIFEST, _graph

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
CLI = ROOT / "galoisgpu_b200" / "bin"
DROPIN = ROOT / "oracle" / "_ref"

CASES = ["grid256.bfs.s0", "disconnected.bfs.s5", "road128.sssp.s0.d10000", "zero_degree_tail.sssp.s7.d10000"]
CASES += sorted(k for k, e in MANIFEST.items() if e["graph"].startswith("rmat"))[:4]
CASES += sorted(k for k, e in MANIFEST.items() if e["load_balance"])[:2]


def _run(prog: Path, key: str, tmp_path: Path, gft) -> str:
    e = MANIFEST[key]
    gr = tmp_path / f"{e['graph']}.gr"
    if not gr.exists():
        _graph(gft, e["recipe"], e["graph"]).write(gr)
    out = tmp_path / f"{key}.out"
    args = [str(prog), "-o", str(out), "-s", str(e["src"])]
    if e["app"] == "sssp":
        args += ["-d", str(e["delta"])]
    if e["load_balance"]:
        args += ["-l"]
    r = subprocess.run(args + [str(gr)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    return hashlib.sha256(out.read_bytes()).hexdigest()


@pytest.mark.parametrize("key", CASES)
def test_cli_output_matches_reference(gft, tmp_path, key):
    prog = CLI / MANIFEST[key]["app"]
    assert prog.exists(), "galoisgpu_b200/bin is built by __graft_entry__.build()"
    assert _run(prog, key, tmp_path, gft) == MANIFEST[key]["out_sha256"]


@pytest.mark.parametrize("key", CASES)
def test_reference_driver_with_dropin_kernel(gft, tmp_path, key):
    prog = DROPIN / f"{MANIFEST[key]['app']}_gft"
    if not prog.exists():
        pytest.skip("the drop-in binaries are built only where the reference sources are present")
    assert _run(prog, key, tmp_path, gft) == MANIFEST[key]["out_sha256"]


def test_cases_cover_both_apps_and_balancer_flag():
    assert {MANIFEST[k]["app"] for k in CASES} == {"bfs", "sssp"}
    assert any(MANIFEST[k]["load_balance"] for k in CASES)
