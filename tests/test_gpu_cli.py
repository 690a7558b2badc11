"""The command-line programs against the golden output files.

galoisgpu_b200/bin/{bfs,sssp,cc} take the reference apps' command line
(skelapp/skel.cu:95-125, apps/{bfs,sssp,cc}/support.cu).  BFS and SSSP must
write byte-identical -o output; CC must print the reference's component
count and write the reference's partition (its labels depend on its racy
schedule; ours are canonical).  oracle/_ref/{bfs,sssp,cc}_gft are the
reference's own driver (skel.cu + support.cu) linked with the drop-in
kernel.cu replacements over libgft: the link-level drop-in, held to the same
bar.  Each program runs as a child process on the GPU."""

import hashlib
import json
import re
import subprocess
from pathlib import Path

import numpy as np
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


CC_GOLDEN = Path(__file__).resolve().parent / "golden"
CC_MANIFEST = json.loads((CC_GOLDEN / "cc_manifest.json").read_text())
CC_VALUES = np.load(CC_GOLDEN / "cc_values.npz")
CC_CASES = ["rmat12w.cc", "rmat14.cc", "disconnected.cc", "road200s7.cc", "zero_degree_tail.cc"]


def _run_cc(prog: Path, key: str, tmp_path: Path, gft, orc):
    e = CC_MANIFEST[key]
    g = _graph(gft, e["recipe"], e["graph"])
    gr = tmp_path / f"{e['graph']}.gr"
    g.write(gr)
    out = tmp_path / f"{key}.out"
    r = subprocess.run([str(prog), "-o", str(out), str(gr)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    comps = int(re.search(r"components: (\d+)", r.stdout).group(1))
    labels = np.array([int(ln.split()[1]) for ln in out.read_text().splitlines() if not ln.startswith("\t")],
                      dtype=np.int32)
    want = tmp_path / "want.out"
    orc.write_cc_output(want, g.row_start, g.edge_dst, g.edge_data, CC_VALUES[key])
    return comps, labels, out.read_bytes() == want.read_bytes()


@pytest.mark.parametrize("key", CC_CASES)
def test_cc_cli_matches_reference_partition(gft, orc, tmp_path, key):
    comps, labels, same_text = _run_cc(CLI / "cc", key, tmp_path, gft, orc)
    assert comps == CC_MANIFEST[key]["components"]
    np.testing.assert_array_equal(orc.canonical_labels(labels), CC_VALUES[key])
    assert same_text  # canonical labels: byte-identical to the oracle's text


@pytest.mark.parametrize("key", CC_CASES)
def test_reference_cc_driver_with_dropin_kernel(gft, orc, tmp_path, key):
    prog = DROPIN / "cc_gft"
    if not prog.exists():
        pytest.skip("the drop-in binaries are built only where the reference sources are present")
    comps, labels, same_text = _run_cc(prog, key, tmp_path, gft, orc)
    assert comps == CC_MANIFEST[key]["components"]
    np.testing.assert_array_equal(labels, CC_VALUES[key])
    assert same_text


@pytest.mark.parametrize("key", ["grid256.bfs.s0", "road128.sssp.s0.d10000"])
def test_cli_gz_output_and_binary_dump(gft, tmp_path, key):
    """`-o x.gz` writes the golden text gzip-compressed; `-b` dumps the same
    values in binary."""
    import gzip

    e = MANIFEST[key]
    gr = tmp_path / f"{e['graph']}.gr"
    _graph(gft, e["recipe"], e["graph"]).write(gr)
    z, b = tmp_path / "out.gz", tmp_path / "out.bin"
    args = [str(CLI / e["app"]), "-o", str(z), "-b", str(b), "-s", str(e["src"])]
    if e["app"] == "sssp":
        args += ["-d", str(e["delta"])]
    r = subprocess.run(args + [str(gr)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    text = gzip.decompress(z.read_bytes())
    assert hashlib.sha256(text).hexdigest() == e["out_sha256"]
    vals = gft.read_node_data(b)
    want = np.array([0x7FFFFFFF if ln.split()[1] == b"INF" else int(ln.split()[1]) for ln in text.splitlines()],
                    dtype=np.int32)
    np.testing.assert_array_equal(vals, want)
