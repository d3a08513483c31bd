"""Host-side logic of bench.py that feeds the JSON line (no GPU).

* read_traffic: the DRAM bytes of the roofline come from a committed ncu
  summary under profiles/; the summary names the kernel sources it was
  captured from with their sha256, and a changed source voids the figure
  (the line then reports null instead of a capture of other code).
* The committed summary of the default line's kernel matches the source in
  the tree, so the default line carries a measured traffic figure.
"""
import hashlib
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def _fake_root(tmp_path, src_text, recorded_hash, traffic_lines):
    (tmp_path / "profiles").mkdir()
    src = tmp_path / "k.cu"
    src.write_text(src_text)
    lines = ["# a summary", f"kernel_source_sha256: k.cu {recorded_hash}"] + traffic_lines
    (tmp_path / "profiles" / "p.md").write_text("\n".join(lines) + "\n")
    return tmp_path


def test_read_traffic_prefers_whole_spmv_and_checks_the_source(tmp_path, monkeypatch):
    text = "__global__ void k() {}\n"
    h = hashlib.sha256(text.encode()).hexdigest()
    root = _fake_root(tmp_path, text, h, ["traffic_bytes_per_launch: 100", "traffic_bytes_per_spmv: 120"])
    monkeypatch.setattr(bench, "ROOT", root)
    assert bench.read_traffic("p") == 120.0
    assert bench.read_traffic("missing") is None
    # the kernel changed after the capture: the figure is dropped
    (root / "k.cu").write_text(text + "// changed\n")
    assert bench.read_traffic("p") is None


def test_read_traffic_without_source_record(tmp_path, monkeypatch):
    (tmp_path / "profiles").mkdir()
    (tmp_path / "profiles" / "q.md").write_text("traffic_bytes_per_launch: 42 bytes\n")
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.read_traffic("q") == 42.0


def test_default_line_profile_matches_the_tree():
    kern, prof = bench.dominant_kernel("SELL_C", 22, "rmat", staged=True)
    assert "k_sellw" in kern
    t = bench.read_traffic(prof)
    assert t is not None and 4e8 < t < 6e8, (prof, t)


def test_csr_line_names_the_kernel_that_runs():
    # the default CSR kernel takes runs of 256 entries from 2^23 entries on
    kern, prof = bench.dominant_kernel("CSR", 22, "rmat", csr_kernel=0, nnz=65_243_159)
    assert "k_spmv_chunks" in kern and prof == "spmv_csr_chunks_rmat22"
    kern, prof = bench.dominant_kernel("CSR", 18, "rmat", csr_kernel=0, nnz=3_937_938)
    assert "k_spmv_binned" in kern
    kern, _ = bench.dominant_kernel("CSR", 22, "rmat", csr_kernel=2, nnz=65_243_159)
    assert "k_spmv_binned" in kern
