"""bench.py takes a kernel's ncu counts from profiles/traffic.json only while
the kernel's source files hash to the digest stored with them."""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _tree(tmp_path, source):
    csrc = tmp_path / "p3m-standalone_b200" / "csrc"
    csrc.mkdir(parents=True)
    (csrc / "p3mg_gather_tile.cu").write_text(source)
    (tmp_path / "profiles").mkdir()
    return tmp_path


def test_counts_used_while_the_source_hashes_the_same(tmp_path, monkeypatch):
    root = _tree(tmp_path, "__global__ void gather_tile_kernel() {}\n")
    monkeypatch.setattr(bench, "ROOT", str(root))
    entry = {"bytes_per_launch": 123, "warp_instructions_per_launch": 456,
             "source_digest": bench.kernel_source_digest("gather_tile_kernel")}
    (root / "profiles" / "traffic.json").write_text(json.dumps({"gather_tile_kernel": entry}))
    assert bench.profile_counters("gather_tile_kernel")["warp_instructions_per_launch"] == 456
    assert bench.profile_traffic("gather_tile_kernel") == 123.0
    # the kernel's source changes after the capture: its counts are not used
    (root / "p3m-standalone_b200" / "csrc" / "p3mg_gather_tile.cu").write_text(
        "__global__ void gather_tile_kernel() { /* changed */ }\n")
    assert bench.profile_counters("gather_tile_kernel") == {}
    assert bench.profile_traffic("gather_tile_kernel") is None


def test_no_summary_means_no_counts(tmp_path, monkeypatch):
    root = _tree(tmp_path, "x\n")
    monkeypatch.setattr(bench, "ROOT", str(root))
    assert bench.profile_counters("gather_tile_kernel") == {}
    assert bench.profile_counters("pairs_cell_kernel") == {}
