"""bench.py's roofline bookkeeping on CPU: which kernel and bytes a run
reports (single steps or two steps per pass), and the committed ncu traffic
summaries it reads, scaled to the workload's voxel count."""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def test_single_and_two_step_kernels():
    single = {"time_blocking": {"active": False}}
    pair = {"time_blocking": {"active": True}}
    b, steps, name, traffic = bench.stencil_roofline(single, "f32")
    assert (b, steps) == (13.0, 1) and name.startswith("k_step_tma<float>")
    assert traffic.name == "k_step_tma_dram_traffic.txt"
    b, steps, name, traffic = bench.stencil_roofline(pair, "f32")
    assert (b, steps) == (17.0, 2) and name.startswith("k_pair_tma<float>")
    assert traffic.name == "k_pair_tma_dram_traffic.txt"
    b, steps, name, _ = bench.stencil_roofline(pair, "bf16")
    assert (b, steps) == (9.0, 2) and "__nv_bfloat16" in name
    assert bench.stencil_roofline(single, "bf16")[:2] == (7.0, 1)


def test_committed_traffic_summaries():
    hall = 1024 * 768 * 512
    for f, storages in (("k_pair_tma_dram_traffic.txt", ["f32"]), ("k_step_tma_dram_traffic.txt", ["f32", "bf16"])):
        for st in storages:
            tr = bench.measured_traffic(ROOT / "profiles" / f, st, hall)
            # captured on the 512x384x256 crop and scaled to the hall
            assert tr is not None and "captured on 50331648 voxels and scaled by 8.000" in tr["source"]
            per_voxel = tr["bytes"] / hall
            # no re-reads: at or below the algorithmic bytes per voxel and launch
            want = {"k_pair_tma_dram_traffic.txt": 17.0}.get(f, 13.0 if st == "f32" else 7.0)
            assert 0.8 * want < per_voxel <= want
    # a smaller workload: scaled by the voxel count, and said so
    tr = bench.measured_traffic(ROOT / "profiles" / "k_pair_tma_dram_traffic.txt", "f32", hall // 2)
    assert "scaled by 4.000" in tr["source"]
    tr = bench.measured_traffic(ROOT / "profiles" / "k_pair_tma_dram_traffic.txt", "f32", 512 * 384 * 256)
    assert "captured on" not in tr["source"]
    assert bench.measured_traffic(ROOT / "profiles" / "k_pair_tma_dram_traffic.txt", "bf16", hall) is None
