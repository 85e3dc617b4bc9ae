"""bench.py's host-side helpers on the CPU: the roofline entry of the split
product kernel (int8 operations from its profiler range, DRAM traffic scaled
from the committed capture), the bounded CPU sample and the frequency cube."""
import json
from pathlib import Path

import numpy as np

import bench

ROOT = Path(__file__).resolve().parent.parent


def test_split_kernel_roofline_entry():
    # one launch of 10 ms carrying 2e13 int8 operations and 2 GB of algorithmic bytes
    top = {"name": "oz_gemm_tma_kernel", "launches": 4, "ms": 40.0, "flops": 8e13, "bytes": 8e9}
    r = bench.roofline_entry(top, 2, None, "ring8")
    assert r["bound"] == "int8-tensor" and r["unit"] == "TOPS"
    assert abs(r["achieved"] - 2e13 / 10e-3 / 1e12) < 1e-6
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = 2.0 * peaks["bf16_tflops"] if peaks.get("bf16_tflops") else 2.0 * 1590.0
    assert abs(r["peak"] - peak) < 1e-9 and abs(r["frac"] - r["achieved"] / peak) < 1e-12
    cap = json.loads((ROOT / "profiles" / "roofline_traffic.json").read_text())["ring8"]["oz_gemm_tma_kernel"]
    assert abs(r["traffic"] - cap["dram_bytes_per_int8_mac"] * 1e13) < 1.0
    assert abs(r["algorithmic_bytes_per_launch"] - 2e9) < 1e-3
    assert abs(r["traffic_over_algorithmic"] - r["traffic"] / 2e9) < 1e-12
    assert r["launches_per_step"] == 2.0


def test_sample_spec_and_cube():
    dims = [[10, 20, 30, 40], [3920, 4900, 3920, 4900], [100, 100, 100, 100]]
    assert bench.sample_spec("ring8", dims) == (1, 1960, 3920, 4)
    assert bench.sample_spec("a5", dims) == (1, 60, 1, 1)
    idx, z = bench.matsubara_cube(5.0, 4)
    assert idx.shape == (64, 3) and idx.min() == -2 and idx.max() == 1
    assert np.allclose(z, 1j * np.pi * (2 * idx + 1) / 5.0)
