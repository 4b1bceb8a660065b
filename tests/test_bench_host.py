"""CPU checks of bench.py's host-side inputs: the committed ncu traffic
capture it reports as roofline.traffic is found, scaled by the stream
count, and agrees with its own per-level breakdown."""
import json
import os

import bench

CAPTURE = os.path.join(bench.ROOT, "profiles", "dram_traffic_bp_752x480x64_4streams.json")


def test_traffic_capture_found_and_scaled():
    cap = json.load(open(CAPTURE))
    per = cap["kernels"]["bp_sweep"]["dram_bytes_per_launch"]
    t4, src4 = bench.dram_traffic("bp_sweep", cap["streams"])
    assert t4 == per and "scaled" not in src4
    t32, src32 = bench.dram_traffic("bp_sweep", 32)
    assert abs(t32 - 8 * per) <= 8
    assert os.path.basename(CAPTURE) in src32 and "32/4" in src32
    assert bench.dram_traffic("no_such_kind", 32)[0] is None


def test_traffic_capture_matches_its_breakdown():
    """One branch (2 streams): 1 coarse launch, 10 level-1 half-sweeps (the
    first reads the parents' messages), 4 level-0 half-sweeps; two branches,
    15 launches over all 4 streams."""
    cap = json.load(open(CAPTURE))
    k = cap["kernels"]["bp_sweep"]
    b = k["per_launch_2_streams_bytes"]
    branch = (b["coarse"] + b["level1_first"] + 9 * b["level1_next"] + b["level0_first"]
              + 3 * b["level0_next"])
    assert k["launches"] == 15
    assert abs(2 * branch / 15 - k["dram_bytes_per_launch"]) <= 1
