"""bench.py's host-side pieces that need no GPU: the DRAM traffic scaled from the ncu captures."""
import bench


def test_scaled_traffic_only_for_the_adna_warp_tier():
    t, how = bench.scaled_traffic(1, "adna", {"warp_counters": {"pops": 534_500_000}})
    assert abs(t - 65.5e9) < 1e6 and "scaled" in how
    for dom, wl, info in ((0, "adna", {"warp_counters": {"pops": 10}}), (1, "divergent", {"warp_counters": {"pops": 10}}),
                          (1, "adna", {}), (1, "adna", {"warp_counters": None}), (1, "adna", {"warp_counters": {}})):
        assert bench.scaled_traffic(dom, wl, info) == (None, None)


def test_scatter_traffic_per_item():
    assert abs(bench.SCATTER_DRAM_BYTES_PER_ITEM * 2e7 - 437.3e6) < 1e3


def test_both_arms_name_the_workload_alike():
    """The GPU arm and the reference arm print the same config dict for the same workload."""
    import argparse
    args = argparse.Namespace(workload="adna", scale=1.0, reads_scale=None)
    a = bench.workload_config(args, 1, 2_000_000, ["-l", "1024", "-n", "0.01", "-o", "2"])
    b = bench.workload_config(args, 1, 2_000_000, ["-l", "1024", "-n", "0.01", "-o", "2"])
    assert a == b and a["reads_per_gpu"] == 2_000_000 and a["options"] == "-l 1024 -n 0.01 -o 2"
