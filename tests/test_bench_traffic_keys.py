"""bench.py's roofline.traffic comes from the committed ncu summaries: every
measured workload variant maps to a key whose per-launch DRAM traffic line
exists in profiles/ (host logic only, no device work)."""
import argparse

import pytest

import bench


def _args(config, precision="f64", mode="atomic", entries=0, n=6):
    return argparse.Namespace(config=config, precision=precision, mode=mode, entries=entries,
                              n=n)


@pytest.mark.parametrize("config,precision,n,key", [
    (1, "f64", 6, "cfg1"), (2, "f64", 6, "cfg2"), (3, "f64", 4, "cfg3"),
    (3, "f32", 4, "cfg3-f32"), (3, "split", 4, "cfg3-split"),
    (3, "f64", 6, "cfg3-n6"), (3, "f32", 6, "cfg3-f32-n6"),
    (4, "f64", 6, "cfg4"), (5, "f64", 6, "cfg5"), (6, "f64", 6, "cfg6"),
])
def test_every_workload_has_a_traffic_line(config, precision, n, key):
    args = _args(config, precision, n=n)
    assert bench.profile_key(args) == key
    traffic, src = bench.read_profile_traffic(key)
    assert traffic is not None and traffic > 0, key
    assert src.startswith("profiles")


def test_variant_keys_without_a_capture_read_as_null():
    assert bench.profile_key(_args(2, mode="segmented")) == "cfg2-segmented"
    assert bench.read_profile_traffic("cfg2-segmented") == (None, None)
    assert bench.profile_key(_args(5, entries=64)) == "cfg5-e64"
