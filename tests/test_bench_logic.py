"""The bench's host-side arithmetic on the CPU: the algorithmic bytes behind
the roofline figure and the workload config both arms report."""

import argparse

import bench


def test_algorithmic_bytes_per_particle():
    # 256^2 slices into 256^3 at 100,000 particles: the half spectrum
    # (264,192 B), transform and CTF (64 B) and one read and write of both
    # accumulators shared among the particles (2,029 B).
    assert round(bench.bytes_per_particle(256, 256, 100_000)) == 266_285
    assert round(bench.bytes_per_particle(64, 64, 1_000)) == 20_204
    # float64 operands move twice the bytes.
    assert bench.bytes_per_particle(256, 256, 100_000, 8) == 2 * bench.bytes_per_particle(256, 256, 100_000)


def test_both_arms_report_one_config():
    args = argparse.Namespace(particles=100_000, box=256, window="linear", mode="throughput", precision="f32")
    config = bench.insertion_config(args, 1)
    assert config["workload"] == "insert_ctf_slices 100000 x 256^2 into 256^3, trilinear, throughput"
    assert config["parallelism"] == "replicas1"
    args.precision = "f64"
    assert bench.insertion_config(args, 8)["workload"].endswith(", float64")
    assert bench.insertion_config(args, 8)["parallelism"] == "replicas8"


def test_inserted_samples_per_particle():
    # The full disc of a 256^2 slice: 51,797 samples over both signs, as the
    # CPU's row and shell selection gives; the on-chip rates count 8 shared
    # atomics and 4 vector reductions each.
    assert bench.inserted_samples(256, 256) == 51_797
    rates = bench.onchip_rates(1.0e6, 51_797, 1965.0)
    assert rates["shared_atomic_lane_ops_per_s"] == 8 * 51_797 * 1.0e6
    assert abs(rates["shared_atomic_peak_nominal"] - 148 * 32 * 1965e6) < 1.0
