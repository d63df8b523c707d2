"""bench.py's host-side pieces, on CPU: the traffic figures it reads from the
committed ncu summaries, the algorithmic flop count of the RK roofline, the
DSSF error measure, and the lattice override used for profiling a shape."""
import dataclasses
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from classical_mc_and_smd_for_2d_heisenberg_models_b200 import smd, workloads  # noqa: E402


def test_rk_profile_traffic_is_readable_and_scales_with_records():
    t64, src64 = bench.profile_traffic("rk_cluster_kernel_c2.md", 64)
    t128, src128 = bench.profile_traffic("rk_cluster_kernel_c2.md", 128)
    assert t64 and t64 > 0 and src64 == "profiles/rk_cluster_kernel_c2.md"
    assert t128 == 2 * t64 and "scaled to 128" in src128


def test_every_profile_with_a_traffic_line_parses():
    d = os.path.join(ROOT, "profiles")
    for name in sorted(os.listdir(d)):
        text = open(os.path.join(d, name)).read()
        if "dram_bytes_per_launch:" in text:
            t, _ = bench.profile_traffic(name)
            assert t and t > 0, name


def test_missing_profile_gives_no_traffic():
    assert bench.profile_traffic("no_such_kernel.md") == (None, None)


def test_flops_per_site_step_is_the_documented_count():
    # 42 z + 150: six field sweeps of 6 z flops, four stages, combine and
    # normalise, correction, energy sums
    assert bench.flops_per_site_step(12) == 654
    assert bench.flops_per_site_step(18) == 42 * 18 + 150


def test_rel_l2():
    a = np.array([1.0, 2.0, 2.0])
    assert bench.rel_l2(a, a) == 0.0
    assert abs(bench.rel_l2(a * 1.01, a) - 0.01) < 1e-12


def test_active_neighbours_follow_the_switched_on_shells():
    w = workloads.c2(4)
    lat = smd.build_lattice(w.settings.geom, w.settings.L)
    assert bench.z_active(w, lat) == 12                     # J1 + J2 on the triangular lattice
    w4 = workloads.c4(4)
    lat4 = smd.build_lattice(w4.settings.geom, w4.settings.L)
    assert bench.z_active(w4, lat4) == 12                   # J1 + J2 + J3 on the square lattice


def test_lattice_override_keeps_a_buildable_workload():
    """--lattice GEOM:L swaps the lattice of a workload (profiling a shape);
    the inputs it makes have the new lattice's size."""
    w = workloads.c2(8)
    w = dataclasses.replace(w, settings=dataclasses.replace(w.settings, geom="hexagn", L=48),
                            state="ferro", n_rec=64)
    assert w.settings.N == 4608 and w.settings.G == 144
    spins, imp = workloads.make_inputs(w)
    assert spins.shape == (8, 4608, 3) and imp is None
    assert np.allclose(np.linalg.norm(spins, axis=2), 1.0)
