"""The committed ncu summaries that bench.py reads (CPU only).

bench.py reports `roofline.traffic` from the `dram_bytes_per_launch` line of
the summary under profiles/ that covers each workload's dominant kernel (and,
for a capture of a smaller case, scales it by `sites_per_launch`).  These
checks keep the summaries and the bench in step: every summary the bench
names exists and carries a plausible figure (DRAM bytes between 0.5x and 2x
the kernel's algorithmic bytes per launch).
"""
import os
import re

import pytest

import bench

PROFILES = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "profiles")

# summary -> (sites per launch of the captured case, algorithmic bytes per site-step)
CAPTURES = {
    "step_kernel_gpe_imag_2048.md": (2048 * 2048, 40),
    "step_kernel_gpe_imag_2048_fp32.md": (2048 * 2048, 20),
    "step_kernel_rotating_frame_4096.md": (4112 * 4112, 48),
    "step_kernel_rotating_frame_4096_fp32.md": (4112 * 4112, 24),
    "step_kernel_two_component_2048.md": (2048 * 2048, 64),
    "step_kernel_cylindrical_2048.md": (2049 * 2048, 40),
    "step_kernel_moving_trap_2048.md": (2048 * 2048, 40),
    "batch_step_batch512.md": (None, 48),
}


@pytest.mark.parametrize("summary", sorted(CAPTURES))
def test_summary_carries_traffic(summary):
    t = bench.committed_traffic(summary)
    assert t is not None, summary
    sites, per_site = CAPTURES[summary]
    if sites is None:
        with open(os.path.join(PROFILES, summary)) as f:
            sites = int(re.search(r"^sites_per_launch:\s*(\d+)", f.read(), re.M).group(1))
    algorithmic = sites * per_site
    assert 0.5 * algorithmic <= t <= 2.0 * algorithmic, (summary, t, algorithmic)


def test_bench_names_only_existing_summaries():
    with open(bench.__file__) as f:
        src = f.read()
    named = set(re.findall(r'"([a-z0-9_]+\.md)"', src))
    assert named, "bench.py names no summary"
    for name in named:
        assert os.path.exists(os.path.join(PROFILES, name)), name


def test_traffic_scaled_by_sites():
    t = bench.committed_traffic("batch_step_batch512.md")
    scaled = bench.committed_traffic_per_site("batch_step_batch512.md", 2 * 11067392)
    assert scaled == 2 * t
    assert bench.committed_traffic_per_site("step_kernel_gpe_imag_2048.md", 10) is None
