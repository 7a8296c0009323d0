"""The roofline accounting's per-unit figures (no GPU).

bench.py scales soltrace_b200/flops_model.py's per-unit DRAM bytes and warp instructions by
each step's units; the figures come from the ncu captures summarised in profiles/traffic.md,
and the two must not drift apart.  The flop counts per unit are sums of the listed
operation counts.
"""
import os
import re

from soltrace_b200 import flops_model as fm

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_per_unit_figures_match_the_traffic_summary():
    text = open(os.path.join(ROOT, "profiles", "traffic.md")).read()
    rows = {m.group(1): (float(m.group(2)), float(m.group(3)))
            for m in re.finditer(r"^\| (probe group|trace group) \| ([0-9.]+) \| ([0-9.]+) \|", text, re.M)}
    assert rows["probe group"] == (fm.DRAM_BYTES_PER_SUN_RAY_PROBE, fm.WARP_INSTR_PER_SUN_RAY_PROBE)
    assert rows["trace group"] == (fm.DRAM_BYTES_PER_HIT_TRACE, fm.WARP_INSTR_PER_HIT_TRACE)


def test_flop_counts_and_peaks():
    assert fm.PROBE_FLOPS_PER_SUN_RAY == 189
    assert fm.TRACE_FLOPS_PER_HIT == 501
    assert fm.TRACE_FLOPS_PER_RECEIVER_ENTRY == 177
    assert abs(fm.NOMINAL_FP64_TFLOPS - 37.22496) < 1e-9
    assert abs(fm.issue_peak_per_s(1965.0) - 148 * 4 * 1965e6) < 1.0
    assert fm.trace_flops(10, 4) == 10 * 501 + 4 * 177
