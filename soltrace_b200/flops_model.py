"""Algorithmic work of the trace, per unit, for roofline accounting.

Counted from the reference's arithmetic (FMA = 2 flops; sqrt, division and
transcendental calls counted separately as special operations), at one
candidate-element test per ray-stage (culling overhead is not work):

  transform of a ray into a frame (position and direction, 3x3)    33
  sun-ray generation (two affine maps and two transforms)          72
  flat-element test (start plane, aperture, acceptance)            84
  cylinder / quadric closed form with normal                      110
  hit bookkeeping (record transform)                               33
  table sunshape sample (inverse CDF) + perturbation frame         50
  slope-error sample + perturbation frame                         100
  reflection                                                       17
  back-transforms element -> stage -> global                       66
  absorption test                                                   1

Bytes: the probe marks every sun ray in a hit mask (one bit, written and read back
for the ray numbers); every first-stage hit moves 16 bytes (sun index, element, ray
rank) into the sorted hit list and the trace kernel reads them back.  Scene tables
are L2-resident.
"""

GEN, XFORM, FLAT, QUAD, BOOK, SUNSHAPE, SLOPE, REFLECT, BACK, ABSORB = 72, 33, 84, 110, 33, 50, 100, 17, 66, 1

# first-stage probe of one sun ray: generate, transform to the heliostat, one flat test
PROBE_FLOPS_PER_SUN_RAY = GEN + XFORM + FLAT
# a numbered ray in the first stage: re-test of its element, bookkeeping, absorption,
# sunshape, slope error, reflection, back-transforms, one blocking re-test
TRACE_FLOPS_PER_HIT = XFORM + FLAT + BOOK + ABSORB + SUNSHAPE + SLOPE + REFLECT + BACK + XFORM + FLAT
# a ray entering the receiver stage: transform, cylinder test, bookkeeping, absorption
TRACE_FLOPS_PER_RECEIVER_ENTRY = XFORM + QUAD + BOOK + ABSORB

PROBE_BYTES_PER_SUN_RAY = 0.25
HIT_LIST_BYTES_PER_HIT = 16 + 16

# Nominal vector peaks of a B200 (148 SMs at 1965 MHz; 64 FP64 and 128 FP32 lanes
# per SM, 2 flops per FMA).  The pool's measured peaks cover HBM copy bandwidth and
# bf16 GEMM only.
NOMINAL_FP64_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12
NOMINAL_FP32_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


# DRAM bytes (read + written) and warp instructions issued per unit, measured: ncu --set full
# captures of the main-batch launches of the headline field at 2,000 heliostats and 2e6 hits
# (`python bench.py --hits 2000000 --steps 1 --warmup 1 --no-cpu-baseline --no-extra`, mixed
# precision), dram__bytes_read.sum + dram__bytes_write.sum and smsp__inst_executed.sum summed
# over each launch group and divided by the units the launches processed (15.32 M sun rays:
# k_sun_probe_exact, k_sun_resolve_amb, k_scan_parts, k_scan_chunks, k_list_hist_sh,
# k_list_scatter_sh; 1.867 M first-stage hits: k_wf_first, k_wf_search and k_wf_shade of
# rounds 0 and 1).  The probe's lists fit in L2 at 2e6 hits, so its DRAM figure is a lower
# bound at full size; the trace figure is the wavefront's ray state, read and written at
# every kernel step.
DRAM_BYTES_PER_SUN_RAY_PROBE = 2.87
DRAM_BYTES_PER_HIT_TRACE = 365.0
WARP_INSTR_PER_SUN_RAY_PROBE = 9.44
WARP_INSTR_PER_HIT_TRACE = 125.5


def issue_peak_per_s(sm_mhz: float = 1965.0, sms: int = 148) -> float:
    """Warp instructions a B200 can issue per second: one per scheduler (four per SM) per cycle."""
    return sms * 4 * sm_mhz * 1e6


def probe_flops(sun_rays: int) -> float:
    return float(sun_rays) * PROBE_FLOPS_PER_SUN_RAY


def trace_flops(hits: int, receiver_entries: int) -> float:
    return float(hits) * TRACE_FLOPS_PER_HIT + float(receiver_entries) * TRACE_FLOPS_PER_RECEIVER_ENTRY


def probe_bytes(sun_rays: int, hits: int) -> float:
    return float(sun_rays) * PROBE_BYTES_PER_SUN_RAY + float(hits) * 16


def trace_bytes(hits: int) -> float:
    return float(hits) * 16
