// Precision-independent kernels: the grid probe's pre-test, scans, ordered compaction and
// counting sort of the probe's hits, the run-state update.
#define ST_COMMON_KERNELS
#include <algorithm>
#include "st_launch.h"
#include "st_trace_impl.cuh"

namespace stb {
void launch_sun_candidates(const SceneDev &S, uint64_t s0, uint32_t n, const ProbeOut &o, const RunState *rs,
                           cudaStream_t st) {
    const uint32_t nblocks = (n + kCandRays - 1) / kCandRays;
    cudaMemsetAsync(o.cand_count, 0, sizeof(uint32_t), st);
    k_sun_candidates<<<nblocks, kProbeBlock, 0, st>>>(S, s0, n, o, rs);
}
void launch_offsets(const uint32_t *counts, uint32_t nb, uint32_t *offsets, uint32_t *total, cudaStream_t st) {
    k_offsets<<<1, 1024, 0, st>>>(counts, nb, offsets, total);
}
void launch_scan(const uint32_t *counts, uint32_t nb, uint32_t *offsets, uint32_t *total, uint32_t *parts,
                 cudaStream_t st) {
    const uint32_t chunks = std::max(1u, (nb + kScanChunk - 1) / kScanChunk);
    k_scan_parts<<<chunks, kScanBlock, 0, st>>>(counts, nb, parts);
    k_scan_chunks<<<chunks, kScanBlock, 0, st>>>(counts, nb, parts, offsets, total);
}
void launch_compact(uint64_t s0, uint32_t n, const uint32_t *hit_elem, const uint32_t *counts,
                    const uint32_t *offsets, uint64_t *hit_sid, uint32_t *hit_el, cudaStream_t st) {
    const uint32_t nb = (n + kProbeBlock - 1) / kProbeBlock;
    k_compact<<<nb, kProbeBlock, 0, st>>>(s0, n, hit_elem, counts, offsets, hit_sid, hit_el);
}
void launch_advance(const uint32_t *total, const uint64_t *hit_sid, uint64_t s0, uint32_t n, RunState *rs,
                    cudaStream_t st) {
    k_advance<<<1, 1, 0, st>>>(total, hit_sid, s0, n, rs);
}
void launch_list_sort(uint64_t s0, const ProbeOut &o, const uint32_t *offsets, const uint32_t *total, RunState *rs,
                      uint32_t n_elem0, uint32_t *elem_count, uint32_t *elem_cursor, uint32_t *scratch_total,
                      uint64_t *s_sid, uint32_t *s_el, uint32_t *s_idx, uint32_t max_n, cudaStream_t st) {
    cudaMemsetAsync(elem_count, 0, size_t(n_elem0) * 4, st);
    if (n_elem0 <= uint32_t(kSortBins)) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const uint32_t blocks = std::max(1u, std::min<uint32_t>((max_n + 4095) / 4096, uint32_t(2 * sms)));
        k_list_hist_sh<<<blocks, kSortBlock, 0, st>>>(o.cand_count, o.cand_el, n_elem0, elem_count);
        k_offsets<<<1, 1024, 0, st>>>(elem_count, n_elem0, elem_cursor, scratch_total);
        k_list_scatter_sh<<<blocks, kSortBlock, 0, st>>>(s0, o, offsets, total, rs, n_elem0, elem_cursor, s_sid, s_el,
                                                          s_idx);
        return;
    }
    const uint32_t blocks = std::max(1u, std::min<uint32_t>((max_n + 255) / 256, 148u * 8u));
    k_list_hist<<<blocks, 256, 0, st>>>(o.cand_count, o.cand_el, elem_count);
    k_offsets<<<1, 1024, 0, st>>>(elem_count, n_elem0, elem_cursor, scratch_total);
    k_list_scatter<<<blocks, 256, 0, st>>>(s0, o, offsets, total, rs, elem_cursor, s_sid, s_el, s_idx);
}
}  // namespace stb
