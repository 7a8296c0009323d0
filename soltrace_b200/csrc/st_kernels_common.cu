// Precision-independent kernels: ordered compaction of the probe's hits.
#define ST_COMMON_KERNELS
#include <algorithm>
#include "st_launch.h"
#include "st_trace_impl.cuh"

namespace stb {
void launch_sun_candidates(const SceneDev &S, uint64_t s0, uint32_t n, uint32_t *hit_elem, uint32_t *block_counts,
                           uint32_t *cand, uint32_t *cand_count, const RunState *rs, cudaStream_t st) {
    const uint32_t nblocks = (n + kCandRays - 1) / kCandRays;
    cudaMemsetAsync(cand_count, 0, sizeof(uint32_t), st);
    k_sun_candidates<<<nblocks, kProbeBlock, 0, st>>>(S, s0, n, hit_elem, block_counts, cand, cand_count, rs);
}
void launch_offsets(const uint32_t *counts, uint32_t nb, uint32_t *offsets, uint32_t *total, cudaStream_t st) {
    k_offsets<<<1, 1024, 0, st>>>(counts, nb, offsets, total);
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
void launch_sort_by_element(const uint32_t *total, const uint64_t *hit_sid, const uint32_t *hit_el, uint32_t n_elem0,
                            uint32_t *elem_count, uint32_t *elem_cursor, uint32_t *scratch_total, uint64_t *s_sid,
                            uint32_t *s_el, uint32_t *s_idx, uint32_t max_n, cudaStream_t st) {
    cudaMemsetAsync(elem_count, 0, size_t(n_elem0) * 4, st);
    if (n_elem0 <= uint32_t(kSortBins)) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const uint32_t blocks = std::max(1u, std::min<uint32_t>((max_n + 4095) / 4096, uint32_t(2 * sms)));
        k_elem_hist_sh<<<blocks, kSortBlock, 0, st>>>(total, hit_el, n_elem0, elem_count);
        k_offsets<<<1, 1024, 0, st>>>(elem_count, n_elem0, elem_cursor, scratch_total);
        k_elem_scatter_sh<<<blocks, kSortBlock, 0, st>>>(total, hit_sid, hit_el, n_elem0, elem_cursor, s_sid, s_el,
                                                          s_idx);
        return;
    }
    const uint32_t blocks = std::max(1u, std::min<uint32_t>((max_n + 255) / 256, 148u * 8u));
    k_elem_hist<<<blocks, 256, 0, st>>>(total, hit_el, elem_count);
    k_offsets<<<1, 1024, 0, st>>>(elem_count, n_elem0, elem_cursor, scratch_total);
    k_elem_scatter<<<blocks, 256, 0, st>>>(total, hit_sid, hit_el, elem_cursor, s_sid, s_el, s_idx);
}
}  // namespace stb
