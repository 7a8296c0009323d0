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
// chunk scans from the scanned chunk sums (k_scan_chunks with the sum of the chunks before
// each read instead of added up)
__global__ void __launch_bounds__(kScanBlock) k_scan_apply(const uint32_t *counts, uint32_t nb,
                                                           const uint32_t *part_off, uint32_t *offsets) {
    constexpr int kPer = kScanChunk / kScanBlock;
    __shared__ uint32_t wsum[kScanBlock / 32];
    const uint32_t i0 = blockIdx.x * kScanChunk + threadIdx.x * kPer;
    uint32_t v[kPer], sum = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        v[k] = (i0 + k < nb) ? counts[i0 + k] : 0u;
        sum += v[k];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    uint32_t run = part_off[blockIdx.x] + x - sum;
    for (int k = 0; k < w; ++k) run += wsum[k];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        if (i0 + k < nb) offsets[i0 + k] = run;
        run += v[k];
    }
}
void launch_scan_large(const uint32_t *counts, uint32_t nb, uint32_t *offsets, uint32_t *total, uint32_t *parts,
                       uint32_t *parts2, cudaStream_t st) {
    const uint32_t chunks = std::max(1u, (nb + kScanChunk - 1) / kScanChunk);
    k_scan_parts<<<chunks, kScanBlock, 0, st>>>(counts, nb, parts);
    // the chunk sums scanned in place (parts has one spare entry beyond the chunks)
    launch_scan(parts, chunks, parts, total, parts2, st);
    k_scan_apply<<<chunks, kScanBlock, 0, st>>>(counts, nb, parts, offsets);
}

__device__ __forceinline__ bool rec_key(const RecOrder &o, const RecordDev &r, int &s) {
    s = r.stage - 1;
    if (s < 0 || s >= o.nst) return false;
    if (o.drop_later && s >= 1) return false;  // raytrace.cpp:786-797
    if (s >= 1 && r.element == 0 && o.tt_drop[s] != 0 && r.raynum == o.tt_drop[s]) return false;  // 810-811
    return true;
}
__global__ void __launch_bounds__(256) k_rec_count(const RecOrder o) {
    __shared__ unsigned long long per[kMaxStages];
    if (threadIdx.x < kMaxStages) per[threadIdx.x] = 0;
    __syncthreads();
    for (unsigned long long i = blockIdx.x * 256ull + threadIdx.x; i < o.n; i += gridDim.x * 256ull) {
        const RecordDev &r = o.recs[i];
        int s;
        if (!rec_key(o, r, s)) continue;
        if (r.raynum > o.rb) {
            atomicOr(o.bad, 1u);
            continue;
        }
        atomicAdd(&o.key[size_t(s) * (o.rb + 1) + r.raynum], 1u);
        atomicAdd(&per[s], 1ull);
    }
    __syncthreads();
    if (threadIdx.x < o.nst && per[threadIdx.x]) atomicAdd(&o.stage_count[threadIdx.x], per[threadIdx.x]);
}
__global__ void __launch_bounds__(256) k_rec_scatter(const RecOrder o) {
    for (unsigned long long i = blockIdx.x * 256ull + threadIdx.x; i < o.n; i += gridDim.x * 256ull) {
        const RecordDev r = o.recs[i];
        int s;
        if (!rec_key(o, r, s) || r.raynum > o.rb) continue;
        const size_t k0 = size_t(s) * (o.rb + 1);
        // place in the stage's (ray number, hit index) order; the hit indices of a key are 0..m-1
        const uint32_t li = o.key[k0 + r.raynum] + r.seq - o.key[k0];
        int lo = o.run_seg[s], hi = o.run_seg[s + 1] - 1;  // last run starting at or before li
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (o.run_src[mid] <= li)
                lo = mid;
            else
                hi = mid - 1;
        }
        const unsigned long long d = o.run_dst[lo] + (li - o.run_src[lo]);
        if (d >= o.total) {
            atomicOr(o.bad, 2u);
            continue;
        }
        for (int q = 0; q < 3; ++q) {
            o.col_d[q * o.total + d] = r.pos[q];
            o.col_d[(3 + q) * o.total + d] = r.cos[q];
        }
        o.col_i[d] = r.element;
        o.col_i[o.total + d] = r.stage;
        o.col_i[2 * o.total + d] = int(r.raynum);
    }
}
static uint32_t rec_blocks(unsigned long long n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return uint32_t(std::max<unsigned long long>(1, std::min<unsigned long long>((n + 255) / 256, 8ull * sms)));
}
void launch_rec_count(const RecOrder &o, cudaStream_t st) { k_rec_count<<<rec_blocks(o.n), 256, 0, st>>>(o); }
void launch_rec_scatter(const RecOrder &o, cudaStream_t st) { k_rec_scatter<<<rec_blocks(o.n), 256, 0, st>>>(o); }

__global__ void __launch_bounds__(256) k_set_rotations(ElemRec *el, uint32_t n, const double *rot) {
    const uint32_t i = blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int q = 0; q < 9; ++q) el[i].R[q] = rot[size_t(i) * 9 + q];
}
void launch_set_rotations(ElemRec *el, uint32_t n, const double *rot, cudaStream_t st) {
    if (n) k_set_rotations<<<(n + 255) / 256, 256, 0, st>>>(el, n, rot);
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
                      HitRec *hits, uint32_t max_n, cudaStream_t st) {
    cudaMemsetAsync(elem_count, 0, size_t(n_elem0) * 4, st);
    if (n_elem0 <= uint32_t(kSortBins)) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const uint32_t blocks = std::max(1u, std::min<uint32_t>((max_n + 4095) / 4096, uint32_t(2 * sms)));
        k_list_hist_sh<<<blocks, kSortBlock, 0, st>>>(o.cand_count, o.cand_el, n_elem0, elem_count);
        k_offsets<<<1, 1024, 0, st>>>(elem_count, n_elem0, elem_cursor, scratch_total);
        k_list_scatter_sh<<<blocks, kSortBlock, 0, st>>>(s0, o, offsets, total, rs, n_elem0, elem_cursor, hits);
        return;
    }
    const uint32_t blocks = std::max(1u, std::min<uint32_t>((max_n + 255) / 256, 148u * 8u));
    k_list_hist<<<blocks, 256, 0, st>>>(o.cand_count, o.cand_el, elem_count);
    k_offsets<<<1, 1024, 0, st>>>(elem_count, n_elem0, elem_cursor, scratch_total);
    k_list_scatter<<<blocks, 256, 0, st>>>(s0, o, offsets, total, rs, elem_cursor, hits);
}
}  // namespace stb
