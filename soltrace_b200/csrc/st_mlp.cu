// Flux surrogate network kernels: a BF16 multilayer perceptron trained and evaluated on the
// device with the 5th-generation tensor cores (tcgen05), FP32 accumulation in tensor memory.
//
// The surrogate maps one heliostat's inputs (sun vector, field position, aim offset, slope
// error) to the flux image it puts on the receiver; the plain trace (st_sim_run with a
// per-source flux map) makes its training data and measures its error.  It has no counterpart in the
// reference, which traces every ray.
//
// One GEMM kernel does every layer's work, forward and backward:
//     C[M x N] = epilogue(A[M x K] B[N x K]^T)
// with A(m, k) = A[m lam + k lak] and B(n, k) = B[n lbn + k lbk] (bf16), so the backward
// products (dX = dZ W, dW = dZ^T X) read their operands in place through strides.  A CTA of
// 128 threads owns a 128 x BN tile of C: per 64-wide slice of K it stages the A and B tiles in
// shared memory in the K-major, unswizzled core-matrix layout the tensor cores read (8 rows x
// 16 bytes per core matrix), one elected thread issues four tcgen05.mma (K = 16 each) into the
// tile's FP32 accumulator in tensor memory and commits them to an mbarrier, and after the last
// slice the four warps read the accumulator back (tcgen05.ld, one row per thread) and apply
// the epilogue.  Split-K: gridDim.z CTAs share a tile's K range and add their partial sums
// (EPI_F32_ADD).
//
// Every wait is bounded: an mbarrier wait that runs out sets an error flag (read with
// st_b200_mlp_error) and the kernel drains and returns, freeing its tensor memory.
#include <cstdint>
#include <cstdio>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/st_b200.h"

namespace stb {
namespace mlp {

constexpr int kBM = 128;       // rows of a C tile (the tensor-core M)
constexpr int kBK = 64;        // K per shared-memory stage
constexpr int kThreads = 128;  // four warps: loaders, then one accumulator row each in the epilogue
constexpr unsigned kSpinLimit = 1u << 26;

// epilogues
enum Epi : int {
    EPI_BIAS_RELU_BF16 = 0,  // out_bf16 = bf16(max(acc + bias, 0))            (hidden layer)
    EPI_BIAS_F32 = 1,        // out_f32 = acc + bias                             (output layer)
    EPI_RELU_MASK_BF16 = 2,  // out_bf16 = bf16(acc) where aux_bf16 > 0, else 0  (dZ through ReLU)
    EPI_F32 = 3,             // out_f32 = acc                                    (dX of the input)
    EPI_F32_ADD = 4,         // out_f32 += acc (atomic; split-K partial sums)    (dW)
};

struct GemmArgs {
    const __nv_bfloat16 *A, *B;
    long long lam, lak, lbn, lbk;
    int M, N, K;
    int epi;
    void *C;
    long long ldc;
    const float *bias;
    const __nv_bfloat16 *aux;  // EPI_RELU_MASK_BF16: the layer's activations, leading dimension ldc
    int k_per_split;           // K range of one split (multiple of kBK)
    unsigned *err;             // set to 1 when a wait ran out
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor (tcgen05): K-major, no swizzle; start address, leading byte
// offset (between the two K-adjacent core matrices of one K = 16 step) and stride byte offset
// (between M/N-adjacent core matrices) in 16-byte units; version 1 (bits 46-47)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= uint64_t((addr >> 4) & 0x3FFFu);
    d |= uint64_t((lbo >> 4) & 0x3FFFu) << 16;
    d |= uint64_t((sbo >> 4) & 0x3FFFu) << 32;
    d |= uint64_t(1) << 46;
    return d;  // base offset 0, leading-offset mode 0, layout 0 (no swizzle)
}

// instruction descriptor of kind::f16: D f32 (bits 4-5 = 1), A and B bf16 (bits 7-9, 10-12 =
// 1), both K-major, N / 8 at bits 17-22, M / 16 at bits 24-28
__host__ __device__ constexpr uint32_t instr_desc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(kBM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

// wait for phase `parity` of the barrier to complete; false when the spin limit ran out
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity) {
    const uint32_t a = smem_u32(bar);
    for (unsigned it = 0; it < kSpinLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 16 consecutive 32-bit columns of this thread's tensor-memory lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 64 accumulator columns of the warp's 32 lanes in one load and one wait (the fused kernel's
// epilogue: a wait per 16 columns would serialise sixteen tensor-memory round trips per layer)
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float v[64]) {
    uint32_t r[64];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, "
        "%32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, "
        "%48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
          "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
          "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
          "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
          "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 64; ++i) v[i] = __uint_as_float(r[i]);
}

// Stage rows [r0, r0 + R) x K [k0, k0 + kBK) of an operand (element (r, k) at src[r lr + k lk],
// rows < rows_end and k < k_end valid, zero elsewhere) in shared memory as K-major core
// matrices: core matrix (row group g, K chunk c) at byte ((c R/8) + g) 128, its 8 rows 16 bytes
// apart.  One 16-byte chunk (8 K values of one row) per thread and step; with K contiguous the
// chunks of a row go to neighbouring threads, otherwise neighbouring rows do (coalesced either way).
template <int R>
__device__ __forceinline__ void load_tile(unsigned char *dst, const __nv_bfloat16 *src, long long lr, long long lk,
                                          int r0, int rows_end, int k0, int k_end) {
    constexpr int kChunks = R * (kBK / 8);
    const bool k_contig = (lk == 1);
    for (int c = threadIdx.x; c < kChunks; c += kThreads) {
        const int r = k_contig ? c / (kBK / 8) : c % R;
        const int kc = k_contig ? c % (kBK / 8) : c / R;
        const int gr = r0 + r, gk = k0 + kc * 8;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (gr < rows_end) {
            const __nv_bfloat16 *p = src + gr * lr + gk * lk;
            if (k_contig && gk + 8 <= k_end && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
                v = *reinterpret_cast<const uint4 *>(p);
            } else {
                unsigned short h[8];
#pragma unroll
                for (int e = 0; e < 8; ++e)
                    h[e] = (gk + e < k_end) ? __bfloat16_as_ushort(p[e * lk]) : (unsigned short)0;
                v = make_uint4(h[0] | (uint32_t(h[1]) << 16), h[2] | (uint32_t(h[3]) << 16),
                               h[4] | (uint32_t(h[5]) << 16), h[6] | (uint32_t(h[7]) << 16));
            }
        }
        *reinterpret_cast<uint4 *>(dst + (size_t(kc) * (R / 8) + r / 8) * 128 + (r % 8) * 16) = v;
    }
}

template <int BN>
__global__ void __launch_bounds__(kThreads, 1) k_mlp_gemm(GemmArgs g) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *sa = smem;                      // kBM x kBK bf16
    unsigned char *sb = smem + kBM * kBK * 2;      // BN x kBK bf16
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_sh;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * BN;
    const int kb = blockIdx.z * g.k_per_split;
    const int ke = min(g.K, kb + g.k_per_split);
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {  // the tile's FP32 accumulator: 128 lanes x BN columns of tensor memory
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                     "r"(uint32_t(BN)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_sh;
    constexpr uint32_t idesc = instr_desc(BN);
    unsigned phase = 0;
    bool ok = true;
    int steps = 0;
    for (int k0 = kb; k0 < ke; k0 += kBK) {
        load_tile<kBM>(sa, g.A, g.lam, g.lak, m0, g.M, k0, ke);
        load_tile<BN>(sb, g.B, g.lbn, g.lbk, n0, g.N, k0, ke);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the tensor cores read what was stored
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int j = 0; j < kBK / 16; ++j) {
                const uint64_t ad = smem_desc(smem_u32(sa) + uint32_t(j * 2 * (kBM / 8) * 128), (kBM / 8) * 128, 128);
                const uint64_t bd = smem_desc(smem_u32(sb) + uint32_t(j * 2 * (BN / 8) * 128), (BN / 8) * 128, 128);
                mma_bf16(tmem, ad, bd, idesc, (steps > 0 || j > 0) ? 1u : 0u);
            }
            mma_commit(&bar);
        }
        ok = mbar_wait(&bar, phase);
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // block-wide: the next stage overwrites the tiles the finished products read, and a wait
        // that ran out in any thread ends the loop for all of them
        if (__syncthreads_or(!ok)) {
            ok = false;
            break;
        }
        ++steps;
    }
    if (!ok) {
        if (lane == 0) atomicExch(g.err, 1u);
    } else if (steps > 0) {
        // epilogue: warp w reads accumulator lanes [32 w, 32 w + 32), thread = one row of C
        const int row = m0 + warp * 32 + lane;
        const bool row_ok = row < g.M;
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + (uint32_t(warp * 32) << 16) + uint32_t(c0), v);
            if (!row_ok) continue;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int col = n0 + c0 + i;
                if (col >= g.N) continue;
                const long long at = row * g.ldc + col;
                switch (g.epi) {
                    case EPI_BIAS_RELU_BF16:
                        static_cast<__nv_bfloat16 *>(g.C)[at] = __float2bfloat16_rn(fmaxf(v[i] + g.bias[col], 0.f));
                        break;
                    case EPI_BIAS_F32:
                        static_cast<float *>(g.C)[at] = v[i] + g.bias[col];
                        break;
                    case EPI_RELU_MASK_BF16:
                        static_cast<__nv_bfloat16 *>(g.C)[at] =
                            __bfloat162float(g.aux[at]) > 0.f ? __float2bfloat16_rn(v[i]) : __float2bfloat16_rn(0.f);
                        break;
                    case EPI_F32:
                        static_cast<float *>(g.C)[at] = v[i];
                        break;
                    default:
                        atomicAdd(static_cast<float *>(g.C) + at, v[i]);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (!ok) mbar_wait(&bar, phase ^ 1u);  // a product still in flight finishes before its memory is freed
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(uint32_t(BN)));
}

// mean-squared-error loss over rows x cols outputs against float targets: dY = bf16(2 (y - t) /
// (rows cols)); the sum of squared differences is added to *loss (double)
__global__ void k_mse(int rows, int cols, const float *y, const float *t, long long ldt, __nv_bfloat16 *dy,
                      double *loss) {
    const long long n = (long long)rows * cols;
    const float scale = 2.0f / float(n);
    double acc = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long r = i / cols, c = i % cols;
        const float d = y[i] - t[r * ldt + c];
        dy[i] = __float2bfloat16_rn(scale * d);
        acc += double(d) * double(d);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc);
}

// db[c] = sum over rows of dz[r][c] (one thread per column; rows strided by cols)
__global__ void k_colsum(int rows, int cols, const __nv_bfloat16 *dz, float *db) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.f;
    for (int r = 0; r < rows; ++r) s += __bfloat162float(dz[(long long)r * cols + c]);
    db[c] = s;
}

// Adam (Kingma & Ba 2015) on float master weights, with the bf16 copy the GEMMs read
__global__ void k_adam(long long n, float *w, const float *g, float *m, float *v, __nv_bfloat16 *wb, float lr,
                       float b1, float b2, float eps, float c1, float c2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16_rn(wi);
    }
}

__global__ void k_to_bf16(long long n, const float *x, __nv_bfloat16 *y) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16_rn(x[i]);
}

// ---------------------------------------------------------------------------------------
// Fused inference: every layer in one persistent kernel
// ---------------------------------------------------------------------------------------
// A CTA (one per SM) walks 128-row tiles.  The tile's activations X (128 x 256 bf16, the
// K-major core-matrix layout the tensor cores read) stay in shared memory from layer to
// layer; the weights stream through a ring of shared-memory stages, each one bulk copy
// (cp.async.bulk, completion counted on the stage's mbarrier) of a block that the packing
// kernel already laid out in that layout.  Roles:
//   warps 0-3 (epilogue): load the tile's inputs into X; per layer read the accumulator back
//     (warp w owns tensor-memory lanes 32w..32w+31, thread = row), add the bias, ReLU, round
//     to bf16 and write X for the next layer; on the output layer apply scale/clamp and write
//     the rows or add them into their group's sums;
//   warp 4, one thread (loader): issues the weight stages, kRing ahead of their use, across
//     layers and tiles (the next layer's weights arrive while the epilogue runs);
//   warp 5, one thread (MMA issuer): per layer waits for X, per stage for its weights, issues
//     the tcgen05.mma (128 x 256 x 16 each) and commits the stage back to the loader; the
//     accumulator's commit wakes the epilogue.
// Two accumulators (2 x 256 tensor-memory columns) alternate between units (a layer, or a
// 256-wide chunk of the output layer), so an output chunk's epilogue overlaps the next
// chunk's products.  Every wait is bounded; one that runs out sets the error flag and a shared
// abort flag that ends every role's loop, and the CTA drains its own copies and products
// before freeing tensor memory.
constexpr int kWidth = 256;                       // hidden width: the MMA N and the next layer's K
constexpr int kRing = 4;                          // weight stages in flight
constexpr int kStageBytes = kWidth * kBK * 2;     // 32 KB: a 256 x 64 weight block
constexpr int kFirstBytes = kWidth * 16 * 2;      // 8 KB: the first layer's 256 x 16 block
constexpr int kXBytes = kBM * kWidth * 2;         // 64 KB: a 128-row activation tile
constexpr int kFusedThreads = 192;
constexpr int kMaxLayers = 8;
constexpr int kMaxOut = 4096;

struct FusedArgs {
    const __nv_bfloat16 *x;
    long long ldx;
    int M, d_in, n_layers, n_out;
    const unsigned char *packed;
    const float *bias[kMaxLayers];
    float *out;
    int mode, group_rows, clamp;
    float scale;
    unsigned *err;
};

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// one bulk copy global -> this CTA's shared memory, its bytes counted on `bar`
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// bounded wait that also gives up as soon as another role raised the abort flag
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t *bar, unsigned parity, volatile int *abort) {
    const uint32_t a = smem_u32(bar);
    for (unsigned it = 0; it < kSpinLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (*abort) return false;
    }
    return false;
}

// weight stages of one tile: the first layer's block, 4 per hidden layer, 4 per output chunk
__host__ __device__ inline int stages_per_tile(int n_layers, int n_out) {
    return 1 + 4 * (n_layers - 2) + 4 * (n_out / kWidth);
}
__device__ __forceinline__ uint32_t stage_bytes(int j) { return j == 0 ? kFirstBytes : kStageBytes; }
__device__ __forceinline__ size_t stage_offset(int j) {
    return j == 0 ? 0 : size_t(kFirstBytes) + size_t(j - 1) * kStageBytes;
}

__global__ void __launch_bounds__(kFusedThreads, 1) k_mlp_fused(FusedArgs g) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *X = smem;
    unsigned char *ring = smem + kXBytes;
    __shared__ __align__(8) uint64_t full[kRing], empty[kRing], acc_full[2], acc_free[2], x_ready, drain;
    __shared__ uint32_t tmem_sh;
    __shared__ volatile int abort_flag;
    __shared__ unsigned issued_sh, consumed_sh;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int n_tiles = (g.M + kBM - 1) / kBM;
    const int L = g.n_layers, NC = g.n_out / kWidth;
    if (threadIdx.x == 0) {
        for (int i = 0; i < kRing; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&acc_full[i], 1);
            mbar_init(&acc_free[i], 128);
        }
        mbar_init(&x_ready, 128);
        mbar_init(&drain, 1);
        abort_flag = 0;
        issued_sh = consumed_sh = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {  // two 128 x 256 FP32 accumulators
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_sh)),
                     "r"(uint32_t(2 * kWidth)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_sh;
    const int S = stages_per_tile(L, g.n_out);

    if (warp == 4) {
        // ---- loader ----
        if (lane == 0) {
            unsigned q = 0;
            for (int t = blockIdx.x; t < n_tiles && !abort_flag; t += gridDim.x) {
                for (int j = 0; j < S; ++j, ++q) {
                    const int slot = q % kRing;
                    if (q >= kRing && !mbar_wait_or_abort(&empty[slot], ((q / kRing) - 1) & 1u, &abort_flag)) {
                        abort_flag = 1;
                        break;
                    }
                    mbar_expect_tx(&full[slot], stage_bytes(j));
                    bulk_load(ring + slot * kStageBytes, g.packed + stage_offset(j), stage_bytes(j), &full[slot]);
                }
            }
            issued_sh = q;
        }
    } else if (warp == 5) {
        // ---- MMA issuer ----
        if (lane == 0) {
            constexpr uint32_t idesc = instr_desc(kWidth);
            unsigned q = 0, u = 0, xr = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
                for (int l = 0; l < L && ok; ++l) {
                    if (!mbar_wait_or_abort(&x_ready, xr & 1u, &abort_flag)) {
                        ok = false;
                        break;
                    }
                    ++xr;
                    const int chunks = (l == L - 1) ? NC : 1;
                    const int nst = (l == 0) ? 1 : kWidth / kBK;
                    for (int c = 0; c < chunks && ok; ++c, ++u) {
                        const int b = u & 1;
                        if (u >= 2 && !mbar_wait_or_abort(&acc_free[b], ((u >> 1) - 1) & 1u, &abort_flag)) {
                            ok = false;
                            break;
                        }
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                        for (int s = 0; s < nst; ++s, ++q) {
                            const int slot = q % kRing;
                            if (!mbar_wait_or_abort(&full[slot], (q / kRing) & 1u, &abort_flag)) {
                                ok = false;
                                break;
                            }
                            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                            const uint32_t wb = smem_u32(ring + slot * kStageBytes);
                            const int steps = (l == 0) ? 1 : kBK / 16;
                            for (int j = 0; j < steps; ++j) {
                                // X: K chunk kc at kc * 2048 (16 row groups of 128 B); weight block: K
                                // chunk at kc * 4096 (32 row groups); a K = 16 step spans two chunks
                                const int kstep = s * (kBK / 16) + j;
                                const uint64_t ad = smem_desc(smem_u32(X) + uint32_t(kstep * 2 * 2048), 2048, 128);
                                const uint64_t bd = smem_desc(wb + uint32_t(j * 2 * 4096), 4096, 128);
                                mma_bf16(tmem + uint32_t(b * kWidth), ad, bd, idesc, (s > 0 || j > 0) ? 1u : 0u);
                            }
                            mma_commit(&empty[slot]);
                        }
                        if (ok) mma_commit(&acc_full[b]);
                    }
                }
            }
            if (!ok) abort_flag = 1;
            consumed_sh = q;
            // every product this thread issued has finished before the CTA frees its memory
            mma_commit(&drain);
            mbar_wait(&drain, 0);
        }
    } else {
        // ---- epilogue: warps 0-3, thread = row of the tile ----
        const int r = threadIdx.x;
        unsigned u = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < n_tiles && ok; t += gridDim.x) {
            const int row = t * kBM + r;
            // inputs, zero-padded to K = 16 (two core-matrix columns)
            {
                unsigned short h[16];
#pragma unroll
                for (int e = 0; e < 16; ++e)
                    h[e] = (row < g.M && e < g.d_in) ? __bfloat16_as_ushort(g.x[row * g.ldx + e]) : (unsigned short)0;
#pragma unroll
                for (int kc = 0; kc < 2; ++kc) {
                    const uint4 v = make_uint4(h[8 * kc] | (uint32_t(h[8 * kc + 1]) << 16),
                                               h[8 * kc + 2] | (uint32_t(h[8 * kc + 3]) << 16),
                                               h[8 * kc + 4] | (uint32_t(h[8 * kc + 5]) << 16),
                                               h[8 * kc + 6] | (uint32_t(h[8 * kc + 7]) << 16));
                    *reinterpret_cast<uint4 *>(X + (kc * 16 + r / 8) * 128 + (r % 8) * 16) = v;
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive(&x_ready);
            for (int l = 0; l < L && ok; ++l) {
                const int chunks = (l == L - 1) ? NC : 1;
                const float *bias = g.bias[l];
                for (int c = 0; c < chunks; ++c, ++u) {
                    const int b = u & 1;
                    // warp-uniform: the tensor-memory loads below are warp-collective
                    if (!__all_sync(0xffffffffu, mbar_wait_or_abort(&acc_full[b], (u >> 1) & 1u, &abort_flag))) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t ta = tmem + (uint32_t(warp * 32) << 16) + uint32_t(b * kWidth);
                    if (l < L - 1) {
                        for (int c64 = 0; c64 < kWidth; c64 += 64) {
                            float w64[64];
                            tmem_ld64(ta + uint32_t(c64), w64);
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                const float *v = w64 + 16 * q;
                                const int c0 = c64 + 16 * q;
                                uint32_t p[8];
#pragma unroll
                                for (int i = 0; i < 8; ++i) {
                                    const float a0 = fmaxf(v[2 * i] + __ldg(bias + c0 + 2 * i), 0.f);
                                    const float a1 = fmaxf(v[2 * i + 1] + __ldg(bias + c0 + 2 * i + 1), 0.f);
                                    p[i] = uint32_t(__bfloat16_as_ushort(__float2bfloat16_rn(a0))) |
                                           (uint32_t(__bfloat16_as_ushort(__float2bfloat16_rn(a1))) << 16);
                                }
                                const int kc = c0 / 8;
                                *reinterpret_cast<uint4 *>(X + (kc * 16 + r / 8) * 128 + (r % 8) * 16) =
                                    make_uint4(p[0], p[1], p[2], p[3]);
                                *reinterpret_cast<uint4 *>(X + ((kc + 1) * 16 + r / 8) * 128 + (r % 8) * 16) =
                                    make_uint4(p[4], p[5], p[6], p[7]);
                            }
                        }
                        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                        mbar_arrive(&acc_free[b]);
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        mbar_arrive(&x_ready);
                    } else {
                        const int n0 = c * kWidth;
                        const bool valid = row < g.M;
                        const long long grp = (long long)(valid ? row : g.M - 1) / (g.mode == 1 ? g.group_rows : 1);
                        const long long grp0 = __shfl_sync(0xffffffffu, grp, 0);
                        const bool uniform = __all_sync(0xffffffffu, grp0 == grp) && g.mode == 1;
                        for (int c64 = 0; c64 < kWidth; c64 += 64) {
                          float w64[64];
                          tmem_ld64(ta + uint32_t(c64), w64);
#pragma unroll
                          for (int q = 0; q < 4; ++q) {
                            float *v = w64 + 16 * q;
                            const int c0 = c64 + 16 * q;
#pragma unroll
                            for (int i = 0; i < 16; ++i) {
                                float y = (v[i] + __ldg(bias + n0 + c0 + i)) * g.scale;
                                if (g.clamp) y = fmaxf(y, 0.f);
                                v[i] = valid ? y : 0.f;
                            }
                            const int col = n0 + c0;
                            if (g.mode == 0) {
                                if (valid) {
                                    float4 *o = reinterpret_cast<float4 *>(g.out + (long long)row * g.n_out + col);
#pragma unroll
                                    for (int i = 0; i < 4; ++i)
                                        o[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                                }
                            } else if (uniform) {
                                // the warp's 32 rows share a group: halve the 16 columns' sums across
                                // lanes (16 shuffles), then one atomic per column
#pragma unroll
                                for (int d = 16, w = 8; d >= 2; d >>= 1, w >>= 1) {
#pragma unroll
                                    for (int i = 0; i < w; ++i) {
                                        const bool hi = (lane & d) != 0;
                                        const float send = hi ? v[i] : v[i + w];
                                        const float keep = hi ? v[i + w] : v[i];
                                        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, d);
                                    }
                                }
                                v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1);
                                const int k = ((lane & 16) ? 8 : 0) + ((lane & 8) ? 4 : 0) + ((lane & 4) ? 2 : 0) +
                                              ((lane & 2) ? 1 : 0);
                                if ((lane & 1) == 0) atomicAdd(g.out + grp * g.n_out + col + k, v[0]);
                            } else if (valid) {
#pragma unroll
                                for (int i = 0; i < 16; ++i) atomicAdd(g.out + grp * g.n_out + col + i, v[i]);
                            }
                          }
                        }
                        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                        mbar_arrive(&acc_free[b]);
                    }
                }
            }
        }
        if (!ok) abort_flag = 1;
    }
    __syncthreads();
    if (abort_flag) {
        if (threadIdx.x == 0) {
            atomicExch(g.err, 1u);
            // weight copies issued but never consumed land before their shared memory goes away
            for (unsigned q = consumed_sh; q < issued_sh; ++q) mbar_wait(&full[q % kRing], (q / kRing) & 1u);
        }
        __syncthreads();
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(uint32_t(2 * kWidth)));
}

// packed weights, in bf16 elements: the first layer's 256 x 16 block, then per hidden layer
// and per output chunk four 256 x 64 blocks (K slices 0-63, ..., 192-255), each block K-major
// core matrices: element (n, k) at byte ((k / 8) 32 + n / 8) 128 + (n % 8) 16 + (k % 8) 2
struct PackArgs {
    const __nv_bfloat16 *w[kMaxLayers];
    int dims[kMaxLayers + 1];
    int n_layers;
    long long n_elems;
    __nv_bfloat16 *out;
};

__global__ void k_mlp_pack(PackArgs a) {
    constexpr long long kFirst = kFirstBytes / 2, kBlock = kStageBytes / 2;
    const int L = a.n_layers;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < a.n_elems;
         e += (long long)gridDim.x * blockDim.x) {
        int l, n, k;
        long long off;
        if (e < kFirst) {
            l = 0;
            off = e * 2;
            n = int((off % 4096) / 128) * 8 + int((off % 128) / 16);
            k = int(off / 4096) * 8 + int((off % 16) / 2);
        } else {
            const long long blk = (e - kFirst) / kBlock;
            off = ((e - kFirst) % kBlock) * 2;
            int chunk = 0, slice;
            if (blk < 4LL * (L - 2)) {
                l = 1 + int(blk / 4);
                slice = int(blk % 4);
            } else {
                l = L - 1;
                chunk = int((blk - 4LL * (L - 2)) / 4);
                slice = int((blk - 4LL * (L - 2)) % 4);
            }
            n = chunk * kWidth + int((off % 4096) / 128) * 8 + int((off % 128) / 16);
            k = slice * kBK + int(off / 4096) * 8 + int((off % 16) / 2);
        }
        const int din = a.dims[l], dout = a.dims[l + 1];
        a.out[e] = (n < dout && k < din) ? a.w[l][(long long)n * din + k] : __float2bfloat16_rn(0.f);
    }
}

__device__ unsigned g_mlp_err = 0;

unsigned *err_flag() {
    static unsigned *addr[64] = {nullptr};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return nullptr;
    if (!addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_mlp_err) != cudaSuccess) return nullptr;
        addr[dev] = static_cast<unsigned *>(p);
    }
    return addr[dev];
}

template <int BN>
int launch_gemm(const GemmArgs &a, int splits, cudaStream_t st) {
    const size_t smem = size_t(kBM + BN) * kBK * 2;
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_mlp_gemm<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
            return -1;
        attr = true;
    }
    const dim3 grid((a.M + kBM - 1) / kBM, (a.N + BN - 1) / BN, splits);
    k_mlp_gemm<BN><<<grid, kThreads, smem, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? 1 : -1;
}

// the fused kernel's shape rules; -1 or the packed size in bf16 elements
long long packed_elems(int n_layers, const int *dims) {
    if (!dims || n_layers < 2 || n_layers > kMaxLayers) return -1;
    if (dims[0] < 1 || dims[0] > 16) return -1;
    for (int l = 1; l < n_layers; ++l)
        if (dims[l] != kWidth) return -1;
    const int n_out = dims[n_layers];
    if (n_out < kWidth || n_out > kMaxOut || n_out % kWidth) return -1;
    return kFirstBytes / 2 + (long long)(stages_per_tile(n_layers, n_out) - 1) * (kStageBytes / 2);
}

int launch_fused(const FusedArgs &a, cudaStream_t st) {
    constexpr int smem = kXBytes + kRing * kStageBytes;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return -1;
    static int sms[64] = {0};
    if (!sms[dev]) {
        if (cudaFuncSetAttribute(k_mlp_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
            return -1;
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) return -1;
        sms[dev] = n;
    }
    const int tiles = (a.M + kBM - 1) / kBM;
    k_mlp_fused<<<tiles < sms[dev] ? tiles : sms[dev], kFusedThreads, smem, st>>>(a);
    return cudaGetLastError() == cudaSuccess ? 1 : -1;
}

}  // namespace mlp
}  // namespace stb

using namespace stb::mlp;

extern "C" {

int st_b200_mlp_gemm(int m, int n, int k, const void *A, long long lam, long long lak, const void *B, long long lbn,
                     long long lbk, void *C, long long ldc, int epilogue, const float *bias, const void *aux, int splits,
                     void *stream) {
    if (m <= 0 || n <= 0 || k <= 0 || !A || !B || !C || epilogue < EPI_BIAS_RELU_BF16 || epilogue > EPI_F32_ADD)
        return -1;
    if ((epilogue == EPI_BIAS_RELU_BF16 || epilogue == EPI_BIAS_F32) && !bias) return -1;
    if (epilogue == EPI_RELU_MASK_BF16 && !aux) return -1;
    if (splits < 1 || (splits > 1 && epilogue != EPI_F32_ADD)) return -1;
    GemmArgs a;
    a.A = static_cast<const __nv_bfloat16 *>(A);
    a.B = static_cast<const __nv_bfloat16 *>(B);
    a.lam = lam;
    a.lak = lak;
    a.lbn = lbn;
    a.lbk = lbk;
    a.M = m;
    a.N = n;
    a.K = k;
    a.epi = epilogue;
    a.C = C;
    a.ldc = ldc;
    a.bias = bias;
    a.aux = static_cast<const __nv_bfloat16 *>(aux);
    const int kb = (k + kBK - 1) / kBK;
    a.k_per_split = ((kb + splits - 1) / splits) * kBK;
    a.err = err_flag();
    if (!a.err) return -1;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n >= 256) return launch_gemm<256>(a, splits, st);
    if (n <= 64) return launch_gemm<64>(a, splits, st);
    return launch_gemm<128>(a, splits, st);
}

int st_b200_mlp_mse(int rows, int cols, const float *y, const float *target, long long ldt, void *dy, double *loss,
                    void *stream) {
    if (rows <= 0 || cols <= 0 || !y || !target || !dy || !loss) return -1;
    k_mse<<<592, 256, 0, static_cast<cudaStream_t>(stream)>>>(rows, cols, y, target, ldt,
                                                              static_cast<__nv_bfloat16 *>(dy), loss);
    return cudaGetLastError() == cudaSuccess ? 1 : -1;
}

int st_b200_mlp_colsum(int rows, int cols, const void *dz, float *db, void *stream) {
    if (rows <= 0 || cols <= 0 || !dz || !db) return -1;
    k_colsum<<<(cols + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        rows, cols, static_cast<const __nv_bfloat16 *>(dz), db);
    return cudaGetLastError() == cudaSuccess ? 1 : -1;
}

int st_b200_mlp_adam(long long n, float *w, const float *g, float *m, float *v, void *w_bf16, float lr, float beta1,
                     float beta2, float eps, int step, void *stream) {
    if (n <= 0 || !w || !g || !m || !v || step < 1) return -1;
    const float c1 = 1.f - powf(beta1, float(step)), c2 = 1.f - powf(beta2, float(step));
    k_adam<<<592, 256, 0, static_cast<cudaStream_t>(stream)>>>(n, w, g, m, v, static_cast<__nv_bfloat16 *>(w_bf16), lr,
                                                               beta1, beta2, eps, c1, c2);
    return cudaGetLastError() == cudaSuccess ? 1 : -1;
}

int st_b200_mlp_to_bf16(long long n, const float *x, void *y, void *stream) {
    if (n <= 0 || !x || !y) return -1;
    k_to_bf16<<<592, 256, 0, static_cast<cudaStream_t>(stream)>>>(n, x, static_cast<__nv_bfloat16 *>(y));
    return cudaGetLastError() == cudaSuccess ? 1 : -1;
}

long long st_b200_mlp_packed_bytes(int n_layers, const int *dims) {
    const long long e = packed_elems(n_layers, dims);
    return e < 0 ? -1 : 2 * e;
}

int st_b200_mlp_pack(int n_layers, const int *dims, const void *const *w, void *packed, void *stream) {
    const long long e = packed_elems(n_layers, dims);
    if (e < 0 || !w || !packed) return -1;
    PackArgs a;
    for (int l = 0; l < n_layers; ++l) {
        if (!w[l]) return -1;
        a.w[l] = static_cast<const __nv_bfloat16 *>(w[l]);
    }
    for (int l = 0; l <= n_layers; ++l) a.dims[l] = dims[l];
    a.n_layers = n_layers;
    a.n_elems = e;
    a.out = static_cast<__nv_bfloat16 *>(packed);
    k_mlp_pack<<<592, 256, 0, static_cast<cudaStream_t>(stream)>>>(a);
    return cudaGetLastError() == cudaSuccess ? 1 : -1;
}

int st_b200_mlp_forward_fused(int n_layers, const int *dims, const void *packed, const float *const *bias, int m,
                              const void *x, long long ldx, float *out, int mode, int group_rows, float scale,
                              int clamp, void *stream) {
    if (packed_elems(n_layers, dims) < 0 || !packed || !bias || m <= 0 || !x || ldx < dims[0] || !out) return -1;
    if (mode < 0 || mode > 1 || (mode == 1 && group_rows < 1)) return -1;
    if ((reinterpret_cast<uintptr_t>(packed) & 15) || (reinterpret_cast<uintptr_t>(out) & 15)) return -1;
    FusedArgs a;
    for (int l = 0; l < n_layers; ++l) {
        if (!bias[l]) return -1;
        a.bias[l] = bias[l];
    }
    a.x = static_cast<const __nv_bfloat16 *>(x);
    a.ldx = ldx;
    a.M = m;
    a.d_in = dims[0];
    a.n_layers = n_layers;
    a.n_out = dims[n_layers];
    a.packed = static_cast<const unsigned char *>(packed);
    a.out = out;
    a.mode = mode;
    a.group_rows = mode == 1 ? group_rows : 1;
    a.clamp = clamp ? 1 : 0;
    a.scale = scale;
    a.err = err_flag();
    if (!a.err) return -1;
    return launch_fused(a, static_cast<cudaStream_t>(stream));
}

// the GEMM error flag of the current device (1: a wait ran out), cleared by the read
int st_b200_mlp_error(void) {
    unsigned *f = err_flag();
    if (!f) return -1;
    unsigned v = 0;
    if (cudaMemcpy(&v, f, sizeof v, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    if (v) {
        const unsigned z = 0;
        cudaMemcpy(f, &z, sizeof z, cudaMemcpyHostToDevice);
    }
    return int(v);
}

}  // extern "C"
