// Mixed FP32/FP64 instantiation of the trace kernels (fused multiply-add allowed).
#include "st_launch.h"
#include "st_trace_impl.cuh"

namespace stb {
// Register-budget variants (same code, different __launch_bounds__ minimum blocks per
// SM): kProbeMinBlocks in st_launch.h; the autotuner picks one.
template <int V, int FLAT>
static void resolve_one(const SceneDev &S, uint64_t s0, const ProbeOut &o, const RunState *rs, cudaStream_t st) {
    // persistent grid: every resident block of the variant on every SM
    static int per_sm = 0;
    if (per_sm == 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sun_resolve<1, kProbeMinBlocks[V], FLAT>,
                                                      kResolveBlock, 0);
        per_sm = per_sm > 0 ? per_sm : 1;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k_sun_resolve<1, kProbeMinBlocks[V], FLAT><<<sms * per_sm, kResolveBlock, 0, st>>>(S, s0, o, rs);
}
int launch_probe_mixed(const SceneDev &S, uint64_t s0, uint32_t n, const ProbeOut &o, const RunState *rs, int variant,
                       cudaStream_t st) {
    const uint32_t nb = (n + kProbeBlock - 1) / kProbeBlock;
    if (S.sun.grid_on && !S.explicit_rays && !S.sun.point_source) {
        if (S.sun.exact_flat && S.stages[0].flat_only && o.amb) {  // flat rectangles: float probe
            cudaMemsetAsync(o.cand_count, 0, sizeof(uint32_t), st);
            cudaMemsetAsync(o.amb_count, 0, sizeof(uint32_t), st);
            // the autotuner's variant: rays per thread (kExactRpt)
            if (variant == 0)
                k_sun_probe_exact<1, kExactRpt[0]><<<(n + kExactRpt[0] * kProbeBlock - 1) / (kExactRpt[0] * kProbeBlock),
                                                     kProbeBlock, 0, st>>>(S, s0, n, o, rs);
            else if (variant == 2)
                k_sun_probe_exact<1, kExactRpt[2]><<<(n + kExactRpt[2] * kProbeBlock - 1) / (kExactRpt[2] * kProbeBlock),
                                                     kProbeBlock, 0, st>>>(S, s0, n, o, rs);
            else
                k_sun_probe_exact<1, kExactRpt[1]><<<(n + kExactRpt[1] * kProbeBlock - 1) / (kExactRpt[1] * kProbeBlock),
                                                     kProbeBlock, 0, st>>>(S, s0, n, o, rs);
            int dev = 0, sms = 148;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            k_sun_resolve_amb<1><<<sms, kResolveBlock, 0, st>>>(S, s0, o);
            return 2;
        }
        launch_sun_candidates(S, s0, n, o, rs, st);
        // first stages of flat elements only (heliostat fields) take the flat-only variant
        const bool flat = S.stages[0].flat_only != 0;
        switch (variant * 2 + (flat ? 1 : 0)) {
            case 1: resolve_one<0, 1>(S, s0, o, rs, st); break;
            case 2: resolve_one<1, 0>(S, s0, o, rs, st); break;
            case 3: resolve_one<1, 1>(S, s0, o, rs, st); break;
            case 4: resolve_one<2, 0>(S, s0, o, rs, st); break;
            case 5: resolve_one<2, 1>(S, s0, o, rs, st); break;
            default: resolve_one<0, 0>(S, s0, o, rs, st);
        }
        return 2;
    }
    k_probe<1><<<nb, kProbeBlock, 0, st>>>(S, s0, n, o, rs);
    return 1;
}

int launch_trace_mixed(bool records, const SceneDev &S, const HitRec *hits, const uint32_t *total,
                      const RunState *rs, const TraceOut &O, const WfState &W, const WfQueues &Q,
                      const ReplayIn *replay, cudaStream_t st) {
    return records ? wf_launch<1, 1>(S, hits, total, rs, O, W, Q, replay, st)
                   : wf_launch<1, 0>(S, hits, total, rs, O, W, Q, replay, st);
}
// finite-element queries of this precision's kernels that found too few nodes since the
// last call (the flag is cleared)
unsigned take_fe_failures_mixed() {
    unsigned v = 0;
    if (cudaMemcpyFromSymbol(&v, g_fe_fail, sizeof v) != cudaSuccess) return 0;
    if (v) {
        const unsigned z = 0;
        cudaMemcpyToSymbol(g_fe_fail, &z, sizeof z);
    }
    return v;
}
}  // namespace stb
