// st_b200_probe_noalloc: the first-stage probe and its ordered compaction, run without
// allocating device memory, for callers that cannot call cudaMalloc -- code running
// under a framework that owns the device's memory pool, or a real-time loop in which
// device allocation (which can synchronise the device) is not allowed.
//
// Scene tables and per-call scratch live in one file-scope device array of
// kNoAllocBytes (48 MiB).  Every GPU that loads this library holds that array until
// the process exits; all calls share it and it keeps the last call's contents, so
// everything that must start at zero is cleared by each call, and calls that overlap
// on the GPU (from different host threads or on different streams) race.
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/st_b200.h"
#include "st_host.h"
#include "st_launch.h"

namespace stb {
namespace {

constexpr size_t kNoAllocBytes = size_t(48) << 20;
constexpr uint32_t kNoAllocMaxRays = uint32_t(1) << 22;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Host code cannot use g_noalloc_scratch's name as a device address: its address is
// looked up once per device with that device current.
std::mutex g_setup_mutex;
void *g_scratch_addr[256];

cudaError_t scratch_on_current_device(unsigned char **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 256) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = p;
    }
    *out = static_cast<unsigned char *>(g_scratch_addr[dev]);
    return cudaSuccess;
}

// bump placement of the tables inside the static array (256-byte aligned pieces)
struct Carve {
    unsigned char *base;
    size_t used = 0;
    bool ok = true;
    template <typename T>
    T *take(size_t count) {
        const size_t at = (used + 255) & ~size_t(255);
        const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
        if (at + bytes > kNoAllocBytes) {
            ok = false;
            return nullptr;
        }
        used = at + bytes;
        return reinterpret_cast<T *>(base + at);
    }
};

// makes the context's device current for the call and restores the caller's on return
struct DeviceScope {
    int saved = -1;
    cudaError_t enter(int device) {
        cudaError_t e = cudaGetDevice(&saved);
        if (e != cudaSuccess) {
            saved = -1;
            return e;
        }
        return saved == device ? cudaSuccess : cudaSetDevice(device);
    }
    ~DeviceScope() {
        int now = -1;
        if (saved >= 0 && cudaGetDevice(&now) == cudaSuccess && now != saved) cudaSetDevice(saved);
    }
};

template <typename T>
cudaError_t put(T *dst, const std::vector<T> &v, cudaStream_t st) {
    if (v.empty()) return cudaSuccess;
    return cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st);
}

}  // namespace
}  // namespace stb

using namespace stb;

extern "C" int st_b200_probe_noalloc(st_context_t pcxt, unsigned int seed, unsigned long long s0, unsigned int n,
                                     unsigned long long *hit_sid, unsigned int *hit_elem, unsigned int *n_hits,
                                     void *stream) {
    if (!pcxt) return -1;
    if (n_hits) *n_hits = 0;
    if (n == 0) return 1;
    if (!hit_sid || !hit_elem || !n_hits) {
        report(pcxt, "st_b200_probe_noalloc: hit_sid, hit_elem and n_hits must be given");
        return -1;
    }
    if (n > kNoAllocMaxRays) {
        report(pcxt, "st_b200_probe_noalloc: " + std::to_string(n) + " sun rays requested; at most " +
                         std::to_string(kNoAllocMaxRays) + " per call");
        return -1;
    }
    int device = 0;
    bool sun_rays = true;
    if (!context_device(pcxt, device, sun_rays)) return -1;
    if (!sun_rays) {
        report(pcxt, "st_b200_probe_noalloc: the context traces explicit rays (st_b200_explicit_rays); "
                     "the probe lists generated sun rays only");
        return -1;
    }
    HostScene hs;
    if (!prepare_scene(pcxt, hs)) return -1;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    DeviceScope scope;
    cudaError_t e = scope.enter(device);
    if (e != cudaSuccess) {
        report(pcxt, std::string("st_b200_probe_noalloc: cannot use the context's device: ") + cudaGetErrorString(e));
        return -1;
    }
    unsigned char *scratch = nullptr;
    e = scratch_on_current_device(&scratch);
    if (e != cudaSuccess) {
        report(pcxt, std::string("st_b200_probe_noalloc: no device scratch: ") + cudaGetErrorString(e));
        return -1;
    }
    // layout: scene tables the probe reads, then the batch scratch
    const uint32_t nb = (n + kProbeBlock - 1) / kProbeBlock;
    Carve cv{scratch};
    ElemRec *d_elems = cv.take<ElemRec>(hs.elems.size());
    float4 *d_sphere = cv.take<float4>(hs.elem_sphere.size());
    int2 *d_scells = cv.take<int2>(hs.stage_cells.size());
    float4 *d_gsph = cv.take<float4>(hs.grid_sphere.size());
    int *d_gel = cv.take<int>(hs.grid_elem.size());
    double *d_surf = cv.take<double>(hs.surf_data.size());
    BvhNode *d_bvh = cv.take<BvhNode>(hs.bvh.size());
    int *d_bvh_items = cv.take<int>(hs.bvh_items.size());
    int *d_cells = cv.take<int>(hs.cell_start.size());
    float4 *d_cdisc = cv.take<float4>(hs.cell_disc.size());
    float4 *d_cpar = cv.take<float4>(hs.cell_par.size());
    uint32_t *d_hit_elem = cv.take<uint32_t>(n);
    uint32_t *d_cand = cv.take<uint32_t>(size_t(n) + 1);  // probe candidate count, then list
    uint32_t *d_counts = cv.take<uint32_t>(nb);
    uint32_t *d_offsets = cv.take<uint32_t>(nb);
    uint32_t *d_total = cv.take<uint32_t>(2);
    RunState *d_rs = cv.take<RunState>(1);
    if (!cv.ok) {
        report(pcxt, "st_b200_probe_noalloc: the scene and " + std::to_string(n) +
                         " sun rays need more than the " + std::to_string(kNoAllocBytes >> 20) +
                         " MiB of static device scratch");
        return -1;
    }
    SceneDev S = hs.dev;
    S.elems = d_elems;
    S.elem_sphere = d_sphere;
    S.stage_cells = d_scells;
    S.grid_sphere = d_gsph;
    S.grid_elem = d_gel;
    S.beam_axis = nullptr;  // the probe does not search from a known element
    S.beam_range = nullptr;
    S.beam_elem = nullptr;
    S.surf_data = d_surf;
    S.bvh = d_bvh;
    S.bvh_items = d_bvh_items;
    S.sun.cell_start = d_cells;
    S.sun.cell_disc = d_cdisc;
    S.sun.cell_par = d_cpar;
    S.sun.exact_flat = 0;  // FP64 probe: the exact flat footprints are not carved out
    S.sun.inv_cdf = nullptr;
    S.optics = nullptr;
    S.tables = nullptr;
    S.seed = seed;
    S.precision = 0;
    S.explicit_rays = 0;
    S.n_flux = 0;
    RunState r0;
    memset(&r0, 0, sizeof r0);
    r0.target = ~0ull;  // no cut-off: every hit of the range is listed
    if ((e = put(d_elems, hs.elems, st)) != cudaSuccess || (e = put(d_sphere, hs.elem_sphere, st)) != cudaSuccess ||
        (e = put(d_scells, hs.stage_cells, st)) != cudaSuccess || (e = put(d_gsph, hs.grid_sphere, st)) != cudaSuccess ||
        (e = put(d_gel, hs.grid_elem, st)) != cudaSuccess ||
        (e = put(d_surf, hs.surf_data, st)) != cudaSuccess ||
        (e = put(d_bvh, hs.bvh, st)) != cudaSuccess || (e = put(d_bvh_items, hs.bvh_items, st)) != cudaSuccess ||
        (e = put(d_cells, hs.cell_start, st)) != cudaSuccess || (e = put(d_cdisc, hs.cell_disc, st)) != cudaSuccess ||
        (e = put(d_cpar, hs.cell_par, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_rs, &r0, sizeof r0, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(d_total, 0, 8, st)) != cudaSuccess) {
        report(pcxt, std::string("st_b200_probe_noalloc: ") + cudaGetErrorString(e));
        return -1;
    }
    ProbeOut po{};
    po.block_counts = d_counts;
    po.hit_elem = d_hit_elem;
    po.cand = d_cand + 1;
    po.cand_count = d_cand;
    launch_probe_fp64(S, s0, n, po, d_rs, 0, st);
    launch_offsets(d_counts, nb, d_offsets, d_total, st);
    launch_compact(s0, n, d_hit_elem, d_counts, d_offsets, reinterpret_cast<uint64_t *>(hit_sid), hit_elem, st);
    uint32_t total = 0;
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(&total, d_total, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
        report(pcxt, std::string("st_b200_probe_noalloc: ") + cudaGetErrorString(e));
        return -1;
    }
    *n_hits = total;
    return 1;
}
