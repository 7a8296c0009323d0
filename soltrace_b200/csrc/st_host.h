// Host-side interface between the scene/context code (st_host.cpp, plain C++)
// and the CUDA run driver (st_run.cu).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include <vector_types.h>

#include "st_scene.h"

namespace stb {

// Flattened scene in host memory; gpu_run() uploads it once per run.
struct HostScene {
    std::vector<ElemRec> elems;
    std::vector<OpticRec> optics;
    std::vector<double> surf_data, tables;
    std::vector<BvhNode> bvh;
    std::vector<int> bvh_items;
    std::vector<int> cell_start;
    std::vector<int2> stage_cells;    // ground-grid cells ([start, end) into the grid entries)
    std::vector<float4> grid_sphere;  // ground-grid entries: element bounding sphere
    std::vector<int> grid_elem;       // ground-grid entries: element index within the stage
    std::vector<float4> beam_axis;    // per element: outgoing-beam axis and cosine limit (w > 1: none)
    std::vector<int2> beam_range;     // per element: [start, end) in beam_elem
    std::vector<int> beam_elem;       // outgoing-beam candidate lists (element index within the stage)
    std::vector<float4> elem_sphere;  // per element: origin (stage coordinates), padded bounding radius
    std::vector<float4> cell_disc;  // sun-plane grid entries: disc centre x, y, radius, element
    std::vector<float4> cell_par;   // sun-plane grid entries: footprint parallelogram (dual basis rows)
    std::vector<float4> cell_xa, cell_xb, cell_xc;  // sun-plane grid entries: exact flat footprints (SunDev)
    std::vector<double> inv_cdf;  // table-sunshape inverse CDF (kSunInvCells + 1 entries)
    SceneDev dev;  // stages, sun scalars and flags; device pointers are filled by gpu_run
};

struct FluxMapReq {
    int stage, elem, kind, nx, ny, absorbed_only;
    double x0, x1, y0, y1;
    int per_source = 0;  // one nx x ny map per first-stage element (the rays' first heliostat)
};

struct RunRequest {
    uint64_t n_hits = 0;      // rays to number (first-stage hits); explicit mode: ignored
    uint64_t max_sun = 0;     // sun-ray cap (st_sim_params maxcount)
    uint32_t seed = 0;
    int precision = 0;
    bool records = true;
    int device = 0;
    std::vector<double> ex_pos, ex_cos;  // explicit rays (global frame)
    std::vector<FluxMapReq> flux;
    int (*callback)(unsigned long, unsigned long, unsigned long, unsigned long, unsigned long, void *) = nullptr;
    void *cbdata = nullptr;
    double hit_rate_hint = 0.0;  // expected first-stage hits per sun ray (0 = measure with a pilot batch)
    bool save_stage_data = false;       // keep the rays leaving stages 1 and 2 (RunResult::saved)
    bool replay = false;                // rays enter stage 2 from replay_rows instead of the sun
    std::vector<double> replay_rows;    // 7 doubles per ray: global position, direction, ray number
    std::vector<int> replay_fe0;        // per ray: global index of its first first-stage element, -1
    uint64_t replay_sun_rays = 0;       // SunRayCount of a replay (the last saved stage-1 ray number)
    std::vector<RecordDev> pre_records; // replay: the saved stage-1 records, ordered with the traced ones
    // one rank of a run split over several GPUs (st_b200_set_ranks): this rank traces its
    // contiguous slice of every batch's sun-ray range and exchanges through the callbacks
    int rank = 0, nranks = 1;
    int (*allgather)(const unsigned long long *send, unsigned long long *recv, int count, void *user) = nullptr;
    int (*allreduce)(unsigned long long *buf, unsigned long long count, int op, void *user) = nullptr;
    void *comm_user = nullptr;
};

// The records of a run in the reference's readback order (TRayData::Merge), as columns in
// host memory that the context's workspace owns; valid until its next run.
struct RecordColumns {
    const double *x = nullptr, *y = nullptr, *z = nullptr, *cx = nullptr, *cy = nullptr, *cz = nullptr;
    const int *element = nullptr, *stage = nullptr, *raynum = nullptr;
    size_t n = 0;
};

struct RunResult {
    bool ok = false;
    bool cancelled = false;
    std::string error;
    uint64_t sun_rays = 0, ray_hits = 0;
    RecordColumns rec;               // the run's records in the reference's order (host memory of the workspace)
    std::vector<uint64_t> stage_entries;
    std::vector<uint32_t> max_enter, max_ttmiss;
    std::vector<std::vector<unsigned long long>> flux;
    std::vector<unsigned long long> first_hits, absorbed, delivered;
    double device_ms = 0;  // first launch to last completion, CUDA events on the run's stream
    double probe_ms = 0, trace_ms = 0, setup_ms = 0, readback_ms = 0;
    int batches = 0, gpu_launches = 0;
    unsigned flags = 0;
    uint64_t intersections = 0;  // records of the run by the reference's rules, kept or not
    std::vector<double> saved[2];  // rays leaving stage 1 and stage 2 (7 doubles per ray), unordered
    uint64_t h2d_bytes = 0, d2h_bytes = 0;
    int probe_variant = 0, trace_variant = 0;
};

// One sun position of a batched run (st_b200_sim_run_batch): the tables that depend on the
// sun (sun frame and box, sun-plane grid) and, when the first stage tracks the
// sun, the scene's elements with the first stage re-aimed.
struct SunPosition {
    SunDev sun;                       // device pointers are filled by gpu_run_batch
    std::vector<int> cell_start;
    std::vector<float4> cell_disc, cell_par, cell_xa, cell_xb, cell_xc;
    std::vector<double> rot;          // tracking: the first stage's re-aimed rotations, 9 per element
                                      // (empty: the scene's elements as they are)
    uint64_t n_hits = 0;
    uint32_t seed = 0;
};

struct PositionResult {
    uint64_t sun_rays = 0, ray_hits = 0, intersections = 0;
    std::vector<uint64_t> stage_entries;
    std::vector<uint32_t> max_enter;
    std::vector<std::vector<unsigned long long>> flux;  // per flux map of the request
    std::vector<unsigned long long> absorbed;           // per element of the scene
};

struct BatchResult {
    bool ok = false;
    std::string error;
    std::vector<PositionResult> pos;
    double device_ms = 0, probe_ms = 0, trace_ms = 0, setup_ms = 0;
    int gpu_launches = 0, batches = 0, waves = 0;
    uint64_t h2d_bytes = 0, d2h_bytes = 0;
    int probe_variant = 0;
};

struct Workspace;
Workspace *workspace_create();
void workspace_destroy(Workspace *w);
bool gpu_run(const HostScene &hs, const RunRequest &rq, RunResult &out, Workspace &ws);
// K sun positions over one scene in one launch sequence: every position's sun-ray batches
// are queued without a host round trip, the host reading the positions' progress once per
// wave.  rq supplies precision, device, flux maps and the sun-ray cap per position.
// `slot`: the staging area (0 or 1) that stage_positions filled with `pos`, -1 for none.
bool gpu_run_batch(const HostScene &hs, const std::vector<SunPosition> &pos, const RunRequest &rq, BatchResult &out,
                   Workspace &ws, int slot);
// Binds a workspace to a device (a workspace bound to another is started afresh) and gives it
// its stream; called before positions are staged into it.
bool workspace_bind(Workspace &ws, int device);
// Gathers the positions' sun-plane tables and tracking rotations, on all host cores, into the
// workspace's page-locked staging area `slot` (0 or 1), laid out as gpu_run_batch copies them
// to the device, so that a chunk is staged while the device runs the previous one.  false
// (nothing staged; gpu_run_batch then copies from the vectors) when page-locked memory cannot
// be had or the workspace is not bound to `device`.
bool stage_positions(Workspace &ws, int slot, const std::vector<SunPosition> &pos, int device);

// st_host.cpp: set up and flatten the scene of a context; append a message to it
bool prepare_scene(void *ctx, HostScene &hs);
void report(void *ctx, const std::string &msg);
// the device a context runs on (st_b200_set_device), and whether its rays come from the sun
// (false when it was given explicit rays or is replaying saved stage data)
bool context_device(void *ctx, int &device, bool &sun_rays);

}  // namespace stb
