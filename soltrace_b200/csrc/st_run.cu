// Run driver: uploads the flattened scene, loops sun-ray batches through the
// probe / compact / trace kernels until the requested number of first-stage hits
// is numbered, and brings counters, flux maps and records back to the host.
//
// Semantics kept from the reference (coretrace/raytrace.cpp:582-604, 780-798):
// ray numbers go to first-stage hits in sun-ray order; the run stops at the
// hit numbered `raycount`, and SunRayCount is the number of sun rays generated
// up to and including that ray; running out of `maxcount` sun rays first is an
// error.  Because every ray has its own Philox stream keyed by its sun index,
// batch boundaries do not change any result.
#include <chrono>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <thread>

#include "st_host.h"
#include "st_launch.h"

namespace stb {

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    // at least b bytes; a buffer that must grow gets a quarter more than asked, so that runs
    // whose sizes drift by a little (batch sizes planned from the last run's hit rate) do not
    // reallocate (cudaFree waits for the whole device)
    cudaError_t ensure(size_t b) {
        if (b <= bytes && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        const size_t want = b ? b + b / 4 : 16;
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {  // without the headroom
            cudaGetLastError();
            e = cudaMalloc(&p, b ? b : 16);
            if (e == cudaSuccess) bytes = b ? b : 16;
            return e;
        }
        bytes = want;
        return e;
    }
    // grow to at least b bytes keeping the first `keep` bytes (stream-ordered copy)
    cudaError_t grow_keep(size_t b, size_t keep, cudaStream_t s) {
        if (b <= bytes && p) return cudaSuccess;
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, b ? b : 16);
        if (e != cudaSuccess) return e;
        if (p && keep && (e = cudaMemcpyAsync(q, p, std::min(keep, bytes), cudaMemcpyDeviceToDevice, s))) {
            cudaFree(q);
            return e;
        }
        if (p) cudaFree(p);  // waits for the copy
        p = q;
        bytes = b;
        return cudaSuccess;
    }
    template <typename T>
    T *as() const {
        return static_cast<T *>(p);
    }
};

template <typename T>
cudaError_t upload(DevBuf &b, const std::vector<T> &v, cudaStream_t s, uint64_t &bytes) {
    cudaError_t e = b.ensure(std::max<size_t>(v.size() * sizeof(T), 16));
    if (e != cudaSuccess || v.empty()) return e;
    bytes += v.size() * sizeof(T);
    return cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s);
}

}  // namespace

// Device buffers, stream and events of one context, kept across runs so that a
// repeated st_sim_run pays no allocation: every buffer only grows.
struct Workspace {
    int device = -1;
    cudaStream_t stream = nullptr;
    DevBuf stage_cells, grid_sphere, grid_elem, beam_axis, beam_range, beam_elem;
    DevBuf elems, elem_sphere, optics, surf, tables, bvh, bvh_items, cell_start, cell_disc, cell_par, inv_cdf, expos,
        excos;
    DevBuf acc, ctr, rs, rec_count, counts, offsets, total, scan_parts, recs;
    DevBuf cand;      // probe's ray list: count, then one sun-ray index per entry
    DevBuf cand_el;   // probe's result per list entry (element + 1, 0 for a miss)
    DevBuf hit_mask;  // one bit per sun ray of the batch, set for a hit
    DevBuf amb;       // mixed probe: count, then the rays left to the double-precision search
    // trace state and queues (one slot per hit-list entry of a batch)
    DevBuf wf_sid, wf_raynum, wf_draw, wf_meta, wf_fe0, wf_p, wf_c, wf_q0, wf_q1, wf_qs, wf_counts;
    DevBuf save_rows[2], save_count, replay_rows, replay_fe0;  // stage-data save / replay
    DevBuf ecount, ecursor, etotal, s_hits;  // the batch's hits sorted by first-stage element (HitRec)
    // record ordering: key counts / slots, scan partials, per-stage counts, merge runs, columns
    DevBuf rec_key, rec_parts, rec_parts2, rec_stage, rec_runs, rec_cols, rec_bad;
    // batched runs: two page-locked staging areas, the positions' tables of a chunk gathered
    // in one while the device runs the chunk staged in the other
    void *pos_host[2] = {nullptr, nullptr};
    size_t pos_host_bytes[2] = {0, 0};
    size_t pos_staged_bytes[2] = {0, 0}, pos_staged_k[2] = {0, 0};  // what each area holds
    bool pos_dma_pending[2] = {false, false};  // a copy out of the area may still be running
    void *rec_host = nullptr;  // the ordered records' columns in host memory (pinned when possible)
    size_t rec_host_bytes = 0;
    bool rec_host_pinned = false;
    // batched runs: per-position sun tables, element copies, run states, counters, accumulators
    DevBuf pos_cells, pos_disc, pos_par, pos_xa, pos_xb, pos_xc, pos_elems, pos_rot, pos_rs, pos_ctr, pos_acc;
    DevBuf cell_xa, cell_xb, cell_xc;  // exact flat footprints of the sun-plane grid
    std::vector<cudaEvent_t> events;
    // autotuned kernel variants per precision (FP64, mixed), chosen on the first run
    struct Tuning {
        bool done = false;
        int probe = 0;
    } tune[2];
    DevBuf tune_rs;
    ~Workspace() {
        if (device >= 0) cudaSetDevice(device);
        for (int k = 0; k < 2; ++k)
            if (pos_host[k]) cudaFreeHost(pos_host[k]);
        if (rec_host) {
            if (rec_host_pinned)
                cudaFreeHost(rec_host);
            else
                free(rec_host);
        }
        for (auto e : events) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
    }
};

Workspace *workspace_create() { return new Workspace; }
void workspace_destroy(Workspace *w) { delete w; }

namespace {
double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

// The probe outputs of a batch of n sun rays, in the workspace's buffers.
static cudaError_t probe_buffers(Workspace &ws, uint64_t n, ProbeOut &o) {
    const size_t nb = size_t((n + kProbeBlock - 1) / kProbeBlock);
    cudaError_t e;
    if ((e = ws.counts.ensure(nb * 4)) || (e = ws.cand.ensure((n + 1) * 4)) || (e = ws.cand_el.ensure(n * 4)) ||
        (e = ws.hit_mask.ensure(hit_mask_words(n) * 4)) || (e = ws.amb.ensure((n + 1) * 4)))
        return e;
    o = ProbeOut{};
    o.amb_count = ws.amb.as<uint32_t>();
    o.amb = o.amb_count + 1;
    o.block_counts = ws.counts.as<uint32_t>();
    o.cand_count = ws.cand.as<uint32_t>();
    o.cand = o.cand_count + 1;
    o.cand_el = ws.cand_el.as<uint32_t>();
    o.hit_mask = ws.hit_mask.as<uint32_t>();
    return cudaSuccess;
}

// Autotuner: time every variant of the probe (register budgets, or rays per thread of the
// mixed flat-rectangle probe) on the same 2^24 sun rays (indices 0.., outputs discarded into
// scratch buffers: enough blocks to fill the GPU at every variant's rays per block, as the
// 2^26-ray batches do) and keep the fastest for this workspace and precision.  Variants share
// their arithmetic, so the choice changes timing only.
static cudaError_t autotune(Workspace &ws, const SceneDev &S0, int precision, uint64_t max_sun, cudaStream_t st,
                            int &launches) {
    Workspace::Tuning &tu = ws.tune[precision ? 1 : 0];
    const uint64_t n = std::min<uint64_t>(uint64_t(1) << 24, max_sun);
    if (n == 0) return cudaSuccess;
    cudaError_t e;
    ProbeOut po;
    if ((e = probe_buffers(ws, n, po)) || (e = ws.tune_rs.ensure(sizeof(RunState)))) return e;
    SceneDev S = S0;
    S.n_flux = 0;
    RunState r0;
    memset(&r0, 0, sizeof r0);
    r0.target = ~0ull;
    RunState *rs = ws.tune_rs.as<RunState>();
    cudaMemcpyAsync(rs, &r0, sizeof r0, cudaMemcpyHostToDevice, st);
    cudaEvent_t ev[2 * kProbeVariants];
    for (auto &x : ev) cudaEventCreate(&x);
    auto probe = [&](int v) {
        if (precision)
            launches += launch_probe_mixed(S, 0, uint32_t(n), po, rs, v, st);
        else
            launches += launch_probe_fp64(S, 0, uint32_t(n), po, rs, v, st);
    };
    probe(0);  // warm the caches
    for (int v = 0; v < kProbeVariants; ++v) {
        cudaEventRecord(ev[2 * v], st);
        probe(v);
        cudaEventRecord(ev[2 * v + 1], st);
    }
    e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) {
        float best = 1e30f;
        for (int v = 0; v < kProbeVariants; ++v) {
            float ms = 0;
            cudaEventElapsedTime(&ms, ev[2 * v], ev[2 * v + 1]);
            if (ms < best * 0.98f) {
                best = ms;
                tu.probe = v;
            }
        }
        tu.done = true;
    }
    for (auto &x : ev) cudaEventDestroy(x);
    return e;
}

// trace state and queues for up to `cap` rays: one search queue per search kind among the
// stages (and round parity)
static cudaError_t wf_buffers(Workspace &ws, const SceneDev &S, uint64_t cap, WfState &W, WfQueues &Q) {
    cudaError_t e;
    cap = std::max<uint64_t>(cap, 1);
    const int nst = S.n_stages;
    Q = WfQueues{};
    int queue_of_kind[kSearchKinds];
    for (int &q : queue_of_kind) q = -1;
    for (int s = 0; s < nst; ++s) {
        const int k = stage_search_kind(S.stages[s]);
        if (queue_of_kind[k] < 0) {
            queue_of_kind[k] = Q.n_queues;
            Q.queue_kind[Q.n_queues++] = k;
        }
        Q.stage_queue[s] = (unsigned char)queue_of_kind[k];
    }
    const uint64_t nq = uint64_t(std::max(Q.n_queues, 1));
    if ((e = ws.wf_sid.ensure(cap * 8)) || (e = ws.wf_raynum.ensure(cap * 4)) || (e = ws.wf_draw.ensure(cap * 4)) ||
        (e = ws.wf_meta.ensure(cap * 16)) || (e = ws.wf_fe0.ensure(cap * 4)) || (e = ws.wf_p.ensure(cap * 24)) ||
        (e = ws.wf_c.ensure(cap * 24)) || (e = ws.wf_q0.ensure(nq * cap * 4)) ||
        (e = ws.wf_q1.ensure(nq * cap * 4)) || (e = ws.wf_qs.ensure(cap * 4)))
        return e;
    Q.rounds = 2 * nst;
    Q.cap = uint32_t(cap);
    if ((e = ws.wf_counts.ensure(sizeof(uint32_t) * (Q.rounds + 1) * (nq + 1)))) return e;
    Q.search[0] = ws.wf_q0.as<uint32_t>();
    Q.search[1] = ws.wf_q1.as<uint32_t>();
    Q.shade = ws.wf_qs.as<uint32_t>();
    Q.counts = ws.wf_counts.as<uint32_t>();
    W.sid = ws.wf_sid.as<uint64_t>();
    W.raynum = ws.wf_raynum.as<uint32_t>();
    W.draw = ws.wf_draw.as<uint32_t>();
    W.meta = ws.wf_meta.as<int4>();
    W.fe0 = ws.wf_fe0.as<int>();
    W.p = ws.wf_p.as<double>();
    W.c = ws.wf_c.as<double>();
    W.cap = uint32_t(cap);
    return cudaSuccess;
}

// TRayData::Merge (types.cpp:311-355): a stage's records are kept in blocks of 8192; merging
// the stages in turn puts the full blocks of all stages so far first and packs the partial
// blocks' records after them.  Returns the runs of the merged order: (stage, start in the
// stage's sorted order, length), in output order.
struct MergeRun {
    int s;
    uint64_t start, n;
};
static std::vector<MergeRun> merge_runs(const std::vector<uint64_t> &per_stage) {
    const uint64_t B = 8192;
    auto blk_size = [](const std::vector<MergeRun> &b) {
        uint64_t t = 0;
        for (auto &r : b) t += r.n;
        return t;
    };
    std::vector<std::vector<MergeRun>> all;
    for (int s = 0; s < int(per_stage.size()); ++s) {
        const uint64_t n = per_stage[size_t(s)];
        std::vector<std::vector<MergeRun>> full, partial;
        for (auto &b : all) (blk_size(b) == B ? full : partial).push_back(b);
        for (uint64_t i = 0; i < n; i += B) {
            std::vector<MergeRun> b{MergeRun{s, i, std::min(B, n - i)}};
            (b[0].n == B ? full : partial).push_back(b);
        }
        all = full;
        for (auto &b : partial)
            for (const MergeRun &r : b) {
                uint64_t done = 0;
                while (done < r.n) {
                    if (all.empty() || blk_size(all.back()) == B) all.push_back({});
                    const uint64_t k = std::min(B - blk_size(all.back()), r.n - done);
                    all.back().push_back(MergeRun{r.s, r.start + done, k});
                    done += k;
                }
            }
    }
    std::vector<MergeRun> out;
    for (auto &b : all)
        for (const MergeRun &r : b) {
            if (!out.empty() && out.back().s == r.s && out.back().start + out.back().n == r.start)
                out.back().n += r.n;  // contiguous pieces of one stage
            else
                out.push_back(r);
        }
    return out;
}

// Put the run's nrec device records into the reference's readback order (per stage by ray
// number and hit index, then the block merge), dropping the records the reference does not
// write (drop_later: every record after the first stage; tt_drop[s]: the miss record of that
// ray number in trace-through stage s), as columns in the workspace's host buffer.
static std::string order_records(Workspace &ws, const RecordDev *recs, unsigned long long nrec, int nst,
                                 bool drop_later, const uint32_t *tt_drop, uint32_t rb, RecordColumns &col,
                                 uint64_t &d2h, cudaStream_t st) {
    col = RecordColumns{};
    const uint64_t nkeys = uint64_t(nst) * (uint64_t(rb) + 1);
    if (nkeys >= (uint64_t(1) << 31) || nrec >= (uint64_t(1) << 31))
        return "too many records to order (at most 2^31 records and stages x ray numbers)";
    cudaError_t e;
    RecOrder o{};
    o.recs = recs;
    o.n = nrec;
    o.rb = rb;
    o.nst = nst;
    o.drop_later = drop_later ? 1 : 0;
    for (int s = 0; s < nst; ++s) o.tt_drop[s] = tt_drop[s];
    if ((e = ws.rec_key.ensure(nkeys * 4)) || (e = ws.rec_stage.ensure(kMaxStages * 8)) ||
        (e = ws.rec_bad.ensure(8)) || (e = ws.rec_parts.ensure(scan_parts(uint32_t(nkeys)) * 4)) ||
        (e = ws.rec_parts2.ensure(scan_parts(uint32_t(scan_parts(uint32_t(nkeys)))) * 4)))
        return std::string("CUDA error: ") + cudaGetErrorString(e);
    o.key = ws.rec_key.as<uint32_t>();
    o.stage_count = ws.rec_stage.as<unsigned long long>();
    o.bad = ws.rec_bad.as<unsigned int>();
    cudaMemsetAsync(o.key, 0, nkeys * 4, st);
    cudaMemsetAsync(o.stage_count, 0, kMaxStages * 8, st);
    cudaMemsetAsync(o.bad, 0, 8, st);
    if (nrec) launch_rec_count(o, st);
    unsigned long long cnt[kMaxStages] = {0};
    unsigned int bad = 0;
    cudaMemcpyAsync(cnt, o.stage_count, kMaxStages * 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&bad, o.bad, 4, cudaMemcpyDeviceToHost, st);
    // the key slots: exclusive scan of the counts, in place (runs while the host plans the merge)
    launch_scan_large(o.key, uint32_t(nkeys), o.key, ws.rec_bad.as<uint32_t>() + 1, ws.rec_parts.as<uint32_t>(),
                      ws.rec_parts2.as<uint32_t>(), st);
    if ((e = cudaStreamSynchronize(st))) return std::string("CUDA error: ") + cudaGetErrorString(e);
    if (bad) return "a record's ray number lies outside the run's ray numbers";
    std::vector<uint64_t> per(static_cast<size_t>(nst));
    uint64_t total = 0;
    for (int s = 0; s < nst; ++s) total += (per[size_t(s)] = cnt[s]);
    // merge runs per stage, by start: (source start, destination) pairs and per-stage segments
    const std::vector<MergeRun> runs = merge_runs(per);
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> by_stage(static_cast<size_t>(nst));
    uint64_t dst = 0;
    for (const MergeRun &r : runs) {
        by_stage[size_t(r.s)].push_back({uint32_t(r.start), uint32_t(dst)});
        dst += r.n;
    }
    std::vector<uint32_t> table;  // run_src | run_dst | run_seg (as uint32)
    std::vector<uint32_t> src, dsts;
    std::vector<int> seg(static_cast<size_t>(nst) + 1, 0);
    for (int s = 0; s < nst; ++s) {
        auto &v = by_stage[size_t(s)];
        std::sort(v.begin(), v.end());
        seg[size_t(s)] = int(src.size());
        for (auto &pr : v) {
            src.push_back(pr.first);
            dsts.push_back(pr.second);
        }
        if (v.empty()) {  // a stage without records: one empty run keeps the search in range
            src.push_back(0);
            dsts.push_back(0);
        }
    }
    seg[size_t(nst)] = int(src.size());
    const size_t nr = src.size();
    table.resize(2 * nr + seg.size());
    std::copy(src.begin(), src.end(), table.begin());
    std::copy(dsts.begin(), dsts.end(), table.begin() + nr);
    for (size_t k = 0; k < seg.size(); ++k) table[2 * nr + k] = uint32_t(seg[k]);
    const size_t col_bytes = size_t(total) * (6 * sizeof(double) + 3 * sizeof(int));
    if ((e = ws.rec_runs.ensure(table.size() * 4)) || (e = ws.rec_cols.ensure(std::max<size_t>(col_bytes, 16))))
        return std::string("CUDA error: ") + cudaGetErrorString(e);
    if ((e = cudaMemcpyAsync(ws.rec_runs.p, table.data(), table.size() * 4, cudaMemcpyHostToDevice, st)))
        return std::string("CUDA error: ") + cudaGetErrorString(e);
    o.run_src = ws.rec_runs.as<uint32_t>();
    o.run_dst = o.run_src + nr;
    o.run_seg = reinterpret_cast<const int *>(o.run_src + 2 * nr);
    o.col_d = ws.rec_cols.as<double>();
    o.col_i = reinterpret_cast<int *>(o.col_d + 6 * total);
    o.total = total;
    if (nrec && total) launch_rec_scatter(o, st);
    // host buffer (grows only; page-locked when the system allows it)
    if (ws.rec_host_bytes < col_bytes) {
        if (ws.rec_host) {
            if (ws.rec_host_pinned)
                cudaFreeHost(ws.rec_host);
            else
                free(ws.rec_host);
        }
        ws.rec_host = nullptr;
        ws.rec_host_bytes = 0;
        ws.rec_host_pinned = cudaMallocHost(&ws.rec_host, col_bytes) == cudaSuccess;
        if (!ws.rec_host_pinned) {
            cudaGetLastError();
            ws.rec_host = malloc(col_bytes);
        }
        if (!ws.rec_host) return "out of host memory for the records";
        ws.rec_host_bytes = col_bytes;
    }
    if (col_bytes && (e = cudaMemcpyAsync(ws.rec_host, ws.rec_cols.p, col_bytes, cudaMemcpyDeviceToHost, st)))
        return std::string("CUDA error: ") + cudaGetErrorString(e);
    cudaMemcpyAsync(&bad, o.bad, 4, cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st))) return std::string("CUDA error: ") + cudaGetErrorString(e);
    if (bad) return "the records could not be put in order";
    d2h += col_bytes + 8 * kMaxStages + 8;
    const double *cd = static_cast<const double *>(ws.rec_host);
    const int *ci = reinterpret_cast<const int *>(cd + 6 * total);
    col.x = cd;
    col.y = cd + total;
    col.z = cd + 2 * total;
    col.cx = cd + 3 * total;
    col.cy = cd + 4 * total;
    col.cz = cd + 5 * total;
    col.element = ci;
    col.stage = ci + total;
    col.raynum = ci + 2 * total;
    col.n = size_t(total);
    return "";
}

#define CK(x)                                                                                 \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess) {                                                              \
            out.error = std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #x;     \
            return false;                                                                     \
        }                                                                                     \
    } while (0)

bool gpu_run(const HostScene &hs, const RunRequest &rq, RunResult &out, Workspace &ws) {
    const auto t_setup = std::chrono::steady_clock::now();
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        out.error = "no CUDA device is available to the B200 trace";
        return false;
    }
    if (rq.device < 0 || rq.device >= ndev) {
        out.error = "CUDA device ordinal out of range";
        return false;
    }
    CK(cudaSetDevice(rq.device));
    if (ws.device != rq.device) {  // a workspace serves one device: start afresh on another
        ws.~Workspace();
        new (&ws) Workspace();
        ws.device = rq.device;
    }
    if (!ws.stream) CK(cudaStreamCreateWithFlags(&ws.stream, cudaStreamNonBlocking));
    cudaStream_t st = ws.stream;
    DevBuf &d_elems = ws.elems, &d_optics = ws.optics, &d_surf = ws.surf, &d_tables = ws.tables, &d_bvh = ws.bvh,
           &d_bvh_items = ws.bvh_items, &d_cell_start = ws.cell_start, &d_cell_disc = ws.cell_disc,
           &d_inv_cdf = ws.inv_cdf, &d_expos = ws.expos, &d_excos = ws.excos;
    CK(upload(d_elems, hs.elems, st, out.h2d_bytes));
    CK(upload(ws.elem_sphere, hs.elem_sphere, st, out.h2d_bytes));
    CK(upload(ws.stage_cells, hs.stage_cells, st, out.h2d_bytes));
    CK(upload(ws.grid_sphere, hs.grid_sphere, st, out.h2d_bytes));
    CK(upload(ws.grid_elem, hs.grid_elem, st, out.h2d_bytes));
    CK(upload(ws.beam_axis, hs.beam_axis, st, out.h2d_bytes));
    CK(upload(ws.beam_range, hs.beam_range, st, out.h2d_bytes));
    CK(upload(ws.beam_elem, hs.beam_elem, st, out.h2d_bytes));
    CK(upload(d_optics, hs.optics, st, out.h2d_bytes));
    CK(upload(d_surf, hs.surf_data, st, out.h2d_bytes));
    CK(upload(d_tables, hs.tables, st, out.h2d_bytes));
    CK(upload(d_bvh, hs.bvh, st, out.h2d_bytes));
    CK(upload(d_bvh_items, hs.bvh_items, st, out.h2d_bytes));
    CK(upload(d_cell_start, hs.cell_start, st, out.h2d_bytes));
    CK(upload(d_cell_disc, hs.cell_disc, st, out.h2d_bytes));
    CK(upload(ws.cell_par, hs.cell_par, st, out.h2d_bytes));
    CK(upload(ws.cell_xa, hs.cell_xa, st, out.h2d_bytes));
    CK(upload(ws.cell_xb, hs.cell_xb, st, out.h2d_bytes));
    CK(upload(ws.cell_xc, hs.cell_xc, st, out.h2d_bytes));
    CK(upload(d_inv_cdf, hs.inv_cdf, st, out.h2d_bytes));
    CK(upload(d_expos, rq.ex_pos, st, out.h2d_bytes));
    CK(upload(d_excos, rq.ex_cos, st, out.h2d_bytes));

    SceneDev S = hs.dev;
    S.elems = d_elems.as<ElemRec>();
    S.elem_sphere = ws.elem_sphere.as<float4>();
    S.stage_cells = ws.stage_cells.as<int2>();
    S.grid_sphere = ws.grid_sphere.as<float4>();
    S.grid_elem = ws.grid_elem.as<int>();
    S.beam_axis = hs.beam_axis.empty() ? nullptr : ws.beam_axis.as<float4>();
    S.beam_range = ws.beam_range.as<int2>();
    S.beam_elem = ws.beam_elem.as<int>();
    S.optics = d_optics.as<OpticRec>();
    S.surf_data = d_surf.as<double>();
    S.tables = d_tables.as<double>();
    S.bvh = d_bvh.as<BvhNode>();
    S.bvh_items = d_bvh_items.as<int>();
    S.sun.cell_start = d_cell_start.as<int>();
    S.sun.cell_disc = d_cell_disc.as<float4>();
    S.sun.cell_par = ws.cell_par.as<float4>();
    S.sun.cell_xa = ws.cell_xa.as<float4>();
    S.sun.cell_xb = ws.cell_xb.as<float4>();
    S.sun.cell_xc = ws.cell_xc.as<float4>();
    if (hs.cell_xa.size() != hs.cell_disc.size() || hs.cell_xa.empty()) S.sun.exact_flat = 0;
    S.sun.inv_cdf = hs.inv_cdf.empty() ? nullptr : d_inv_cdf.as<double>();
    S.seed = rq.seed;
    S.precision = rq.precision;
    const bool explicit_mode = !rq.ex_pos.empty();
    const uint64_t n_explicit = rq.ex_pos.size() / 3;
    S.explicit_rays = explicit_mode ? 1 : 0;
    S.ex_pos = d_expos.as<double>();
    S.ex_cos = d_excos.as<double>();

    // run-level accumulators: [first_hits | absorbed | delivered | flux bins of every map]
    const size_t ne = hs.elems.size();
    std::vector<size_t> flux_off;
    size_t acc_n = 3 * ne;
    const size_t n_src0 = size_t(hs.dev.stages[0].n_elem);
    auto map_size = [n_src0](const FluxMapReq &f) { return size_t(f.nx) * f.ny * (f.per_source ? n_src0 : 1); };
    for (const auto &f : rq.flux) {
        flux_off.push_back(acc_n);
        acc_n += map_size(f);
    }
    if (rq.flux.size() > size_t(kMaxFluxMaps)) {
        out.error = "too many flux maps";
        return false;
    }
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, rq.device);

    const int nst = S.n_stages;
    const uint64_t kMaxBatch = uint64_t(1) << 26;
    // one rank of a run over several GPUs: every batch's sun-ray range is split contiguously
    // over the ranks; after the probe the ranks exchange their hit counts, so that each numbers
    // its hits after the hits of the ranks before it and the run stops at the same hit as on
    // one GPU (app/src/trace.cpp:709-735 is the reference's independent-context convention
    // this replaces)
    const bool multi = rq.nranks > 1;
    const int R = multi ? rq.nranks : 1;
    if (multi && (explicit_mode || rq.replay || rq.save_stage_data || !rq.allgather || !rq.allreduce ||
                  rq.rank < 0 || rq.rank >= rq.nranks)) {
        out.error = "runs over several ranks trace sun rays with both exchange callbacks set (no explicit rays, "
                    "replay or stage-data saving)";
        return false;
    }
    auto exchange = [&](const std::vector<unsigned long long> &send, std::vector<unsigned long long> &recv) -> bool {
        recv.assign(send.size() * size_t(R), 0ull);
        return rq.allgather(send.data(), recv.data(), int(send.size()), rq.comm_user) != 0;
    };
    DevBuf &d_acc = ws.acc, &d_ctr = ws.ctr, &d_rs = ws.rs, &d_rec_count = ws.rec_count, &d_offsets = ws.offsets,
           &d_total = ws.total, &d_recs = ws.recs;
    // the batch's hits are grouped by first-stage element (the rays of a warp then leave
    // one element and walk the same candidates)
    const uint32_t n_elem0 = uint32_t(S.stages[0].n_elem);
    DevBuf &d_ecount = ws.ecount, &d_ecursor = ws.ecursor, &d_etotal = ws.etotal, &d_s_hits = ws.s_hits;
    CK(d_ecount.ensure(size_t(n_elem0) * 4));
    CK(d_ecursor.ensure(size_t(n_elem0) * 4));
    CK(d_etotal.ensure(8));
    unsigned long long rec_cap = 0, save_cap = 0;
    Workspace::Tuning &tu = ws.tune[rq.precision ? 1 : 0];
    if (!tu.done && !explicit_mode && !rq.replay) CK(autotune(ws, S, rq.precision, rq.max_sun, st, out.gpu_launches));
    out.probe_variant = tu.probe;
    out.trace_variant = 0;
    (void)dev_sms;
    CK(cudaStreamSynchronize(st));
    out.setup_ms = ms_since(t_setup);

    // room for `need` records in the run's record buffer, keeping the first `keep`
    auto rec_room = [&](unsigned long long need, unsigned long long keep) -> cudaError_t {
        if (need <= rec_cap) return cudaSuccess;
        const unsigned long long cap = std::max(need, rec_cap + rec_cap / 2);
        cudaError_t e = d_recs.grow_keep(cap * sizeof(RecordDev), keep * sizeof(RecordDev), st);
        if (e == cudaSuccess) rec_cap = cap;
        return e;
    };
    double rec_per_ray = 2.0 * nst;  // records per numbered ray expected when sizing the buffer
    for (int attempt = 0; attempt < 4; ++attempt) {
        bool restart = false;
        out.rec = RecordColumns{};
        out.stage_entries.assign(nst, 0);
        out.max_enter.assign(nst, 0);
        out.max_ttmiss.assign(nst, 0);
        out.batches = 0;
        out.probe_ms = out.trace_ms = 0;
        CK(d_acc.ensure(std::max<size_t>(acc_n, 1) * 8));
        CK(d_ctr.ensure(sizeof(RunCounters)));
        CK(d_rs.ensure(sizeof(RunState)));
        CK(d_rec_count.ensure(8));
        // the run's records accumulate on the device over its batches and are put in order at
        // the end; a replay's saved stage-1 records come first
        const unsigned long long n_pre = rq.pre_records.size();
        unsigned long long nrec_run = 0;  // records written so far (read after every batch)
        if (rq.records) {
            CK(d_recs.ensure(std::max<unsigned long long>(rec_cap, n_pre + 4096) * sizeof(RecordDev)));
            rec_cap = d_recs.bytes / sizeof(RecordDev);
            if (n_pre)
                CK(cudaMemcpyAsync(d_recs.p, rq.pre_records.data(), n_pre * sizeof(RecordDev),
                                   cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(d_rec_count.p, &n_pre, 8, cudaMemcpyHostToDevice, st));
            out.h2d_bytes += n_pre * sizeof(RecordDev) + 8;
            nrec_run = n_pre;
        }
        CK(cudaMemsetAsync(d_acc.p, 0, std::max<size_t>(acc_n, 1) * 8, st));
        CK(cudaMemsetAsync(d_ctr.p, 0, sizeof(RunCounters), st));
        RunState rs0;
        memset(&rs0, 0, sizeof rs0);
        rs0.target = explicit_mode ? ~0ull : rq.n_hits;
        CK(cudaMemcpyAsync(d_rs.p, &rs0, sizeof rs0, cudaMemcpyHostToDevice, st));
        out.h2d_bytes += sizeof rs0;
        unsigned long long *acc = d_acc.as<unsigned long long>();
        S.n_flux = int(rq.flux.size());
        for (size_t m = 0; m < rq.flux.size(); ++m) {
            const FluxMapReq &f = rq.flux[m];
            FluxMapDev &fd = S.flux[m];
            fd.stage = f.stage;
            fd.elem = f.elem;
            fd.kind = f.kind;
            fd.nx = f.nx;
            fd.ny = f.ny;
            fd.absorbed_only = f.absorbed_only;
            fd.n_src = f.per_source ? int(n_src0) : 0;
            fd.x0 = f.x0;
            fd.x1 = f.x1;
            fd.y0 = f.y0;
            fd.y1 = f.y1;
            fd.bins = acc + flux_off[m];
        }
        TraceOut O;
        O.ctr = d_ctr.as<RunCounters>();
        O.first_hits = acc;
        O.absorbed = acc + ne;
        O.delivered = acc + 2 * ne;
        O.rec_count = d_rec_count.as<unsigned long long>();
        RunState *drs = d_rs.as<RunState>();

        // Batches are queued without host round trips unless records are kept (each
        // batch's records are copied out) or a progress callback is installed.
        const bool sync_each = rq.records || rq.callback != nullptr || rq.save_stage_data;
        out.saved[0].clear();
        out.saved[1].clear();
        // stage-data saving: room for every numbered ray of a batch in each of the two lists
        O.save_rows[0] = O.save_rows[1] = nullptr;
        O.save_count[0] = O.save_count[1] = nullptr;
        O.save_cap = 0;
        auto save_setup = [&](uint64_t rays) -> cudaError_t {
            if (!rq.save_stage_data) return cudaSuccess;
            cudaError_t e;
            const uint64_t cap =
                std::max<uint64_t>(save_cap, std::min<uint64_t>(rays, explicit_mode || rq.replay ? rays : rq.n_hits) + 16);
            for (int k = 0; k < 2; ++k)
                if ((e = ws.save_rows[k].ensure(cap * 7 * sizeof(double)))) return e;
            if ((e = ws.save_count.ensure(16)) || (e = cudaMemsetAsync(ws.save_count.p, 0, 16, st))) return e;
            for (int k = 0; k < 2; ++k) {
                O.save_rows[k] = ws.save_rows[k].as<double>();
                O.save_count[k] = ws.save_count.as<unsigned long long>() + k;
            }
            O.save_cap = cap;
            return cudaSuccess;
        };
        // after a synchronised batch: append its saved rays (overflow: re-run with more room)
        auto save_collect = [&](bool &overflow) -> cudaError_t {
            overflow = false;
            if (!rq.save_stage_data) return cudaSuccess;
            unsigned long long cnt[2] = {0, 0};
            cudaError_t e = cudaMemcpy(cnt, ws.save_count.p, 16, cudaMemcpyDeviceToHost);
            if (e) return e;
            for (int k = 0; k < 2; ++k)
                if (cnt[k] > O.save_cap) {
                    save_cap = cnt[k] + cnt[k] / 4 + 1024;
                    overflow = true;
                    return cudaSuccess;
                }
            for (int k = 0; k < 2; ++k) {
                const size_t old = out.saved[k].size();
                out.saved[k].resize(old + size_t(cnt[k]) * 7);
                if (cnt[k] && (e = cudaMemcpy(out.saved[k].data() + old, O.save_rows[k],
                                              size_t(cnt[k]) * 7 * sizeof(double), cudaMemcpyDeviceToHost)))
                    return e;
                out.d2h_bytes += 8 + cnt[k] * 7 * sizeof(double);
            }
            return cudaSuccess;
        };
        uint64_t sun_next = 0;
        uint64_t global_done = 0;  // over several ranks: hits numbered by all ranks so far
        double p_est = rq.hit_rate_hint > 0 ? rq.hit_rate_hint : 0.0;
        RunState rs = rs0;
        size_t ev_used = 0;
        auto new_event = [&]() {
            if (ev_used == ws.events.size()) {
                cudaEvent_t e;
                cudaEventCreate(&e);
                ws.events.push_back(e);
            }
            return ws.events[ev_used++];
        };
        std::vector<std::pair<cudaEvent_t, cudaEvent_t>> probe_ev, trace_ev;
        cudaEvent_t t_first = new_event(), t_last = new_event();
        CK(cudaEventRecord(t_first, st));
        bool done = false;
        if (rq.replay) {
            // saved stage data: the rays enter the second stage directly (no sun rays, no probe)
            const uint64_t n1 = rq.replay_rows.size() / 7;
            CK(upload(ws.replay_rows, rq.replay_rows, st, out.h2d_bytes));
            CK(upload(ws.replay_fe0, rq.replay_fe0, st, out.h2d_bytes));
            if (rq.records) CK(rec_room(nrec_run + std::max<uint64_t>(n1, 1) * uint64_t(nst) * 2 + 4096, nrec_run));
            O.recs = rq.records ? d_recs.as<RecordDev>() : nullptr;
            O.rec_cap = rq.records ? rec_cap : 0;
            WfState W;
            WfQueues Q;
            CK(wf_buffers(ws, S, n1, W, Q));
            CK(save_setup(n1));
            ReplayIn rin;
            rin.rows = ws.replay_rows.as<double>();
            rin.fe0 = rq.replay_fe0.empty() ? nullptr : ws.replay_fe0.as<int>();
            rin.n = uint32_t(n1);
            cudaEvent_t p1 = new_event(), p2 = new_event();
            CK(cudaEventRecord(p1, st));
            if (rq.precision)
                out.gpu_launches +=
                    launch_trace_mixed(rq.records, S, nullptr, nullptr, drs, O, W, Q, &rin, st);
            else
                out.gpu_launches +=
                    launch_trace_fp64(rq.records, S, nullptr, nullptr, drs, O, W, Q, &rin, st);
            CK(cudaEventRecord(p2, st));
            CK(cudaGetLastError());
            trace_ev.push_back({p1, p2});
            out.batches = 1;
            unsigned long long nrec = 0;
            if (rq.records) CK(cudaMemcpyAsync(&nrec, d_rec_count.p, 8, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (rq.records && nrec > rec_cap) {
                rec_cap = nrec + nrec / 4 + 4096;
                continue;
            }
            bool save_over = false;
            CK(save_collect(save_over));
            if (save_over) continue;
            nrec_run = nrec;
            rs.hits_done = rs.sun_rays = rq.replay_sun_rays;
            rs.reached = 1;
            done = true;
        }
        while (!done) {
            // plan the next group of batches
            uint64_t want;
            if (explicit_mode) {
                want = n_explicit - sun_next;
            } else {
                const uint64_t need = rq.n_hits - (multi ? global_done : rs.hits_done);
                if (p_est <= 0.0)
                    want = std::min<uint64_t>(uint64_t(1) << 20, rq.max_sun - sun_next);  // pilot batch
                else
                    want = uint64_t(1.03 * double(need) / p_est) + 65536;
                want = std::min<uint64_t>(want, rq.max_sun - sun_next);
            }
            if (want == 0) {
                if (explicit_mode) break;
                char buf[160];
                snprintf(buf, sizeof buf, "generated sun rays reached maximum count: %llu",
                         (unsigned long long)rq.max_sun);
                out.error = buf;
                return false;
            }
            uint64_t queued = 0;
            while (queued < want) {
                // this batch's global sun-ray range [sun_next, sun_next + n_all) and, over several
                // ranks, this rank's contiguous slice [s0, s0 + n) of it
                const uint64_t n_all = std::min<uint64_t>(kMaxBatch * uint64_t(R), want - queued);
                uint64_t n = n_all, s0 = sun_next;
                if (multi) {
                    const uint64_t base = n_all / uint64_t(R), rem = n_all % uint64_t(R);
                    const uint64_t rk = uint64_t(rq.rank);
                    n = base + (rk < rem ? 1 : 0);
                    s0 = sun_next + rk * base + std::min<uint64_t>(rk, rem);
                }
                const uint32_t nb = uint32_t((std::max<uint64_t>(n, 1) + kProbeBlock - 1) / kProbeBlock);
                ProbeOut po;
                CK(probe_buffers(ws, std::max<uint64_t>(n, 1), po));
                CK(d_offsets.ensure(size_t(nb) * 4));
                CK(ws.scan_parts.ensure(scan_parts(nb) * 4));
                CK(d_total.ensure(8));
                CK(d_s_hits.ensure(std::max<uint64_t>(n, 1) * sizeof(HitRec)));
                if (rq.records) {
                    // room for this batch's records: its numbered rays at the records per ray seen so far
                    const uint64_t numbered = multi ? global_done : rs.hits_done;
                    const uint64_t left = explicit_mode ? n : rq.n_hits - std::min<uint64_t>(rq.n_hits, numbered);
                    const double est = double(std::min<uint64_t>(n, left)) * rec_per_ray;
                    CK(rec_room(nrec_run + uint64_t(est) + 4096, nrec_run));
                }
                O.recs = rq.records ? d_recs.as<RecordDev>() : nullptr;
                O.rec_cap = rq.records ? rec_cap : 0;
                cudaEvent_t p0 = new_event(), p1 = new_event(), p2 = new_event();
                CK(cudaEventRecord(p0, st));
                if (n > 0) {
                    if (rq.precision)
                        out.gpu_launches += launch_probe_mixed(S, s0, uint32_t(n), po, drs, tu.probe, st);
                    else
                        out.gpu_launches += launch_probe_fp64(S, s0, uint32_t(n), po, drs, tu.probe, st);
                    launch_scan(po.block_counts, nb, d_offsets.as<uint32_t>(), d_total.as<uint32_t>(),
                                ws.scan_parts.as<uint32_t>(), st);
                    out.gpu_launches += 2;
                } else {
                    CK(cudaMemsetAsync(d_total.p, 0, 8, st));
                }
                if (multi) {
                    // every rank's hit count in this batch: this rank's hits are numbered after those of
                    // the ranks before it, and the ranks after the run's last hit trace nothing
                    uint32_t tot = 0;
                    CK(cudaMemcpyAsync(&tot, d_total.p, 4, cudaMemcpyDeviceToHost, st));
                    CK(cudaMemcpyAsync(&rs, drs, sizeof rs, cudaMemcpyDeviceToHost, st));
                    CK(cudaStreamSynchronize(st));
                    out.d2h_bytes += 4 + sizeof rs;
                    std::vector<unsigned long long> got;
                    if (!exchange({(unsigned long long)tot}, got)) {
                        out.error = "the exchange of hit counts between ranks failed";
                        return false;
                    }
                    uint64_t before = 0, all = 0;
                    for (int k = 0; k < R; ++k) {
                        if (k < rq.rank) before += got[size_t(k)];
                        all += got[size_t(k)];
                    }
                    const uint64_t base = global_done + before;
                    rs.target = rq.n_hits;
                    rs.hits_done = std::min<uint64_t>(base, rq.n_hits);
                    rs.reached = base >= rq.n_hits ? 1u : 0u;
                    rs.cursor = 0;
                    rs.cut_sid = 0;
                    CK(cudaMemcpyAsync(drs, &rs, sizeof rs, cudaMemcpyHostToDevice, st));
                    out.h2d_bytes += sizeof rs;
                    global_done += std::min<uint64_t>(all, rq.n_hits - global_done);
                }
                if (n > 0) {
                    launch_list_sort(s0, po, d_offsets.as<uint32_t>(), d_total.as<uint32_t>(), drs, n_elem0,
                                     d_ecount.as<uint32_t>(), d_ecursor.as<uint32_t>(), d_etotal.as<uint32_t>(),
                                     d_s_hits.as<HitRec>(),
                                     uint32_t(n), st);
                    out.gpu_launches += 3;  // element counts, their scan, scatter
                }
                const HitRec *t_hits = d_s_hits.as<HitRec>();
                // trace state and queues: one slot per hit-list entry (at most n)
                WfState W;
                WfQueues Q;
                CK(wf_buffers(ws, S, n, W, Q));
                CK(save_setup(n));
                CK(cudaEventRecord(p1, st));
                if (n > 0) {
                    if (rq.precision)
                        out.gpu_launches += launch_trace_mixed(rq.records, S, t_hits,
                                                               d_total.as<uint32_t>(), drs, O, W, Q, nullptr, st);
                    else
                        out.gpu_launches += launch_trace_fp64(rq.records, S, t_hits,
                                                              d_total.as<uint32_t>(), drs, O, W, Q, nullptr, st);
                }
                CK(cudaEventRecord(p2, st));
                if (n > 0) {
                    launch_advance(d_total.as<uint32_t>(), nullptr, s0, uint32_t(n), drs, st);
                    out.gpu_launches += 1;
                }
                CK(cudaGetLastError());
                probe_ev.push_back({p0, p1});
                trace_ev.push_back({p1, p2});
                queued += n_all;
                sun_next += n_all;
                out.batches++;
                if (sync_each) {
                    CK(cudaMemcpyAsync(&rs, drs, sizeof rs, cudaMemcpyDeviceToHost, st));
                    out.d2h_bytes += sizeof rs;
                    unsigned long long nrec = 0;
                    if (rq.records) CK(cudaMemcpyAsync(&nrec, d_rec_count.p, 8, cudaMemcpyDeviceToHost, st));
                    CK(cudaStreamSynchronize(st));
                    const unsigned long long nrec_local = nrec;
                    bool overflow = rq.records && nrec > rec_cap;
                    if (multi) {  // a rank out of record room makes every rank re-run, in step
                        std::vector<unsigned long long> got;
                        if (!exchange({overflow ? 1ull : 0ull, rec_cap, nrec}, got)) {
                            out.error = "the exchange of record counts between ranks failed";
                            return false;
                        }
                        for (int k = 0; k < R; ++k) {
                            overflow = overflow || got[3 * size_t(k)] != 0;
                            rec_cap = std::max<unsigned long long>(rec_cap, got[3 * size_t(k) + 1]);
                            nrec = std::max<unsigned long long>(nrec, got[3 * size_t(k) + 2]);
                        }
                    }
                    if (overflow) {
                        rec_cap = nrec + nrec / 4 + 4096;  // re-run the whole job with room for it
                        restart = true;
                        break;
                    }
                    bool save_over = false;
                    CK(save_collect(save_over));
                    if (save_over) {
                        restart = true;
                        break;
                    }
                    if (rq.records) {
                        nrec_run = nrec_local;
                        out.d2h_bytes += 8;
                        if (!multi && rs.hits_done > 0)
                            rec_per_ray = std::max(1.0, 1.5 * double(nrec_run - n_pre) / double(rs.hits_done));
                    }
                    if (rq.callback &&
                        !rq.callback((unsigned long)rs.sun_rays, (unsigned long)rs.hits_done,
                                     (unsigned long)(explicit_mode ? n_explicit : rq.n_hits), 1ul, (unsigned long)nst,
                                     rq.cbdata)) {
                        out.cancelled = true;
                        done = true;
                        break;
                    }
                    if (multi ? global_done == rq.n_hits : rs.reached != 0) break;
                }
                if (multi && global_done == rq.n_hits) break;
            }
            if (restart) break;
            CK(cudaMemcpyAsync(&rs, drs, sizeof rs, cudaMemcpyDeviceToHost, st));
            out.d2h_bytes += sizeof rs;
            CK(cudaStreamSynchronize(st));
            const uint64_t done_hits = multi ? global_done : rs.hits_done;
            if ((multi ? global_done == rq.n_hits : rs.reached != 0) || out.cancelled ||
                (explicit_mode && sun_next >= n_explicit))
                done = true;
            if (!explicit_mode && sun_next > 0) p_est = std::max(double(done_hits) / double(sun_next), 1e-9);
        }
        if (restart) continue;
        CK(cudaEventRecord(t_last, st));
        CK(cudaStreamSynchronize(st));
        float ms = 0;
        cudaEventElapsedTime(&ms, t_first, t_last);
        out.device_ms = ms;
        for (auto &pe : probe_ev) {
            float x = 0;
            cudaEventElapsedTime(&x, pe.first, pe.second);
            out.probe_ms += x;
        }
        for (auto &pe : trace_ev) {
            float x = 0;
            cudaEventElapsedTime(&x, pe.first, pe.second);
            out.trace_ms += x;
        }
        out.ray_hits = multi ? global_done : rs.hits_done;
        out.sun_rays = explicit_mode ? n_explicit : rs.sun_rays;
        if (!explicit_mode && !(multi ? global_done == rq.n_hits : rs.reached != 0) && !out.cancelled) {
            out.error = "run ended before the requested hits were numbered";
            return false;
        }
        RunCounters c;
        CK(cudaMemcpyAsync(&c, d_ctr.p, sizeof c, cudaMemcpyDeviceToHost, st));
        const auto tr = std::chrono::steady_clock::now();
        std::vector<unsigned long long> accv(acc_n);
        if (acc_n) CK(cudaMemcpyAsync(accv.data(), d_acc.p, acc_n * 8, cudaMemcpyDeviceToHost, st));
        out.d2h_bytes += acc_n * 8 + sizeof c;
        CK(cudaStreamSynchronize(st));
        unsigned fe_fail = rq.precision ? take_fe_failures_mixed() : take_fe_failures_fp64();
        if (multi) {
            // the run's totals over all ranks: counts summed, SunRayCount (the cutting rank's;
            // the others' are below it), largest ray numbers and flags by max; integer, so exact
            std::vector<unsigned long long> sum(kMaxStages + 1 + acc_n), mx(2 * kMaxStages + 2 + 32);
            for (int k = 0; k < kMaxStages; ++k) sum[size_t(k)] = c.stage_entries[k];
            sum[kMaxStages] = c.records;
            std::copy(accv.begin(), accv.end(), sum.begin() + kMaxStages + 1);
            for (int k = 0; k < kMaxStages; ++k) {
                mx[size_t(k)] = c.max_enter[k];
                mx[size_t(kMaxStages + k)] = c.max_ttmiss[k];
            }
            mx[2 * kMaxStages] = rs.sun_rays;
            mx[2 * kMaxStages + 1] = fe_fail ? 1 : 0;
            for (int b = 0; b < 32; ++b) mx[size_t(2 * kMaxStages + 2 + b)] = (c.flags >> b) & 1u;
            if (!rq.allreduce(sum.data(), sum.size(), 0, rq.comm_user) ||
                !rq.allreduce(mx.data(), mx.size(), 1, rq.comm_user)) {
                out.error = "the reduction of the run's counters over ranks failed";
                return false;
            }
            for (int k = 0; k < kMaxStages; ++k) c.stage_entries[k] = sum[size_t(k)];
            c.records = sum[kMaxStages];
            std::copy(sum.begin() + kMaxStages + 1, sum.end(), accv.begin());
            for (int k = 0; k < kMaxStages; ++k) {
                c.max_enter[k] = unsigned(mx[size_t(k)]);
                c.max_ttmiss[k] = unsigned(mx[size_t(kMaxStages + k)]);
            }
            out.sun_rays = mx[2 * kMaxStages];
            fe_fail = mx[2 * kMaxStages + 1] ? 1u : 0u;
            c.flags = 0;
            for (int b = 0; b < 32; ++b)
                if (mx[size_t(2 * kMaxStages + 2 + b)]) c.flags |= 1u << b;
        }
        for (int s = 0; s < nst; ++s) {
            out.stage_entries[s] = c.stage_entries[s];
            out.max_enter[s] = c.max_enter[s];
            out.max_ttmiss[s] = c.max_ttmiss[s];
        }
        out.flags = c.flags;
        out.intersections = c.records;
        out.first_hits.assign(accv.begin(), accv.begin() + ne);
        out.absorbed.assign(accv.begin() + ne, accv.begin() + 2 * ne);
        out.delivered.assign(accv.begin() + 2 * ne, accv.begin() + 3 * ne);
        out.flux.clear();
        for (size_t m = 0; m < rq.flux.size(); ++m)
            out.flux.emplace_back(accv.begin() + flux_off[m], accv.begin() + flux_off[m] + map_size(rq.flux[m]));
        out.readback_ms += ms_since(tr);
        if (fe_fail) {
            // the reference throws at such a query (vshot.cpp:177-178) and returns no result
            out.error = "Interpolation failed to find nearby nodes to ray hit in FEA surface.";
            return false;
        }
        if (out.flags & kFlagBadInteraction) {
            out.error = "Bad optical interaction type (only 1 = refraction and 2 = reflection are traced)";
            return false;
        }
        if (rq.records) {
            // the records the reference writes, in its order: the ray that alone left the first
            // stage as the last numbered one is not traced further (raytrace.cpp:786-797); the
            // last ray of a trace-through stage that misses leaves no record (810-811)
            const auto to = std::chrono::steady_clock::now();
            const uint32_t N = uint32_t(out.ray_hits);
            const bool drop_later = !rq.replay && nst > 1 && out.stage_entries[1] == 1 && out.max_enter[1] == N;
            uint32_t tt_drop[kMaxStages] = {0};
            uint32_t rb = N;
            for (int s = 0; s < nst; ++s) {
                rb = std::max(rb, out.max_enter[size_t(s)]);
                if (s >= 1 && S.stages[s].tracethrough && out.max_ttmiss[size_t(s)] != 0 &&
                    out.max_ttmiss[size_t(s)] == out.max_enter[size_t(s)])
                    tt_drop[s] = out.max_enter[size_t(s)];
            }
            for (const RecordDev &r : rq.pre_records) rb = std::max(rb, r.raynum);
            const std::string err = order_records(ws, d_recs.as<RecordDev>(), std::min(nrec_run, rec_cap), nst,
                                                  drop_later, tt_drop, rb, out.rec, out.d2h_bytes, st);
            if (!err.empty()) {
                out.error = err;
                return false;
            }
            out.readback_ms += ms_since(to);
        }
        out.ok = true;
        return true;
    }
    out.error = "record buffer could not be sized for this run";
    return false;
}

#undef CK
#define CK(x)                                                                                 \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess) {                                                              \
            out.error = std::string("CUDA error: ") + cudaGetErrorString(e_) + " at " #x;     \
            return false;                                                                     \
        }                                                                                     \
    } while (0)

// Batched run of K sun positions (st_b200_sim_run_batch).  Every position p has its own
// scene view S_p (its sun frame, sun-plane grid and, when tracking, elements),
// run state, counters and accumulators; its rays draw from the streams of its own seed, so
// position p's results are those of a single run with that sun and seed.  Positions advance
// in waves: a wave queues, for every position still short of its hits, the sun rays its hit
// rate (measured by the previous wave; the first wave probes 2^20 rays) says it needs, with
// no host round trip inside the wave; the host then reads all positions' run states at once.
namespace {
// Where a chunk's positions sit in the device tables (and in a staging area laid out the
// same way: one region per array, positions end to end).
struct PosLayout {
    std::vector<size_t> off_cells, off_disc, off_rot;
    size_t n_cells = 0, n_disc = 0, n_rot = 0;
    bool all_exact = true;
    size_t b_cells = 0, b_disc = 0, b_rot = 0, nx = 0, b_all = 0;
    explicit PosLayout(const std::vector<SunPosition> &pos) : off_cells(pos.size()), off_disc(pos.size()),
                                                              off_rot(pos.size()) {
        for (const SunPosition &sp : pos)
            if (!sp.sun.exact_flat || sp.cell_xa.size() != sp.cell_disc.size() || sp.cell_xa.empty()) all_exact = false;
        for (size_t p = 0; p < pos.size(); ++p) {
            off_cells[p] = n_cells;
            n_cells += pos[p].cell_start.size();
            off_disc[p] = n_disc;
            n_disc += pos[p].cell_disc.size();
            off_rot[p] = n_rot;
            n_rot += pos[p].rot.size();
        }
        nx = all_exact ? 3 : 0;
        b_cells = n_cells * sizeof(int);
        b_disc = n_disc * sizeof(float4);
        b_rot = n_rot * sizeof(double);
        b_all = b_cells + (2 + nx) * b_disc + b_rot;
    }
    // region starts in a staging area: cells, disc, par, xa, xb, xc, rot
    void regions(char *base, char *r[7]) const {
        r[0] = base;
        r[1] = r[0] + b_cells;
        r[2] = r[1] + b_disc;
        r[3] = r[2] + b_disc;
        r[4] = r[3] + (nx ? b_disc : 0);
        r[5] = r[4] + (nx ? b_disc : 0);
        r[6] = r[5] + (nx ? b_disc : 0);
    }
};
}  // namespace

bool workspace_bind(Workspace &ws, int device) {
    if (cudaSetDevice(device) != cudaSuccess) return false;
    if (ws.device != device) {  // a workspace serves one device: start afresh on another
        ws.~Workspace();
        new (&ws) Workspace();
        ws.device = device;
    }
    return ws.stream || cudaStreamCreateWithFlags(&ws.stream, cudaStreamNonBlocking) == cudaSuccess;
}

bool stage_positions(Workspace &ws, int slot, const std::vector<SunPosition> &pos, int device) {
    if (slot < 0 || slot > 1) return false;
    ws.pos_staged_bytes[slot] = ws.pos_staged_k[slot] = 0;
    const PosLayout L(pos);
    // only into a workspace already bound to the device (workspace_bind), which the batch
    // run will not start afresh
    if (L.b_all == 0 || ws.device != device || cudaSetDevice(device) != cudaSuccess) return false;
    if (ws.pos_dma_pending[slot] && ws.stream) {  // a run that failed may have left its copy running
        cudaStreamSynchronize(ws.stream);
        cudaGetLastError();
        ws.pos_dma_pending[slot] = false;
    }
    if (ws.pos_host_bytes[slot] < L.b_all) {
        if (ws.pos_host[slot]) cudaFreeHost(ws.pos_host[slot]);
        ws.pos_host[slot] = nullptr;
        ws.pos_host_bytes[slot] = 0;
        const size_t want = L.b_all + L.b_all / 4;
        if (cudaMallocHost(&ws.pos_host[slot], want) != cudaSuccess) {
            ws.pos_host[slot] = nullptr;
            cudaGetLastError();  // the vectors are copied instead
            return false;
        }
        ws.pos_host_bytes[slot] = want;
    }
    char *r[7];
    L.regions(static_cast<char *>(ws.pos_host[slot]), r);
    auto cp = [](char *dst, const void *src, size_t bytes) {
        if (bytes) memcpy(dst, src, bytes);
    };
    auto gather = [&](size_t p) {
        const SunPosition &sp = pos[p];
        const size_t od = L.off_disc[p] * sizeof(float4), nd = sp.cell_disc.size() * sizeof(float4);
        cp(r[0] + L.off_cells[p] * sizeof(int), sp.cell_start.data(), sp.cell_start.size() * sizeof(int));
        cp(r[1] + od, sp.cell_disc.data(), nd);
        cp(r[2] + od, sp.cell_par.data(), sp.cell_par.size() * sizeof(float4));
        if (L.nx) {
            cp(r[3] + od, sp.cell_xa.data(), nd);
            cp(r[4] + od, sp.cell_xb.data(), nd);
            cp(r[5] + od, sp.cell_xc.data(), nd);
        }
        cp(r[6] + L.off_rot[p] * sizeof(double), sp.rot.data(), sp.rot.size() * sizeof(double));
    };
    const size_t K = pos.size();
    const size_t nth = std::max<size_t>(1, std::min<size_t>(K, std::thread::hardware_concurrency()));
    std::vector<std::thread> th;
    for (size_t t = 0; t < nth; ++t)
        th.emplace_back([&gather, t, nth, K]() {
            for (size_t p = t; p < K; p += nth) gather(p);
        });
    for (auto &x : th) x.join();
    ws.pos_staged_bytes[slot] = L.b_all;
    ws.pos_staged_k[slot] = K;
    return true;
}

bool gpu_run_batch(const HostScene &hs, const std::vector<SunPosition> &pos, const RunRequest &rq, BatchResult &out,
                   Workspace &ws, int slot) {
    const auto t_setup = std::chrono::steady_clock::now();
    const size_t K = pos.size();
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        out.error = "no CUDA device is available to the B200 trace";
        return false;
    }
    if (rq.device < 0 || rq.device >= ndev) {
        out.error = "CUDA device ordinal out of range";
        return false;
    }
    if (K == 0) {
        out.ok = true;
        return true;
    }
    CK(cudaSetDevice(rq.device));
    if (ws.device != rq.device) {
        ws.~Workspace();
        new (&ws) Workspace();
        ws.device = rq.device;
    }
    if (!ws.stream) CK(cudaStreamCreateWithFlags(&ws.stream, cudaStreamNonBlocking));
    cudaStream_t st = ws.stream;
    uint64_t &h2d = out.h2d_bytes;
    // the scene's shared tables
    CK(upload(ws.elems, hs.elems, st, h2d));
    CK(upload(ws.elem_sphere, hs.elem_sphere, st, h2d));
    CK(upload(ws.stage_cells, hs.stage_cells, st, h2d));
    CK(upload(ws.grid_sphere, hs.grid_sphere, st, h2d));
    CK(upload(ws.grid_elem, hs.grid_elem, st, h2d));
    CK(upload(ws.optics, hs.optics, st, h2d));
    CK(upload(ws.surf, hs.surf_data, st, h2d));
    CK(upload(ws.tables, hs.tables, st, h2d));
    CK(upload(ws.bvh, hs.bvh, st, h2d));
    CK(upload(ws.bvh_items, hs.bvh_items, st, h2d));
    CK(upload(ws.inv_cdf, hs.inv_cdf, st, h2d));
    // every position's tables, laid end to end on the device: sized first, then each position's
    // arrays copied straight from its own vectors (no host-side concatenation)
    std::vector<size_t> off_cells(K), off_disc(K), off_elems(K), off_rot(K);
    bool all_exact = true;
    for (const SunPosition &sp : pos)
        if (!sp.sun.exact_flat || sp.cell_xa.size() != sp.cell_disc.size() || sp.cell_xa.empty()) all_exact = false;
    const size_t n_elem_all = hs.elems.size(), n_first = size_t(hs.dev.stages[0].n_elem);
    size_t n_cells = 0, n_disc = 0, n_elems = 0, n_rot = 0;
    for (size_t p = 0; p < K; ++p) {
        const SunPosition &sp = pos[p];
        if (!sp.rot.empty() && sp.rot.size() != n_first * 9) {
            out.error = "sun position " + std::to_string(p) + ": rotations do not match the first stage";
            return false;
        }
        off_cells[p] = n_cells;
        n_cells += sp.cell_start.size();
        off_disc[p] = n_disc;
        n_disc += sp.cell_disc.size();
        off_elems[p] = sp.rot.empty() ? size_t(-1) : n_elems;  // a re-aimed copy of the element table
        n_elems += sp.rot.empty() ? 0 : n_elem_all;
        off_rot[p] = n_rot;
        n_rot += sp.rot.size();
    }
    CK(ws.pos_cells.ensure(std::max<size_t>(n_cells * sizeof(int), 16)));
    CK(ws.pos_disc.ensure(std::max<size_t>(n_disc * sizeof(float4), 16)));
    CK(ws.pos_par.ensure(std::max<size_t>(n_disc * sizeof(float4), 16)));
    if (all_exact) {
        CK(ws.pos_xa.ensure(std::max<size_t>(n_disc * sizeof(float4), 16)));
        CK(ws.pos_xb.ensure(std::max<size_t>(n_disc * sizeof(float4), 16)));
        CK(ws.pos_xc.ensure(std::max<size_t>(n_disc * sizeof(float4), 16)));
    }
    CK(ws.pos_elems.ensure(std::max<size_t>(n_elems * sizeof(ElemRec), 16)));
    CK(ws.pos_rot.ensure(std::max<size_t>(n_rot * sizeof(double), 16)));
    auto put = [&](DevBuf &dst, size_t off_elems_of_t, const void *src, size_t bytes) -> cudaError_t {
        if (!bytes) return cudaSuccess;
        h2d += bytes;
        return cudaMemcpyAsync(static_cast<char *>(dst.p) + off_elems_of_t, src, bytes, cudaMemcpyHostToDevice, st);
    };
    // The positions' tables, staged by stage_positions in page-locked memory laid out as on the
    // device, go over with one copy per array; otherwise each position's arrays are copied from
    // its own vectors.
    const PosLayout L(pos);
    const bool staged = slot >= 0 && slot <= 1 && ws.pos_host[slot] && ws.pos_staged_k[slot] == K &&
                        ws.pos_staged_bytes[slot] == L.b_all && L.b_all > 0 && L.all_exact == all_exact;
    if (staged) {
        char *r[7];
        L.regions(static_cast<char *>(ws.pos_host[slot]), r);
        ws.pos_dma_pending[slot] = true;
        CK(put(ws.pos_cells, 0, r[0], L.b_cells));
        CK(put(ws.pos_disc, 0, r[1], L.b_disc));
        CK(put(ws.pos_par, 0, r[2], L.b_disc));
        if (L.nx) {
            CK(put(ws.pos_xa, 0, r[3], L.b_disc));
            CK(put(ws.pos_xb, 0, r[4], L.b_disc));
            CK(put(ws.pos_xc, 0, r[5], L.b_disc));
        }
        CK(put(ws.pos_rot, 0, r[6], L.b_rot));
    }
    for (size_t p = 0; p < K; ++p) {
        const SunPosition &sp = pos[p];
        if (!staged) {
            CK(put(ws.pos_cells, off_cells[p] * sizeof(int), sp.cell_start.data(), sp.cell_start.size() * sizeof(int)));
            const size_t od = off_disc[p] * sizeof(float4), nd = sp.cell_disc.size() * sizeof(float4);
            CK(put(ws.pos_disc, od, sp.cell_disc.data(), nd));
            CK(put(ws.pos_par, od, sp.cell_par.data(), sp.cell_par.size() * sizeof(float4)));
            if (all_exact) {
                CK(put(ws.pos_xa, od, sp.cell_xa.data(), nd));
                CK(put(ws.pos_xb, od, sp.cell_xb.data(), nd));
                CK(put(ws.pos_xc, od, sp.cell_xc.data(), nd));
            }
            CK(put(ws.pos_rot, off_rot[p] * sizeof(double), sp.rot.data(), sp.rot.size() * sizeof(double)));
        }
        if (!sp.rot.empty()) {
            // the scene's element table (already on the device) copied, then the re-aimed
            // rotations of the first stage written over it: 72 bytes per heliostat cross PCIe
            // instead of the whole element record
            ElemRec *el = ws.pos_elems.as<ElemRec>() + off_elems[p];
            CK(cudaMemcpyAsync(el, ws.elems.p, n_elem_all * sizeof(ElemRec), cudaMemcpyDeviceToDevice, st));
            launch_set_rotations(el + hs.dev.stages[0].first_elem, uint32_t(n_first), ws.pos_rot.as<double>() + off_rot[p], st);
            ++out.gpu_launches;
        }
    }

    SceneDev S0 = hs.dev;
    S0.elems = ws.elems.as<ElemRec>();
    S0.elem_sphere = ws.elem_sphere.as<float4>();
    S0.stage_cells = ws.stage_cells.as<int2>();
    S0.grid_sphere = ws.grid_sphere.as<float4>();
    S0.grid_elem = ws.grid_elem.as<int>();
    S0.beam_axis = nullptr;  // outgoing-beam lists depend on the sun: blocking searches walk the ground grid
    S0.beam_range = nullptr;
    S0.beam_elem = nullptr;
    S0.optics = ws.optics.as<OpticRec>();
    S0.surf_data = ws.surf.as<double>();
    S0.tables = ws.tables.as<double>();
    S0.bvh = ws.bvh.as<BvhNode>();
    S0.bvh_items = ws.bvh_items.as<int>();
    S0.precision = rq.precision;
    S0.explicit_rays = 0;
    S0.ex_pos = S0.ex_cos = nullptr;

    const int nst = S0.n_stages;
    const size_t ne = hs.elems.size();
    std::vector<size_t> flux_off;
    size_t acc_n = 3 * ne;
    const size_t n_src0 = size_t(hs.dev.stages[0].n_elem);
    auto map_size = [n_src0](const FluxMapReq &f) { return size_t(f.nx) * f.ny * (f.per_source ? n_src0 : 1); };
    for (const auto &f : rq.flux) {
        flux_off.push_back(acc_n);
        acc_n += map_size(f);
    }
    if (rq.flux.size() > size_t(kMaxFluxMaps)) {
        out.error = "too many flux maps";
        return false;
    }
    CK(ws.pos_rs.ensure(K * sizeof(RunState)));
    CK(ws.pos_ctr.ensure(K * sizeof(RunCounters)));
    CK(ws.pos_acc.ensure(K * acc_n * 8 + 8));
    CK(cudaMemsetAsync(ws.pos_ctr.p, 0, K * sizeof(RunCounters), st));
    CK(cudaMemsetAsync(ws.pos_acc.p, 0, K * acc_n * 8 + 8, st));
    std::vector<RunState> rs_h(K);
    for (size_t p = 0; p < K; ++p) {
        memset(&rs_h[p], 0, sizeof(RunState));
        rs_h[p].target = pos[p].n_hits;
    }
    CK(cudaMemcpyAsync(ws.pos_rs.p, rs_h.data(), K * sizeof(RunState), cudaMemcpyHostToDevice, st));
    h2d += K * sizeof(RunState);

    std::vector<SceneDev> Sp(K, S0);
    std::vector<TraceOut> Op(K);
    unsigned long long *acc = ws.pos_acc.as<unsigned long long>();
    for (size_t p = 0; p < K; ++p) {
        SceneDev &S = Sp[p];
        S.sun = pos[p].sun;
        S.sun.cell_start = ws.pos_cells.as<int>() + off_cells[p];
        S.sun.cell_disc = ws.pos_disc.as<float4>() + off_disc[p];
        S.sun.cell_par = ws.pos_par.as<float4>() + off_disc[p];
        S.sun.exact_flat = all_exact ? 1 : 0;
        S.sun.cell_xa = all_exact ? ws.pos_xa.as<float4>() + off_disc[p] : nullptr;
        S.sun.cell_xb = all_exact ? ws.pos_xb.as<float4>() + off_disc[p] : nullptr;
        S.sun.cell_xc = all_exact ? ws.pos_xc.as<float4>() + off_disc[p] : nullptr;
        S.sun.inv_cdf = hs.inv_cdf.empty() ? nullptr : ws.inv_cdf.as<double>();
        if (off_elems[p] != size_t(-1)) S.elems = ws.pos_elems.as<ElemRec>() + off_elems[p];
        S.seed = pos[p].seed;
        unsigned long long *a = acc + p * acc_n;
        S.n_flux = int(rq.flux.size());
        for (size_t m = 0; m < rq.flux.size(); ++m) {
            const FluxMapReq &f = rq.flux[m];
            FluxMapDev &fd = S.flux[m];
            fd.stage = f.stage;
            fd.elem = f.elem;
            fd.kind = f.kind;
            fd.nx = f.nx;
            fd.ny = f.ny;
            fd.absorbed_only = f.absorbed_only;
            fd.n_src = f.per_source ? int(n_src0) : 0;
            fd.x0 = f.x0;
            fd.x1 = f.x1;
            fd.y0 = f.y0;
            fd.y1 = f.y1;
            fd.bins = a + flux_off[m];
        }
        TraceOut &O = Op[p];
        memset(&O, 0, sizeof O);
        O.ctr = ws.pos_ctr.as<RunCounters>() + p;
        O.first_hits = a;
        O.absorbed = a + ne;
        O.delivered = a + 2 * ne;
        O.recs = nullptr;
        O.rec_cap = 0;
        O.rec_count = ws.rec_count.as<unsigned long long>();
    }
    CK(ws.rec_count.ensure(8));
    for (auto &O : Op) O.rec_count = ws.rec_count.as<unsigned long long>();

    // buffers for the largest batch, sized before anything is queued (growing a buffer frees
    // the old one, which must not happen under queued work)
    const uint64_t kMaxBatch = uint64_t(1) << 26;
    const uint32_t n_elem0 = uint32_t(S0.stages[0].n_elem);
    {
        const uint64_t n = kMaxBatch;
        const uint32_t nb = uint32_t((n + kProbeBlock - 1) / kProbeBlock);
        ProbeOut po;
        WfState W;
        WfQueues Q;
        CK(probe_buffers(ws, n, po));
        CK(ws.offsets.ensure(size_t(nb) * 4));
        CK(ws.scan_parts.ensure(scan_parts(nb) * 4));
        CK(ws.total.ensure(8));
        CK(ws.s_hits.ensure(n * sizeof(HitRec)));
        CK(ws.ecount.ensure(size_t(std::max<uint32_t>(n_elem0, 1)) * 4));
        CK(ws.ecursor.ensure(size_t(std::max<uint32_t>(n_elem0, 1)) * 4));
        CK(ws.etotal.ensure(8));
        CK(wf_buffers(ws, S0, n, W, Q));
    }
    Workspace::Tuning &tu = ws.tune[rq.precision ? 1 : 0];
    if (!tu.done) CK(autotune(ws, Sp[0], rq.precision, rq.max_sun, st, out.gpu_launches));
    out.probe_variant = tu.probe;
    CK(cudaStreamSynchronize(st));
    out.setup_ms = ms_since(t_setup);

    size_t ev_used = 0;
    auto new_event = [&]() {
        if (ev_used == ws.events.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            ws.events.push_back(e);
        }
        return ws.events[ev_used++];
    };
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> probe_ev, trace_ev;
    cudaEvent_t t_first = new_event(), t_last = new_event();
    CK(cudaEventRecord(t_first, st));
    RunState *drs = ws.pos_rs.as<RunState>();
    std::vector<uint64_t> sun_next(K, 0);
    std::vector<double> p_est(K, 0.0);
    std::vector<bool> reached(K, false);
    size_t left = K;
    for (size_t p = 0; p < K; ++p)
        if (pos[p].n_hits == 0) {  // nothing to trace: SunRayCount 0
            reached[p] = true;
            --left;
        }
    while (left > 0) {
        out.waves++;
        for (size_t p = 0; p < K; ++p) {
            if (reached[p]) continue;
            uint64_t want;
            const uint64_t need = pos[p].n_hits - rs_h[p].hits_done;
            if (p_est[p] <= 0.0)
                want = std::min<uint64_t>(uint64_t(1) << 20, rq.max_sun - sun_next[p]);
            else
                want = std::min<uint64_t>(uint64_t(1.03 * double(need) / p_est[p]) + 65536, rq.max_sun - sun_next[p]);
            if (want == 0) {
                char buf[200];
                snprintf(buf, sizeof buf, "sun position %zu: generated sun rays reached maximum count: %llu", p,
                         (unsigned long long)rq.max_sun);
                out.error = buf;
                return false;
            }
            const SceneDev &S = Sp[p];
            for (uint64_t queued = 0; queued < want;) {
                const uint64_t n = std::min<uint64_t>(kMaxBatch, want - queued);
                const uint32_t nb = uint32_t((n + kProbeBlock - 1) / kProbeBlock);
                ProbeOut po;
                WfState W;
                WfQueues Q;
                CK(probe_buffers(ws, n, po));
                CK(wf_buffers(ws, S, n, W, Q));
                cudaEvent_t p0 = new_event(), p1 = new_event(), p2 = new_event();
                CK(cudaEventRecord(p0, st));
                const uint64_t s0 = sun_next[p];
                if (rq.precision)
                    out.gpu_launches += launch_probe_mixed(S, s0, uint32_t(n), po, drs + p, tu.probe, st);
                else
                    out.gpu_launches += launch_probe_fp64(S, s0, uint32_t(n), po, drs + p, tu.probe, st);
                launch_scan(po.block_counts, nb, ws.offsets.as<uint32_t>(), ws.total.as<uint32_t>(),
                            ws.scan_parts.as<uint32_t>(), st);
                launch_list_sort(s0, po, ws.offsets.as<uint32_t>(), ws.total.as<uint32_t>(), drs + p, n_elem0,
                                 ws.ecount.as<uint32_t>(), ws.ecursor.as<uint32_t>(), ws.etotal.as<uint32_t>(),
                                 ws.s_hits.as<HitRec>(),
                                 uint32_t(n), st);
                CK(cudaEventRecord(p1, st));
                if (rq.precision)
                    out.gpu_launches += launch_trace_mixed(false, S, ws.s_hits.as<HitRec>(), ws.total.as<uint32_t>(), drs + p,
                                                           Op[p], W, Q, nullptr, st);
                else
                    out.gpu_launches += launch_trace_fp64(false, S, ws.s_hits.as<HitRec>(), ws.total.as<uint32_t>(), drs + p,
                                                          Op[p], W, Q, nullptr, st);
                CK(cudaEventRecord(p2, st));
                launch_advance(ws.total.as<uint32_t>(), nullptr, s0, uint32_t(n), drs + p, st);
                CK(cudaGetLastError());
                out.gpu_launches += 6;  // scan (two kernels), sort (three), advance
                probe_ev.push_back({p0, p1});
                trace_ev.push_back({p1, p2});
                queued += n;
                sun_next[p] += n;
                out.batches++;
            }
        }
        CK(cudaMemcpyAsync(rs_h.data(), drs, K * sizeof(RunState), cudaMemcpyDeviceToHost, st));
        out.d2h_bytes += K * sizeof(RunState);
        CK(cudaStreamSynchronize(st));
        for (size_t p = 0; p < K; ++p) {
            if (reached[p]) continue;
            if (rs_h[p].reached) {
                reached[p] = true;
                --left;
            } else if (sun_next[p] > 0) {
                p_est[p] = std::max(double(rs_h[p].hits_done) / double(sun_next[p]), 1e-9);
            }
        }
    }
    CK(cudaEventRecord(t_last, st));
    CK(cudaStreamSynchronize(st));
    float ms = 0;
    cudaEventElapsedTime(&ms, t_first, t_last);
    out.device_ms = ms;
    for (auto &pe : probe_ev) {
        float x = 0;
        cudaEventElapsedTime(&x, pe.first, pe.second);
        out.probe_ms += x;
    }
    for (auto &pe : trace_ev) {
        float x = 0;
        cudaEventElapsedTime(&x, pe.first, pe.second);
        out.trace_ms += x;
    }
    std::vector<RunCounters> ctr(K);
    std::vector<unsigned long long> accv(K * acc_n);
    CK(cudaMemcpyAsync(ctr.data(), ws.pos_ctr.p, K * sizeof(RunCounters), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(accv.data(), ws.pos_acc.p, K * acc_n * 8, cudaMemcpyDeviceToHost, st));
    out.d2h_bytes += K * (sizeof(RunCounters) + acc_n * 8);
    CK(cudaStreamSynchronize(st));
    if (slot >= 0 && slot <= 1) ws.pos_dma_pending[slot] = false;
    out.pos.assign(K, PositionResult());
    for (size_t p = 0; p < K; ++p) {
        PositionResult &r = out.pos[p];
        r.sun_rays = pos[p].n_hits ? rs_h[p].sun_rays : 0;
        r.ray_hits = rs_h[p].hits_done;
        r.intersections = ctr[p].records;
        r.stage_entries.assign(ctr[p].stage_entries, ctr[p].stage_entries + nst);
        r.max_enter.assign(ctr[p].max_enter, ctr[p].max_enter + nst);
        const unsigned long long *a = accv.data() + p * acc_n;
        r.absorbed.assign(a + ne, a + 2 * ne);
        for (size_t m = 0; m < rq.flux.size(); ++m)
            r.flux.emplace_back(a + flux_off[m], a + flux_off[m] + map_size(rq.flux[m]));
    }
    if (rq.precision ? take_fe_failures_mixed() : take_fe_failures_fp64()) {
        out.error = "Interpolation failed to find nearby nodes to ray hit in FEA surface.";
        return false;
    }
    unsigned flags = 0;
    for (auto &c : ctr) flags |= c.flags;
    if (flags & kFlagBadInteraction) {
        out.error = "Bad optical interaction type (only 1 = refraction and 2 = reflection are traced)";
        return false;
    }
    out.ok = true;
    return true;
}

}  // namespace stb
