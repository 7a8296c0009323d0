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
    cudaError_t ensure(size_t b) {
        if (b <= bytes && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, b ? b : 16);
        if (e == cudaSuccess) bytes = b;
        return e;
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
    // trace state and queues (one slot per hit-list entry of a batch)
    DevBuf wf_sid, wf_raynum, wf_draw, wf_meta, wf_fe0, wf_p, wf_c, wf_q0, wf_q1, wf_qs, wf_counts;
    DevBuf save_rows[2], save_count, replay_rows, replay_fe0;  // stage-data save / replay
    DevBuf ecount, ecursor, etotal, s_sid, s_el, s_idx;
    std::vector<cudaEvent_t> events;
    // autotuned kernel variants per precision (FP64, mixed), chosen on the first run
    struct Tuning {
        bool done = false;
        int probe = 0;
    } tune[2];
    DevBuf tune_rs;
    ~Workspace() {
        if (device >= 0) cudaSetDevice(device);
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
        (e = ws.hit_mask.ensure(hit_mask_words(n) * 4)))
        return e;
    o = ProbeOut{};
    o.block_counts = ws.counts.as<uint32_t>();
    o.cand_count = ws.cand.as<uint32_t>();
    o.cand = o.cand_count + 1;
    o.cand_el = ws.cand_el.as<uint32_t>();
    o.hit_mask = ws.hit_mask.as<uint32_t>();
    return cudaSuccess;
}

// Autotuner: time every register-budget variant of the probe on the same 2^21 sun rays
// (indices 0.., outputs discarded into scratch buffers) and keep the fastest for this
// workspace and precision.  Variants share their arithmetic, so the choice changes
// timing only.
static cudaError_t autotune(Workspace &ws, const SceneDev &S0, int precision, uint64_t max_sun, cudaStream_t st,
                            int &launches) {
    Workspace::Tuning &tu = ws.tune[precision ? 1 : 0];
    const uint64_t n = std::min<uint64_t>(uint64_t(1) << 21, max_sun);
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
    for (const auto &f : rq.flux) {
        flux_off.push_back(acc_n);
        acc_n += size_t(f.nx) * f.ny;
    }
    if (rq.flux.size() > size_t(kMaxFluxMaps)) {
        out.error = "too many flux maps";
        return false;
    }
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, rq.device);

    const int nst = S.n_stages;
    const uint64_t kMaxBatch = uint64_t(1) << 26;
    DevBuf &d_acc = ws.acc, &d_ctr = ws.ctr, &d_rs = ws.rs, &d_rec_count = ws.rec_count, &d_offsets = ws.offsets,
           &d_total = ws.total, &d_recs = ws.recs;
    // the batch's hits are grouped by first-stage element (the rays of a warp then leave
    // one element and walk the same candidates)
    const uint32_t n_elem0 = uint32_t(S.stages[0].n_elem);
    DevBuf &d_ecount = ws.ecount, &d_ecursor = ws.ecursor, &d_etotal = ws.etotal, &d_s_sid = ws.s_sid,
           &d_s_el = ws.s_el, &d_s_idx = ws.s_idx;
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

    for (int attempt = 0; attempt < 4; ++attempt) {
        bool restart = false;
        out.records.clear();
        out.stage_entries.assign(nst, 0);
        out.max_enter.assign(nst, 0);
        out.max_ttmiss.assign(nst, 0);
        out.batches = 0;
        out.probe_ms = out.trace_ms = 0;
        CK(d_acc.ensure(std::max<size_t>(acc_n, 1) * 8));
        CK(d_ctr.ensure(sizeof(RunCounters)));
        CK(d_rs.ensure(sizeof(RunState)));
        CK(d_rec_count.ensure(8));
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
            if (rq.records) {
                if (rec_cap == 0) rec_cap = std::max<uint64_t>(n1, 1) * uint64_t(nst) * 2 + 4096;
                CK(d_recs.ensure(rec_cap * sizeof(RecordDev)));
                CK(cudaMemsetAsync(d_rec_count.p, 0, 8, st));
            }
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
                    launch_trace_mixed(rq.records, S, nullptr, nullptr, nullptr, nullptr, drs, O, W, Q, &rin, st);
            else
                out.gpu_launches +=
                    launch_trace_fp64(rq.records, S, nullptr, nullptr, nullptr, nullptr, drs, O, W, Q, &rin, st);
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
            if (nrec) {
                out.records.resize(nrec);
                out.d2h_bytes += nrec * sizeof(RecordDev);
                CK(cudaMemcpy(out.records.data(), d_recs.p, nrec * sizeof(RecordDev), cudaMemcpyDeviceToHost));
            }
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
                const uint64_t need = rq.n_hits - rs.hits_done;
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
                const uint64_t n = std::min<uint64_t>(kMaxBatch, want - queued);
                const uint32_t nb = uint32_t((n + kProbeBlock - 1) / kProbeBlock);
                ProbeOut po;
                CK(probe_buffers(ws, n, po));
                CK(d_offsets.ensure(size_t(nb) * 4));
                CK(ws.scan_parts.ensure(scan_parts(nb) * 4));
                CK(d_total.ensure(8));
                CK(d_s_sid.ensure(n * 8));
                CK(d_s_el.ensure(n * 4));
                CK(d_s_idx.ensure(n * 4));
                if (rq.records) {
                    if (rec_cap == 0) rec_cap = std::min<uint64_t>(n, uint64_t(1) << 22) * uint64_t(nst) * 2 + 4096;
                    CK(d_recs.ensure(rec_cap * sizeof(RecordDev)));
                    CK(cudaMemsetAsync(d_rec_count.p, 0, 8, st));
                }
                O.recs = rq.records ? d_recs.as<RecordDev>() : nullptr;
                O.rec_cap = rq.records ? rec_cap : 0;
                cudaEvent_t p0 = new_event(), p1 = new_event(), p2 = new_event();
                CK(cudaEventRecord(p0, st));
                if (rq.precision)
                    out.gpu_launches += launch_probe_mixed(S, sun_next, uint32_t(n), po, drs, tu.probe, st);
                else
                    out.gpu_launches += launch_probe_fp64(S, sun_next, uint32_t(n), po, drs, tu.probe, st);
                launch_scan(po.block_counts, nb, d_offsets.as<uint32_t>(), d_total.as<uint32_t>(),
                            ws.scan_parts.as<uint32_t>(), st);
                launch_list_sort(sun_next, po, d_offsets.as<uint32_t>(), d_total.as<uint32_t>(), drs, n_elem0,
                                 d_ecount.as<uint32_t>(), d_ecursor.as<uint32_t>(), d_etotal.as<uint32_t>(),
                                 d_s_sid.as<uint64_t>(), d_s_el.as<uint32_t>(), d_s_idx.as<uint32_t>(), uint32_t(n), st);
                out.gpu_launches += 3;  // element counts, their scan, scatter
                const uint64_t *t_sid = d_s_sid.as<uint64_t>();
                const uint32_t *t_el = d_s_el.as<uint32_t>(), *t_idx = d_s_idx.as<uint32_t>();
                // trace state and queues: one slot per hit-list entry (at most n)
                WfState W;
                WfQueues Q;
                CK(wf_buffers(ws, S, n, W, Q));
                CK(save_setup(n));
                CK(cudaEventRecord(p1, st));
                if (rq.precision)
                    out.gpu_launches += launch_trace_mixed(rq.records, S, t_sid, t_el, t_idx, d_total.as<uint32_t>(),
                                                           drs, O, W, Q, nullptr, st);
                else
                    out.gpu_launches += launch_trace_fp64(rq.records, S, t_sid, t_el, t_idx, d_total.as<uint32_t>(),
                                                          drs, O, W, Q, nullptr, st);
                CK(cudaEventRecord(p2, st));
                launch_advance(d_total.as<uint32_t>(), nullptr, sun_next, uint32_t(n), drs, st);
                CK(cudaGetLastError());
                out.gpu_launches += 3;  // scan (two kernels), advance
                probe_ev.push_back({p0, p1});
                trace_ev.push_back({p1, p2});
                queued += n;
                sun_next += n;
                out.batches++;
                if (sync_each) {
                    CK(cudaMemcpyAsync(&rs, drs, sizeof rs, cudaMemcpyDeviceToHost, st));
                    out.d2h_bytes += sizeof rs;
                    unsigned long long nrec = 0;
                    if (rq.records) CK(cudaMemcpyAsync(&nrec, d_rec_count.p, 8, cudaMemcpyDeviceToHost, st));
                    CK(cudaStreamSynchronize(st));
                    if (rq.records && nrec > rec_cap) {
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
                    if (nrec) {
                        const auto tr = std::chrono::steady_clock::now();
                        const size_t old = out.records.size();
                        out.records.resize(old + nrec);
                        out.d2h_bytes += nrec * sizeof(RecordDev);
                        CK(cudaMemcpyAsync(out.records.data() + old, d_recs.p, nrec * sizeof(RecordDev),
                                           cudaMemcpyDeviceToHost, st));
                        CK(cudaStreamSynchronize(st));
                        out.readback_ms += ms_since(tr);
                    }
                    if (rq.callback &&
                        !rq.callback((unsigned long)rs.sun_rays, (unsigned long)rs.hits_done,
                                     (unsigned long)(explicit_mode ? n_explicit : rq.n_hits), 1ul, (unsigned long)nst,
                                     rq.cbdata)) {
                        out.cancelled = true;
                        done = true;
                        break;
                    }
                    if (rs.reached) break;
                }
            }
            if (restart) break;
            CK(cudaMemcpyAsync(&rs, drs, sizeof rs, cudaMemcpyDeviceToHost, st));
            out.d2h_bytes += sizeof rs;
            CK(cudaStreamSynchronize(st));
            if (rs.reached || out.cancelled || (explicit_mode && sun_next >= n_explicit)) done = true;
            if (!explicit_mode && sun_next > 0) p_est = std::max(double(rs.hits_done) / double(sun_next), 1e-9);
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
        out.ray_hits = rs.hits_done;
        out.sun_rays = explicit_mode ? n_explicit : rs.sun_rays;
        if (!explicit_mode && !rs.reached && !out.cancelled) {
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
            out.flux.emplace_back(accv.begin() + flux_off[m],
                                  accv.begin() + flux_off[m] + size_t(rq.flux[m].nx) * rq.flux[m].ny);
        out.readback_ms += ms_since(tr);
        if (rq.precision ? take_fe_failures_mixed() : take_fe_failures_fp64()) {
            // the reference throws at such a query (vshot.cpp:177-178) and returns no result
            out.error = "Interpolation failed to find nearby nodes to ray hit in FEA surface.";
            return false;
        }
        if (out.flags & kFlagBadInteraction) {
            out.error = "Bad optical interaction type (only 1 = refraction and 2 = reflection are traced)";
            return false;
        }
        out.ok = true;
        return true;
    }
    out.error = "record buffer could not be sized for this run";
    return false;
}

}  // namespace stb
