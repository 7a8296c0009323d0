// Trace kernels of the B200 SolTrace path.
//
// A run is a sequence of sun-ray batches.  Per batch:
//   k_probe   one thread per sun ray: generate it (generateray.cpp:58-161), find the
//             nearest first-stage element it hits (raytrace.cpp:653-770), write the
//             element (0 = miss) per ray and a per-block hit count;
//   k_offsets single block: exclusive scan of the block counts;
//   k_compact one thread per sun ray: ordered list of the rays that hit (their sun
//             index and element), i.e. the reference's ray numbering, in which only
//             first-stage hits consume a number (raytrace.cpp:780-798);
//   k_trace   one thread per numbered ray: the rest of the per-ray state machine of
//             raytrace.cpp:582-1040 through every stage, writing records, flux bins
//             and counters.
// Splitting off the probe keeps the trace kernel's warps full: the sun rays that
// miss everything (most of them on a heliostat field) never enter it.
#pragma once
#include <climits>
#include "st_device.cuh"
#include "st_launch.h"

namespace stb {

constexpr int kMaxHitsPerStage = 100000;  // the reference has no bound; a ray trapped between
                                          // mirrors would loop forever there

// ------------------------------------------------------------------------------------
// sun ray / explicit ray generation
// ------------------------------------------------------------------------------------
__device__ __forceinline__ void make_ray(const SceneDev &S, uint64_t sid, RayRng &rng, double pg[3], double cg[3],
                                         double &xs, double &ys) {
    const SunDev &sun = S.sun;
    if (S.explicit_rays) {
        for (int q = 0; q < 3; ++q) {
            pg[q] = S.ex_pos[3 * sid + q];
            cg[q] = S.ex_cos[3 * sid + q];
        }
        xs = ys = 0.0;
        return;
    }
    if (sun.point_source) {  // generateray.cpp:101-133
        for (int q = 0; q < 3; ++q) pg[q] = sun.origin[q];
        for (int q = 0; q < 3; ++q) {
            const double sg = (rng.u() <= 0.5) ? -1.0 : 1.0;
            cg[q] = sg * rng.u();
        }
        const double m = sqrt(cg[0] * cg[0] + cg[1] * cg[1] + cg[2] * cg[2]);
        for (int q = 0; q < 3; ++q) cg[q] = cg[q] / m;
        xs = ys = 0.0;
        return;
    }
    xs = sun.xmin + (sun.xmax - sun.xmin) * rng.u();
    ys = sun.ymin + (sun.ymax - sun.ymin) * rng.u();
    const double psun[3] = {xs, ys, -10000.0}, csun[3] = {0.0, 0.0, 1.0};
    double pst[3], cst[3];
    to_ref(sun.Rsun, sun.pos_sun_stage, psun, csun, pst, cst);
    to_ref(S.stages[0].R, S.stages[0].o, pst, cst, pg, cg);
}

// ------------------------------------------------------------------------------------
// nearest accepted hit in a stage (raytrace.cpp:698-770); -1 if none
// ------------------------------------------------------------------------------------
// element_test without the full hit.  ET (element-test mode): 0 any element, kEtFlat the
// element is known to be flat, kEtClosed its surface is known to be closed-form
constexpr int kEtFlat = 1, kEtClosed = 2;
template <int MIXED, int ET>
__device__ __forceinline__ bool elem_hit(const SceneDev &S, const ElemRec &e, const double ps[3], const double cs[3],
                                         double &pl) {
    if (ET == kEtFlat) return element_test_flat<MIXED>(e, ps, cs, pl);
    return element_test<MIXED, ET == kEtClosed ? 1 : 0>(S, e, ps, cs, pl, nullptr);
}

template <int MIXED, int ET = 0>
__device__ inline int nearest_brute(const SceneDev &S, const StageRec &st, const double ps[3], const double cs[3]) {
    int best = -1;
    double bp = 1e99;
    for (int j = 0; j < st.n_elem; ++j) {
        const ElemRec &e = S.elems[st.first_elem + j];
        if (!e.enabled) continue;
        double pl;
        if (elem_hit<MIXED, ET>(S, e, ps, cs, pl) && pl < bp) {
            bp = pl;
            best = j;
        }
    }
    return best;
}

// BVH over element bounding spheres; nodes farther than the best hit so far are
// skipped (the test is on the entry distance minus the 1e-5 nudge, with slack for
// the float box arithmetic).
template <int MIXED, int ET = 0>
__device__ inline int nearest_bvh(const SceneDev &S, const StageRec &st, const double ps[3], const double cs[3],
                                  int from) {
    const BvhNode *nodes = S.bvh + st.bvh_off;
    const int *items = S.bvh_items + st.bvh_items_off;
    const float ox = float(ps[0]), oy = float(ps[1]), oz = float(ps[2]);
    const float dx = float(cs[0]), dy = float(cs[1]), dz = float(cs[2]);
    // 1/d with zero components replaced by a tiny signed value, so slab products are never 0*inf
    const float ix = 1.0f / (fabsf(dx) > 1e-30f ? dx : copysignf(1e-30f, dx));
    const float iy = 1.0f / (fabsf(dy) > 1e-30f ? dy : copysignf(1e-30f, dy));
    const float iz = 1.0f / (fabsf(dz) > 1e-30f ? dz : copysignf(1e-30f, dz));
    int stack[48];
    int sp = 0;
    stack[sp++] = 0;
    int best = -1;
    double bp = 1e99;
    while (sp > 0) {
        const BvhNode nd = nodes[stack[--sp]];
        float t0x = (nd.lo[0] - ox) * ix, t1x = (nd.hi[0] - ox) * ix;
        float t0y = (nd.lo[1] - oy) * iy, t1y = (nd.hi[1] - oy) * iy;
        float t0z = (nd.lo[2] - oz) * iz, t1z = (nd.hi[2] - oz) * iz;
        const float tmin = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fminf(t0z, t1z));
        const float tmax = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fmaxf(t0z, t1z));
        // NaN-safe: a NaN slab (origin on a face of a zero-width box) keeps the node
        if (tmax < 0.0f || tmin > tmax) continue;
        if (double(tmin) > bp * (1.0 + 1e-6) + 1e-3) continue;
        if (nd.count > 0) {
            for (int k = 0; k < nd.count; ++k) {
                const int j = items[nd.first + k];
                // the flat element the ray is leaving, when its test certainly fails
                if (j == from) continue;
                // float pre-test against the element's bounding sphere: the sphere must reach
                // the ray ahead of its origin.  The radius is padded for the float rounding of
                // centre, origin and direction (2e-6 of the L1 norms, over ten times the bound).
                const float4 bs = S.elem_sphere[st.first_elem + j];
                const float vx = bs.x - ox, vy = bs.y - oy, vz = bs.z - oz;
                const float tc = vx * dx + vy * dy + vz * dz;
                const float wx = vx - tc * dx, wy = vy - tc * dy, wz = vz - tc * dz;
                const float rr = bs.w + 2e-6f * (fabsf(ox) + fabsf(oy) + fabsf(oz) + fabsf(vx) + fabsf(vy) + fabsf(vz));
                if (tc < -rr || wx * wx + wy * wy + wz * wz > rr * rr) continue;
                const ElemRec &e = S.elems[st.first_elem + j];
                if (!e.enabled) continue;
                double pl;
                if (elem_hit<MIXED, ET>(S, e, ps, cs, pl) && (pl < bp || (pl == bp && j < best))) {
                    bp = pl;
                    best = j;
                }
            }
        } else if (sp + 2 <= 48) {
            stack[sp++] = nd.first + 1;
            stack[sp++] = nd.first;
        }
    }
    return best;
}

// Nearest element through the stage's ground grid (or, for a ray leaving a flat first-stage
// element within its outgoing beam, through that element's beam list: see
// build_beam_lists in st_host.cpp): a 2-D DDA walk over the cells the ray
// crosses inside the stage's z band, in order of distance.  Entries pass a float test
// against their padded bounding sphere; the few that pass are collected and given the
// double-precision element test after the walk (or when the list fills, after which the
// walk stops at the first cell beyond the nearest hit).  Every element a hit can come
// from is listed in a visited cell (the padded discs absorb the float rounding of the
// walk), and the choice among hits is the serial search's (shortest path, lower index on
// ties), so the result is the brute-force search's.
template <int MIXED, int ET = 0>
__device__ inline int nearest_grid(const SceneDev &S, const StageRec &st, const double ps[3], const double cs[3],
                                   int from) {
    const float ox = float(ps[0]), oy = float(ps[1]), oz = float(ps[2]);
    const float dx = float(cs[0]), dy = float(cs[1]), dz = float(cs[2]);
    // a ray leaving a flat element within its outgoing beam: that element's list stands in
    // for the walk (one pass of the loop below over the list)
    int2 list = make_int2(0, 0);
    bool list_mode = false;
    if (from >= 0 && S.beam_axis) {
        const float4 ax = S.beam_axis[st.first_elem + from];
        if (dx * ax.x + dy * ax.y + dz * ax.z >= ax.w) {
            list_mode = true;
            list = S.beam_range[st.first_elem + from];
        }
    }
    // clip to the z band and the grid box
    float t0 = 0.0f, t1 = 3.0e38f;
    auto clip = [&](float o, float d, float lo, float hi) {
        if (fabsf(d) > 1e-30f) {
            const float a = (lo - o) / d, b = (hi - o) / d;
            t0 = fmaxf(t0, fminf(a, b));
            t1 = fminf(t1, fmaxf(a, b));
        } else if (o < lo || o > hi) {
            t1 = -1.0f;
        }
    };
    if (!list_mode) {
        clip(oz, dz, st.gzlo, st.gzhi);
        clip(ox, dx, st.gx0, st.gx0 + st.gnx * st.gcell);
        clip(oy, dy, st.gy0, st.gy0 + st.gny * st.gcell);
        if (!(t0 <= t1)) return -1;
    }
    const float px = ox + t0 * dx, py = oy + t0 * dy;
    int ix = min(max(int(floorf((px - st.gx0) * st.ginv)), 0), st.gnx - 1);
    int iy = min(max(int(floorf((py - st.gy0) * st.ginv)), 0), st.gny - 1);
    const int sx = dx > 0.0f ? 1 : -1, sy = dy > 0.0f ? 1 : -1;
    const float inf = 3.0e38f;
    float tmx = fabsf(dx) > 1e-30f ? (st.gx0 + (ix + (dx > 0.0f)) * st.gcell - ox) / dx : inf;
    float tmy = fabsf(dy) > 1e-30f ? (st.gy0 + (iy + (dy > 0.0f)) * st.gcell - oy) / dy : inf;
    const float tdx = fabsf(dx) > 1e-30f ? st.gcell / fabsf(dx) : inf;
    const float tdy = fabsf(dy) > 1e-30f ? st.gcell / fabsf(dy) : inf;
    const int2 *cells = S.stage_cells + st.gcell_off;
    const float pad_o = 2e-6f * (fabsf(ox) + fabsf(oy) + fabsf(oz));
    int best = -1;
    double bp = 1e99;
    // the candidate list lives in shared memory, [slot][thread] (blocks have at most 256
    // threads), so that it neither takes registers nor goes to local memory
    constexpr int kCand = 8;
    __shared__ int cand_sh[kCand * 256];
    int *cand = cand_sh + threadIdx.x;
    int nc = 0;
    auto flush = [&]() {
        for (int c = 0; c < nc; ++c) {
            const int j = cand[256 * c];
            double pl;
            if (elem_hit<MIXED, ET>(S, S.elems[st.first_elem + j], ps, cs, pl) &&
                (pl < bp || (pl == bp && j < best))) {
                bp = pl;
                best = j;
            }
        }
        nc = 0;
    };
    int seen1 = -1, seen2 = -1, seen3 = -1;
    float tin = t0;
    for (;;) {
        if (best >= 0 && double(tin) > bp * (1.0 + 1e-6) + 1e-3) break;
        const int2 range = list_mode ? list : cells[iy * st.gnx + ix];
        for (int k = range.x; k < range.y; ++k) {
            const float4 bs = list_mode ? S.elem_sphere[st.first_elem + S.beam_elem[k]] : S.grid_sphere[k];
            const float vx = bs.x - ox, vy = bs.y - oy, vz = bs.z - oz;
            const float tc = vx * dx + vy * dy + vz * dz;
            const float wx = vx - tc * dx, wy = vy - tc * dy, wz = vz - tc * dz;
            // radius padded for the float rounding of centre, origin and direction
            const float rr = bs.w + pad_o + 2e-6f * (fabsf(vx) + fabsf(vy) + fabsf(vz));
            if (tc < -rr || wx * wx + wy * wy + wz * wz > rr * rr) continue;
            const int j = list_mode ? S.beam_elem[k] : S.grid_elem[k];
            // the element the ray is leaving (when it certainly cannot be met again), and
            // elements already collected from the last cells
            if (j == from || j == seen1 || j == seen2 || j == seen3) continue;
            seen3 = seen2;
            seen2 = seen1;
            seen1 = j;
            if (nc == kCand) flush();
            cand[256 * nc++] = j;
        }
        if (list_mode) break;
        // step to the next cell along the ray
        if (tmx < tmy) {
            tin = tmx;
            ix += sx;
            tmx += tdx;
            if (ix < 0 || ix >= st.gnx) break;
        } else {
            tin = tmy;
            iy += sy;
            tmy += tdy;
            if (iy < 0 || iy >= st.gny) break;
        }
        if (tin > t1) break;
    }
    flush();
    return best;
}

template <int MIXED>
__device__ __forceinline__ int nearest(const SceneDev &S, const StageRec &st, const double ps[3], const double cs[3],
                                       int from = -1) {
    if (st.grid_on) return nearest_grid<MIXED>(S, st, ps, cs, from);
    return (st.bvh_off >= 0) ? nearest_bvh<MIXED>(S, st, ps, cs, from) : nearest_brute<MIXED>(S, st, ps, cs);
}

// nearest element with the code of search kind KIND only (stage_search_kind, st_launch.h)
template <int MIXED, int KIND>
__device__ __forceinline__ int nearest_kind(const SceneDev &S, const StageRec &st, const double ps[3],
                                            const double cs[3], int from) {
    constexpr int ET = (KIND & kSearchFlat) ? kEtFlat : (KIND & kSearchClosed) ? kEtClosed : 0;
    if (KIND & kSearchBrute) return nearest_brute<MIXED, ET>(S, st, ps, cs);
    if (st.grid_on) return nearest_grid<MIXED, ET>(S, st, ps, cs, from);
    return (st.bvh_off >= 0) ? nearest_bvh<MIXED, ET>(S, st, ps, cs, from) : nearest_brute<MIXED, ET>(S, st, ps, cs);
}

// first test of a first-stage sun ray through the sun-plane grid (cells list the
// elements, ascending, whose bounding disc in the sun plane overlaps the cell)
// The first-stage ray of sun-frame point (xs, ys), as the reference builds it: sun frame ->
// stage -> global (generateray.cpp:151-159), then global -> stage (raytrace.cpp:625-627).
__device__ __forceinline__ void sun_ray_in_stage(const SceneDev &S, double xs, double ys, double ps[3], double cs[3]) {
    const SunDev &sun = S.sun;
    const StageRec &st = S.stages[0];
    const double psun[3] = {xs, ys, -10000.0}, csun[3] = {0.0, 0.0, 1.0};
    double pst[3], cst[3], pg[3], cg[3];
    to_ref(sun.Rsun, sun.pos_sun_stage, psun, csun, pst, cst);
    to_ref(st.R, st.o, pst, cst, pg, cg);
    to_local(st.R, st.o, pg, cg, ps, cs);
}

// Float pre-test of sun-plane point (fx, fy) against grid entry k: inside the padded disc
// and the padded footprint parallelogram (both contain every point whose ray the element
// can accept, so a rejected entry is one the double-precision test rejects too).
__device__ __forceinline__ bool sun_entry_pass(const SunDev &sun, int k, float fx, float fy) {
    const float4 d = sun.cell_disc[k];
    const float qx = fx - d.x, qy = fy - d.y;
    if (qx * qx + qy * qy > d.z * d.z) return false;
    const float4 p = sun.cell_par[k];
    return fabsf(p.x * qx + p.y * qy) <= 1.0f && fabsf(p.z * qx + p.w * qy) <= 1.0f;
}

// Cell of the sun-plane grid holding point (xs, ys): its entry range [x, y).
__device__ __forceinline__ int2 sun_cell(const SunDev &sun, double xs, double ys) {
    int cx = int(floor((xs - sun.gx0) * sun.ginv)), cy = int(floor((ys - sun.gy0) * sun.ginv));
    cx = min(max(cx, 0), sun.gnx - 1);
    cy = min(max(cy, 0), sun.gny - 1);
    return reinterpret_cast<const int2 *>(sun.cell_start)[cy * sun.gnx + cx];
}

// Sun-ray probe through the grid for one ray; the double-precision ray is built only once
// a cell entry passes the float pre-test.
template <int MIXED, int ET = 0>
__device__ inline int nearest_sun_grid_lazy(const SceneDev &S, const StageRec &st, double xs, double ys) {
    const SunDev &sun = S.sun;
    const int2 range = sun_cell(sun, xs, ys);
    int best = -1;
    double bp = 1e99;
    const float fx = float(xs), fy = float(ys);
    bool have_ray = false;
    double ps[3], cs[3];
    for (int k = range.x; k < range.y; ++k) {
        if (!sun_entry_pass(sun, k, fx, fy)) continue;
        const int j = __float_as_int(sun.cell_disc[k].w);
        const ElemRec &e = S.elems[st.first_elem + j];
        if (!e.enabled) continue;
        if (!have_ray) {
            sun_ray_in_stage(S, xs, ys, ps, cs);
            have_ray = true;
        }
        double pl;
        if (elem_hit<MIXED, ET>(S, e, ps, cs, pl) && pl < bp) {
            bp = pl;
            best = j;
        }
    }
    return best;
}


// ------------------------------------------------------------------------------------
// optics (raytrace.cpp:885-946 test value; interaction.cpp:58-199)
// ------------------------------------------------------------------------------------
template <int MIXED>
__device__ inline double test_value(const SceneDev &S, const OpticRec &op, int type, const double cin[3], const double n[3]) {
    const int off = (type == 1) ? op.trans_tab_off : op.refl_tab_off;
    const int np = (type == 1) ? op.trans_tab_n : op.refl_tab_n;
    if (np <= 0) return (type == 1) ? op.trans : op.refl;
    const double *tab = S.tables + off;  // (angle, value) pairs
    double ia;
    if (MIXED) {
        const float nn = sqrtf(float(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]));
        const float c = -(float(cin[0]) * float(n[0]) + float(cin[1]) * float(n[1]) + float(cin[2]) * float(n[2])) / nn;
        ia = double(acosf(fminf(fmaxf(c, -1.f), 1.f)) * 1000.f);
    } else {
        const double nn = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        const double un[3] = {-n[0] / nn, -n[1] / nn, -n[2] / nn};
        ia = acos(cin[0] * un[0] + cin[1] * un[1] + cin[2] * un[2]) * 1000.;
    }
    if (ia >= tab[2 * (np - 1)]) return tab[2 * (np - 1) + 1];
    int m = 0;
    while (m < np - 1 && tab[2 * m] < ia) m++;
    if (m == 0) return tab[1];
    return (tab[2 * m + 1] + tab[2 * (m - 1) + 1]) / 2.0;
}

__device__ __forceinline__ void reflect(const double cin[3], const double n[3], double out[3]) {
    const double a = (cin[0] * n[0] + cin[1] * n[1] + cin[2] * n[2]) / (n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    for (int q = 0; q < 3; ++q) out[q] = cin[q] - 2.0 * a * n[q];
}

// refraction with an unpolarised Fresnel split; a non-converged Newton leaves the
// incoming direction (the reference leaves the previous output untouched)
template <int MIXED>
__device__ inline void refract(const OpticRec &op, const double cin[3], const double n[3], RayRng &rng, double out[3]) {
    const double r1 = op.n_in, r2 = op.n_out;
    const double mu = r1 / r2;
    const double d2 = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
    const double B = (mu * mu - 1.0) / d2;
    const double A = mu * (cin[0] * n[0] + cin[1] * n[1] + cin[2] * n[2]) / d2;
    if (B > A * A) {  // total internal reflection
        reflect(cin, n, out);
        return;
    }
    double rave;
    if (MIXED) {
        const float nn = sqrtf(float(d2));
        const float c = -(float(cin[0]) * float(n[0]) + float(cin[1]) * float(n[1]) + float(cin[2]) * float(n[2])) / nn;
        const float ia = acosf(fminf(fmaxf(c, -1.f), 1.f));
        const float f1 = float(r1), f2 = float(r2);
        const float st = f1 * sinf(ia) / f2, ct = sqrtf(1.f - st * st), ci = cosf(ia);
        const float rs = (f1 * ci - f2 * ct) / (f1 * ci + f2 * ct), rp = (f1 * ct - f2 * ci) / (f1 * ct + f2 * ci);
        rave = double((rp * rp + rs * rs) / 2.f);
    } else {
        const double nn = sqrt(d2);
        const double un[3] = {-n[0] / nn, -n[1] / nn, -n[2] / nn};
        const double ia = acos(cin[0] * un[0] + cin[1] * un[1] + cin[2] * un[2]);
        const double st = r1 * sin(ia) / r2, ct = sqrt(1 - st * st);
        const double rsn = r1 * cos(ia) - r2 * ct, rsd = r1 * cos(ia) + r2 * ct;
        const double rpn = r1 * ct - r2 * cos(ia), rpd = r1 * ct + r2 * cos(ia);
        rave = ((rpn / rpd) * (rpn / rpd) + (rsn / rsd) * (rsn / rsd)) / 2.0;
    }
    if (rave < rng.u()) {
        double g = -B / (2.0 * A), g1 = g;
        bool ok = false;
        for (int i = 1; i < 10; ++i) {
            g1 = (g * g - B) / (2.0 * (g + A));
            if (fabs(g - g1) < 0.000005) {
                ok = true;
                break;
            }
            g = g1;
        }
        if (!ok) {
            for (int q = 0; q < 3; ++q) out[q] = cin[q];
            return;
        }
        for (int q = 0; q < 3; ++q) out[q] = mu * cin[q] + g1 * n[q];
    } else {
        reflect(cin, n, out);
    }
}

// error sample about `axis` (sunshape: source 1; specularity: source 2 with the
// reflection re-draw of errors.cpp:222-225)
template <int MIXED>
__device__ inline void error_sample(const SceneDev &S, int dist, double delop, const double axis[3], RayRng &rng,
                                    bool redraw_below, const double nrm[3], double out[3]) {
    // mixed precision: a Gaussian or pillbox spread of zero (a perfectly specular mirror)
    // leaves the axis unchanged; its two draws are skipped rather than generated, so the
    // ray's later draws stay where they are
    if (MIXED && delop == 0.0 && (dist == 'g' || dist == 'G' || dist == 'p' || dist == 'P')) {
        rng.k += 2;
        for (int q = 0; q < 3; ++q) out[q] = axis[q];
        return;
    }
    for (unsigned call = 0;; ++call) {
        const double ut = rng.u();
        const double up = rng.u();
        if (MIXED) {
            perturb<float>(axis, sample_theta_f(dist, float(delop), ut, S.sun), float(up) * 6.2831853f, out);
        } else {
            perturb<double>(axis, sample_theta(dist, delop, ut, S.sun), up * 2.0 * 3.1415926535897932385, out);
        }
        if (!(redraw_below && out[0] * nrm[0] + out[1] * nrm[1] + out[2] * nrm[2] < 0 && call < 50000)) break;
    }
}

// ------------------------------------------------------------------------------------
// record, flux and counter output
// ------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long warp_reserve(unsigned long long *counter) {
    const unsigned mask = __activemask();
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    const unsigned rank = __popc(mask & ((1u << lane) - 1u));
    unsigned long long base = 0;
    if (lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + rank;
}

// add 1 to base[idx] for every active lane, one atomic per distinct idx in the warp (the
// trace's warps mostly carry rays of one element, so their counters coincide)
__device__ __forceinline__ void warp_count(unsigned long long *base, int idx) {
    const unsigned mask = __activemask();
    const unsigned peers = __match_any_sync(mask, idx);
    if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&base[idx], (unsigned long long)__popc(peers));
}

// Bin of value v on n bins of width b from vmin, by the GUI's rule: the smallest g >= -1
// with vmin + (g + 1) b >= v (app/src/project.cpp:1392-1396; bins are (lower, upper]);
// -1 when v is outside.
__host__ __device__ inline int gui_bin(double v, double vmin, double b, int n) {
    const double q = (v - vmin) / b;
    if (!(q > -1.0) || !(q <= double(n) + 1.0)) return -1;  // outside (and NaN)
    int g = int(ceil(q)) - 1;
    if (g < -1) g = -1;
    while (g + 1 <= n && vmin + (g + 1) * b < v) ++g;
    while (g >= 0 && !(vmin + g * b < v)) --g;
    return (g >= 0 && g < n) ? g : -1;
}

// The GUI's unwrapped arc length of a point on a full cylinder of radius R about the local
// y axis (app/src/project.cpp:1370-1378).
__host__ __device__ inline double gui_cyl_arc(double x, double z, double R) {
    if (z <= R) return R * asin(x / R);
    return (x < 0) ? -(kPiD * R / 2.0 + R * acos(fabs(x) / R)) : kPiD * R / 2.0 + R * acos(x / R);
}

// Value k of numpy.arange(start, stop, step) as numpy fills it: start, start + step, then
// start + k ((start + step) - start).
__host__ __device__ inline double arange_value(double start, double step, int k) {
    if (k == 0) return start;
    const double v1 = start + step;
    return k == 1 ? v1 : start + double(k) * (v1 - start);
}

// Node i (ascending) of the cell-centre mesh of n cells over a span S centred on 0, built as
// the trough example's create_polar_mesh_cyl builds it
// (app/deploy/api/examples/parabolic-trough-tracking-timeseries/st_processing_functions.py:
// 174-204): even n: +-(d/2 + k d), odd n: 0, +-k d, with d = S / n.
__host__ __device__ inline double mesh_node(int i, int n, double S) {
    const double d = S / n;
    if (n % 2 == 0) {
        const int m = n / 2;
        return i < m ? -arange_value(0.0 + d / 2, d, m - 1 - i) : arange_value(0.0 + d / 2, d, i - m);
    }
    const int m = (n + 1) / 2;
    return i < m - 1 ? -arange_value(0.0, d, m - 1 - i) : arange_value(0.0, d, i - (m - 1));
}

// The node nearest to v, the first of equals (numpy.argmin of |node - v|, the example's
// compute_fluxmap, st_processing_functions.py:245-250); every finite v has one.  The nodes are
// d apart up to rounding, so the nearest is within one of the estimate: the five around it
// are compared in order.  -1 for NaN.
__host__ __device__ inline int mesh_nearest(double v, int n, double S) {
    if (!(v == v)) return -1;
    const double est = v / (S / n) + 0.5 * (n - 1);
    const int i0 = !(est > 0.0) ? 0 : (est >= double(n - 1) ? n - 1 : int(est + 0.5));
    int best = -1;
    double bd = 0.0;
    for (int i = (i0 > 2 ? i0 - 2 : 0); i <= (i0 + 2 < n - 1 ? i0 + 2 : n - 1); ++i) {
        const double dd = fabs(mesh_node(i, n, S) - v);
        if (best < 0 || dd < bd) {
            best = i;
            bd = dd;
        }
    }
    return best;
}

// fe0: the ray's first first-stage element (global index, first stage first; -1 none), which
// selects the map of a per-source flux map
template <int MIXED>
__device__ inline void bin_flux(const SceneDev &S, int si, int ej, bool absorbed, const double pe[3], int fe0) {
    for (int m = 0; m < S.n_flux; ++m) {
        const FluxMapDev &f = S.flux[m];
        if (f.stage != si || f.elem != ej) continue;
        if (f.absorbed_only && !absorbed) continue;
        if (f.n_src > 0 && (fe0 < 0 || fe0 >= f.n_src)) continue;
        int ix, iy;
        if (f.kind >= 2) {  // the GUI's statistics rules, in double
            if (f.kind == 4) {  // nearest node of the tube's polar mesh: arc r atan2(x, z - r) by y
                const double R = f.x1;
                ix = mesh_nearest(R * atan2(pe[0], pe[2] - R), f.nx, kPiD * (2.0 * R));
                iy = mesh_nearest(pe[1] - 0.5 * (f.y0 + f.y1), f.ny, f.y1 - f.y0);
            } else {
                if (f.kind == 2) {
                    ix = gui_bin(pe[0], f.x0, (f.x1 - f.x0) / f.nx, f.nx);
                } else {
                    const double R = f.x1;
                    ix = gui_bin(gui_cyl_arc(pe[0], pe[2], R), -kPiD * R, 2.0 * kPiD * R / f.nx, f.nx);
                }
                iy = gui_bin(pe[1], f.y0, (f.y1 - f.y0) / f.ny, f.ny);
            }
        } else if (MIXED) {
            float u, u0, u1;
            if (f.kind == 0) {
                u = float(pe[0]);
                u0 = float(f.x0);
                u1 = float(f.x1);
            } else {
                u = atan2f(float(pe[0]), float(pe[2] - f.x1)) + 3.14159265f;
                u0 = 0.f;
                u1 = 6.28318531f;
            }
            ix = int(floorf((u - u0) / (u1 - u0) * f.nx));
            iy = int(floorf(float((pe[1] - f.y0) / (f.y1 - f.y0)) * f.ny));
        } else {
            double u, u0, u1;
            if (f.kind == 0) {
                u = pe[0];
                u0 = f.x0;
                u1 = f.x1;
            } else {
                u = atan2(pe[0], pe[2] - f.x1) + kPiD;
                u0 = 0.0;
                u1 = 2.0 * kPiD;
            }
            const double dx = floor((u - u0) / (u1 - u0) * f.nx), dy = floor((pe[1] - f.y0) / (f.y1 - f.y0) * f.ny);
            if (dx < 0 || dx >= f.nx || dy < 0 || dy >= f.ny) continue;
            ix = int(dx);
            iy = int(dy);
        }
        if (ix < 0 || ix >= f.nx || iy < 0 || iy >= f.ny) continue;
        const size_t src = f.n_src > 0 ? size_t(fe0) * size_t(f.nx) * size_t(f.ny) : 0;
        // one atomic per distinct bin among the warp's lanes here: a focusing optic sends most
        // rays of a warp into a few bins, whose single-address atomics would serialise
        unsigned long long *bin = &f.bins[src + size_t(iy) * f.nx + ix];
        const unsigned active = __activemask();
        const unsigned peers = __match_any_sync(active, reinterpret_cast<unsigned long long>(bin));
        if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(bin, (unsigned long long)__popc(peers));
    }
}

// ------------------------------------------------------------------------------------
// kernels
// ------------------------------------------------------------------------------------
template <int MIXED>
__global__ void __launch_bounds__(kProbeBlock) k_probe(const __grid_constant__ SceneDev S, uint64_t s0, uint32_t n,
                                                        ProbeOut o, const RunState *rs) {
    const uint32_t i = blockIdx.x * kProbeBlock + threadIdx.x;
    const bool reached = rs->reached != 0;
    if (o.cand_count && blockIdx.x == 0 && threadIdx.x == 0) *o.cand_count = reached ? 0u : n;
    uint32_t h = 0;
    if (reached) {  // the requested hits are numbered: this batch is surplus
        if (threadIdx.x == 0) o.block_counts[blockIdx.x] = 0;
        return;
    }
    if (i < n) {
        RayRng rng;
        rng.init(S.seed, s0 + i, 0);
        double pg[3], cg[3], xs, ys;
        make_ray(S, s0 + i, rng, pg, cg, xs, ys);
        const StageRec &st = S.stages[0];
        double ps[3], cs[3];
        to_local(st.R, st.o, pg, cg, ps, cs);
        (void)xs;
        (void)ys;
        const int b = nearest<MIXED>(S, st, ps, cs);
        h = (b >= 0) ? uint32_t(b + 1) : 0u;
        if (o.hit_elem) o.hit_elem[i] = h;
        if (o.cand_el) {  // the list is every ray of the batch
            o.cand[i] = i;
            o.cand_el[i] = h;
        }
    }
    const unsigned bal = __ballot_sync(0xffffffffu, h != 0);
    if (o.hit_mask && (threadIdx.x & 31) == 0) o.hit_mask[i / 32] = bal;
    const int c = __syncthreads_count(h != 0);
    if (threadIdx.x == 0) o.block_counts[blockIdx.x] = uint32_t(c);
}

// Probe of generated sun rays on a first stage culled by the sun-plane grid, in two
// kernels so that the double-precision work runs in full warps:
//   k_sun_candidates (four sun rays per thread, few registers): draws the sun-plane point
//     and runs the float pre-tests of its grid cell; a ray with no passing entry is a miss,
//     the others are appended to a candidate list;
//   k_sun_resolve (one thread per listed ray): redraws the point and runs the serial
//     nearest-element search of the reference's loop over the first stage, writing the
//     result per list entry (and per ray, when asked), the ray's bit of the hit mask and
//     the per-kProbeBlock hit counts.
// On a heliostat field most sun rays miss every footprint and never reach the second
// kernel, whose warps are then fully occupied by rays that need the element tests.
template <int MIXED, int MINB, int FLAT>
__global__ void __launch_bounds__(kResolveBlock, MINB) k_sun_resolve(const __grid_constant__ SceneDev S, uint64_t s0,
                                                                     ProbeOut o, const RunState *rs) {
    if (rs->reached) return;
    const uint32_t nc = *o.cand_count;
    const SunDev &sun = S.sun;
    for (uint32_t c = blockIdx.x * kResolveBlock + threadIdx.x; c < nc; c += gridDim.x * kResolveBlock) {
        const uint32_t i = o.cand[c];
        RayRng rng;
        rng.init(S.seed, s0 + i, 0);
        const double xs = sun.xmin + (sun.xmax - sun.xmin) * rng.u();
        const double ys = sun.ymin + (sun.ymax - sun.ymin) * rng.u();
        const int b = nearest_sun_grid_lazy<MIXED, FLAT ? kEtFlat : 0>(S, S.stages[0], xs, ys);
        const uint32_t h = (b >= 0) ? uint32_t(b + 1) : 0u;
        if (o.hit_elem) o.hit_elem[i] = h;
        if (o.cand_el) o.cand_el[c] = h;
        if (b >= 0) {
            // one atomic per distinct count slot (and mask word) among the warp's hitting lanes
            const unsigned mask = __activemask();
            const uint32_t slot = i / kProbeBlock;
            const unsigned peers = __match_any_sync(mask, slot);
            if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&o.block_counts[slot], uint32_t(__popc(peers)));
            if (o.hit_mask) {
                const unsigned wp = __match_any_sync(mask, i / 32);
                const unsigned bits = __reduce_or_sync(wp, 1u << (i & 31));
                if ((threadIdx.x & 31) == __ffs(wp) - 1) atomicOr(&o.hit_mask[i / 32], bits);
            }
        }
    }
}

// Mixed-precision probe of sun rays on a first stage of flat rectangles (SunDev::exact_flat)
// in one kernel.  Each grid entry whose padded disc holds the sun-plane point is tested
// against the element's exact footprint and plane in float: inside the rectangle when
// |u|, |v| <= 1 for (u, v) the point in the projected half-axes' basis, at depth
// z0 + gx qx + gy qy along the sun's z (the nearest accepted element wins, as the path
// lengths of raytrace.cpp:745 order them).  A point within the float rounding margins of a
// footprint edge, an entry without an exact footprint, or two accepted elements within
// rounding of one depth leave the ray undecided: it goes to a list that k_sun_resolve_amb
// searches in double, so the element found is the FP64 probe's.  Output as k_sun_resolve
// leaves it: hitting rays listed with their element, one hit-mask bit per ray, hits per
// kProbeBlock rays.  RPT sun rays per thread at kProbeBlock apart (4, 8 or 16: the autotuner's
// variants), RPT x kProbeBlock per block.
template <int MIXED, int RPT>
__global__ void __launch_bounds__(kProbeBlock, kExactProbeMinBlocks) k_sun_probe_exact(const __grid_constant__ SceneDev S, uint64_t s0,
                                                                  uint32_t n, ProbeOut o, const RunState *rs) {
    const uint32_t nb = (n + kProbeBlock - 1) / kProbeBlock;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (rs->reached) {  // the requested hits are numbered: this batch is surplus
        if (threadIdx.x < RPT && blockIdx.x * RPT + threadIdx.x < nb)
            o.block_counts[blockIdx.x * RPT + threadIdx.x] = 0;
        if (o.hit_mask && threadIdx.x < (RPT * kProbeBlock) / 32) o.hit_mask[blockIdx.x * ((RPT * kProbeBlock) / 32) + threadIdx.x] = 0;
        return;
    }
    const SunDev &sun = S.sun;
    // per ray of the block its result, per warp and ray group the hit ballot
    constexpr uint32_t kUndecided = 0xffffffffu;
    __shared__ uint32_t hsh[RPT][kProbeBlock];
    __shared__ unsigned wb[RPT][kProbeBlock / 32];
    __shared__ uint32_t wn[kProbeBlock / 32], base;
    // pass 1, float only: element + 1, 0 for a miss, kUndecided for the double-precision search
#pragma unroll 1
    for (int m = 0; m < RPT; ++m) {
        const uint32_t i = blockIdx.x * (RPT * kProbeBlock) + m * kProbeBlock + threadIdx.x;
        uint32_t h = 0;
        if (i < n) {
            RayRng rng;
            rng.init(S.seed, s0 + i, 0);
            const double xs = sun.xmin + (sun.xmax - sun.xmin) * rng.u();
            const double ys = sun.ymin + (sun.ymax - sun.ymin) * rng.u();
            int cx = int(floor((xs - sun.gx0) * sun.ginv)), cy = int(floor((ys - sun.gy0) * sun.ginv));
            cx = min(max(cx, 0), sun.gnx - 1);
            cy = min(max(cy, 0), sun.gny - 1);
            const int2 range = reinterpret_cast<const int2 *>(sun.cell_start)[cy * sun.gnx + cx];
            // the point relative to the cell's lower corner (entries hold their centres so)
            const float xr = float(xs - (sun.gx0 + cx * sun.gcell)), yr = float(ys - (sun.gy0 + cy * sun.gcell));
            int best = -1;
            float bz = INFINITY;
            for (int k = range.x; k < range.y; ++k) {
                const float4 a = sun.cell_xa[k];
                const float qx = xr - a.x, qy = yr - a.y;
                if (qx * qx + qy * qy > a.z) continue;  // outside the padded disc
                const float4 c = sun.cell_xc[k];
                if (isnan(c.z)) {  // no exact footprint
                    best = -2;
                    break;
                }
                if (c.z == INFINITY) continue;  // an element that accepts no hit
                const float4 e0 = sun.cell_xb[k];
                const float u1 = e0.x * qx, u2 = e0.y * qy, v1 = e0.z * qx, v2 = e0.w * qy;
                const float au = fabsf(u1 + u2), av = fabsf(v1 + v2);
                const float mu = 2e-6f * (fabsf(u1) + fabsf(u2)) + 1e-6f;
                const float mv = 2e-6f * (fabsf(v1) + fabsf(v2)) + 1e-6f;
                if (au > 1.f + mu || av > 1.f + mv) continue;  // surely outside
                if (au >= 1.f - mu || av >= 1.f - mv) {         // within rounding of an edge
                    best = -2;
                    break;
                }
                const float g1 = c.x * qx, g2 = c.y * qy;
                const float z = c.z + g1 + g2;
                const float tol = 1e-6f * (fabsf(c.z) + fabsf(g1) + fabsf(g2)) + 1e-5f;
                if (fabsf(z - bz) <= tol) {  // two elements within rounding of one depth
                    best = -2;
                    break;
                }
                if (z < bz) {
                    bz = z;
                    best = __float_as_int(a.w);
                }
            }
            h = best == -2 ? kUndecided : uint32_t(best + 1);
        }
        hsh[m][threadIdx.x] = h;
    }
    // pass 2: undecided rays (a few per million) to the double-precision list; ballots, mask
    uint32_t mine = 0;
#pragma unroll 1
    for (int m = 0; m < RPT; ++m) {
        const uint32_t i = blockIdx.x * (RPT * kProbeBlock) + m * kProbeBlock + threadIdx.x;
        uint32_t h = hsh[m][threadIdx.x];
        if (h == kUndecided) {
            o.amb[atomicAdd(o.amb_count, 1u)] = i;
            h = 0;
            hsh[m][threadIdx.x] = 0;
        }
        if (o.hit_elem && i < n) o.hit_elem[i] = h;
        const unsigned bal = __ballot_sync(0xffffffffu, h != 0);
        if (lane == 0) {
            if (o.hit_mask) o.hit_mask[(blockIdx.x * (RPT * kProbeBlock) + m * kProbeBlock) / 32 + w] = bal;
            wb[m][w] = bal;
        }
        mine += __popc(bal);
    }
    // one reservation in the list per block: warp counts, their prefix, one atomic
    if (lane == 0) wn[w] = mine;
    __syncthreads();
    if (threadIdx.x < RPT && blockIdx.x * RPT + threadIdx.x < nb) {
        uint32_t c = 0;
        for (int k = 0; k < kProbeBlock / 32; ++k) c += __popc(wb[threadIdx.x][k]);
        o.block_counts[blockIdx.x * RPT + threadIdx.x] = c;
    }
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int k = 0; k < kProbeBlock / 32; ++k) {
            const uint32_t x = wn[k];
            wn[k] = t;
            t += x;
        }
        base = t ? atomicAdd(o.cand_count, t) : 0u;
    }
    __syncthreads();
    uint32_t at = base + wn[w];
    const unsigned lt = (1u << lane) - 1u;
    for (int m = 0; m < RPT; ++m) {
        const unsigned bal = wb[m][w];
        if ((bal >> lane) & 1u) {
            const uint32_t pos = at + __popc(bal & lt);
            o.cand[pos] = blockIdx.x * (RPT * kProbeBlock) + m * kProbeBlock + threadIdx.x;
            if (o.cand_el) o.cand_el[pos] = hsh[m][threadIdx.x];
        }
        at += __popc(bal);
    }
}

// The rays k_sun_probe_exact left undecided, searched in double (the FP64 probe's arithmetic):
// a hit is appended to the probe's list and counted in its block count and hit mask.
template <int MIXED>
__global__ void __launch_bounds__(kResolveBlock) k_sun_resolve_amb(const __grid_constant__ SceneDev S, uint64_t s0,
                                                                   ProbeOut o) {
    const uint32_t na = *o.amb_count;
    const SunDev &sun = S.sun;
    for (uint32_t c = blockIdx.x * kResolveBlock + threadIdx.x; c < na; c += gridDim.x * kResolveBlock) {
        const uint32_t i = o.amb[c];
        RayRng rng;
        rng.init(S.seed, s0 + i, 0);
        const double xs = sun.xmin + (sun.xmax - sun.xmin) * rng.u();
        const double ys = sun.ymin + (sun.ymax - sun.ymin) * rng.u();
        const int b = nearest_sun_grid_lazy<0, kEtFlat>(S, S.stages[0], xs, ys);
        if (b < 0) continue;
        const uint32_t h = uint32_t(b + 1);
        if (o.hit_elem) o.hit_elem[i] = h;
        const uint32_t pos = atomicAdd(o.cand_count, 1u);
        o.cand[pos] = i;
        if (o.cand_el) o.cand_el[pos] = h;
        atomicAdd(&o.block_counts[i / kProbeBlock], 1u);
        if (o.hit_mask) atomicOr(&o.hit_mask[i / 32], 1u << (i & 31));
    }
}

#ifdef ST_COMMON_KERNELS
// first kernel of the grid probe (above): candidates listed, hit-mask words cleared
__global__ void __launch_bounds__(kProbeBlock) k_sun_candidates(const __grid_constant__ SceneDev S, uint64_t s0,
                                                                uint32_t n, ProbeOut o, const RunState *rs) {
    // a block takes kCandRays sun rays (kCandRays / kProbeBlock per thread, kProbeBlock apart)
    const uint32_t nb = (n + kProbeBlock - 1) / kProbeBlock;
    if (threadIdx.x < kCandPerThread && blockIdx.x * kCandPerThread + threadIdx.x < nb)
        o.block_counts[blockIdx.x * kCandPerThread + threadIdx.x] = 0;
    if (o.hit_mask && threadIdx.x < kCandRays / 32) o.hit_mask[blockIdx.x * (kCandRays / 32) + threadIdx.x] = 0;
    if (rs->reached) return;  // the requested hits are numbered: this batch is surplus
    const SunDev &sun = S.sun;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned bal[kCandPerThread];
    uint32_t mine = 0;
    for (int m = 0; m < kCandPerThread; ++m) {
        const uint32_t i = blockIdx.x * kCandRays + m * kProbeBlock + threadIdx.x;
        bool listed = false;
        if (i < n) {
            RayRng rng;
            rng.init(S.seed, s0 + i, 0);
            const double xs = sun.xmin + (sun.xmax - sun.xmin) * rng.u();
            const double ys = sun.ymin + (sun.ymax - sun.ymin) * rng.u();
            const int2 range = sun_cell(sun, xs, ys);
            const float fx = float(xs), fy = float(ys);
            for (int k = range.x; k < range.y; ++k)
                if (sun_entry_pass(sun, k, fx, fy)) {
                    listed = true;
                    break;
                }
            if (!listed && o.hit_elem) o.hit_elem[i] = 0;
        }
        bal[m] = __ballot_sync(0xffffffffu, listed);
        mine += __popc(bal[m]);
    }
    // one atomic on the shared count per block: warp counts, their prefix, one reservation
    __shared__ uint32_t wn[kProbeBlock / 32], base;
    if (lane == 0) wn[w] = mine;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int k = 0; k < kProbeBlock / 32; ++k) {
            const uint32_t x = wn[k];
            wn[k] = t;
            t += x;
        }
        base = t ? atomicAdd(o.cand_count, t) : 0u;
    }
    __syncthreads();
    uint32_t at = base + wn[w];
    const unsigned lt = (1u << lane) - 1u;
    for (int m = 0; m < kCandPerThread; ++m) {
        if ((bal[m] >> lane) & 1u) o.cand[at + __popc(bal[m] & lt)] = blockIdx.x * kCandRays + m * kProbeBlock + threadIdx.x;
        at += __popc(bal[m]);
    }
}

// exclusive scan of the per-block counts (one block; counts fit in 32 bits per batch):
// each thread scans 8 consecutive counts, the block scans the threads' sums
__global__ void __launch_bounds__(1024) k_offsets(const uint32_t *counts, uint32_t nb, uint32_t *offsets,
                                                   uint32_t *total) {
    constexpr int kPer = 8;
    __shared__ uint32_t warp_sums[32];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t base = 0; base < nb; base += 1024 * kPer) {
        const uint32_t i0 = base + threadIdx.x * kPer;
        uint32_t v[kPer], sum = 0;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            v[k] = (i0 + k < nb) ? counts[i0 + k] : 0u;
            sum += v[k];
        }
        uint32_t x = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[w] = x;
        __syncthreads();
        if (w == 0) {
            uint32_t s = warp_sums[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            warp_sums[lane] = s;
        }
        __syncthreads();
        const uint32_t incl = x + (w > 0 ? warp_sums[w - 1] : 0u) + carry;
        uint32_t run = incl - sum;
#pragma unroll
        for (int k = 0; k < kPer; ++k) {
            if (i0 + k < nb) offsets[i0 + k] = run;
            run += v[k];
        }
        __syncthreads();
        if (threadIdx.x == 1023) carry = incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

// Grid-wide exclusive scan of the per-block counts in two kernels: k_scan_parts sums each
// chunk of kScanChunk counts, k_scan_chunks scans each chunk with the sum of the chunks
// before it (at most a few dozen per batch, added up by every block); kScanChunk and
// kScanBlock in st_launch.h.
__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t *sh) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sh[w] = v;
    __syncthreads();
    uint32_t t = 0;
    for (int k = 0; k < kScanBlock / 32; ++k) t += sh[k];
    __syncthreads();
    return t;
}
__global__ void __launch_bounds__(kScanBlock) k_scan_parts(const uint32_t *counts, uint32_t nb, uint32_t *parts) {
    __shared__ uint32_t sh[kScanBlock / 32];
    const uint32_t i0 = blockIdx.x * kScanChunk + threadIdx.x * (kScanChunk / kScanBlock);
    uint32_t v = 0;
#pragma unroll
    for (int k = 0; k < kScanChunk / kScanBlock; ++k) v += (i0 + k < nb) ? counts[i0 + k] : 0u;
    v = block_sum(v, sh);
    if (threadIdx.x == 0) parts[blockIdx.x] = v;
}
__global__ void __launch_bounds__(kScanBlock) k_scan_chunks(const uint32_t *counts, uint32_t nb, const uint32_t *parts,
                                                            uint32_t *offsets, uint32_t *total) {
    constexpr int kPer = kScanChunk / kScanBlock;
    __shared__ uint32_t sh[kScanBlock / 32];
    __shared__ uint32_t wsum[kScanBlock / 32];
    // sum of the chunks before this one (and of all chunks, for the total)
    uint32_t before = 0, all = 0;
    for (uint32_t b = threadIdx.x; b < gridDim.x; b += kScanBlock) {
        const uint32_t p = parts[b];
        all += p;
        if (b < blockIdx.x) before += p;
    }
    before = block_sum(before, sh);
    all = block_sum(all, sh);
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
    uint32_t run = before + x - sum;
    for (int k = 0; k < w; ++k) run += wsum[k];
#pragma unroll
    for (int k = 0; k < kPer; ++k) {
        if (i0 + k < nb) offsets[i0 + k] = run;
        run += v[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *total = all;
}

__global__ void __launch_bounds__(kProbeBlock) k_compact(uint64_t s0, uint32_t n, const uint32_t *hit_elem,
                                                          const uint32_t *counts, const uint32_t *offsets,
                                                          uint64_t *hit_sid, uint32_t *hit_el) {
    __shared__ uint32_t wsum[kProbeBlock / 32];
    if (counts[blockIdx.x] == 0) return;
    const uint32_t i = blockIdx.x * kProbeBlock + threadIdx.x;
    const uint32_t h = (i < n) ? hit_elem[i] : 0u;
    const unsigned bal = __ballot_sync(0xffffffffu, h != 0);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) wsum[w] = __popc(bal);
    __syncthreads();
    uint32_t pre = 0;
    for (int k = 0; k < w; ++k) pre += wsum[k];
    if (h != 0) {
        const uint32_t pos = offsets[blockIdx.x] + pre + __popc(bal & ((1u << lane) - 1u));
        hit_sid[pos] = s0 + i;
        hit_el[pos] = h - 1;
    }
}

// Counting sort of a batch's hits by first-stage element, so that each warp of the
// trace kernel carries rays leaving the same element (coherent traversals).  The input is
// the probe's list (ray, element + 1 or 0 per entry) in any order; the rank of a hit in
// sun-ray order (its ray number) comes from the scanned per-block counts and the hit mask.
// Order within an element is arbitrary: every result is independent of it (per-ray random
// streams, integer flux atomics, records ordered by ray number).

// rank of the hit on ray i among the batch's hits in ray order: the hits of the kProbeBlock
// rays before its block (off), then those of the block's mask words (a, b) before its own
struct RankIn {
    uint32_t off;
    uint4 a, b;
};
__device__ __forceinline__ RankIn rank_load(const uint32_t *offsets, const uint32_t *mask, uint32_t i) {
    static_assert(kProbeBlock == 256, "eight mask words per count slot");
    const uint32_t blk = i / kProbeBlock;
    const uint4 *m4 = reinterpret_cast<const uint4 *>(mask + size_t(blk) * 8);
    return RankIn{offsets[blk], m4[0], m4[1]};
}
__device__ __forceinline__ uint32_t rank_of(const RankIn &q, uint32_t i) {
    const uint32_t w = (i / 32) % 8;
    const uint32_t words[8] = {q.a.x, q.a.y, q.a.z, q.a.w, q.b.x, q.b.y, q.b.z, q.b.w};
    uint32_t r = q.off;
#pragma unroll
    for (uint32_t k = 0; k < 8; ++k) {
        if (k < w) r += __popc(words[k]);
        if (k == w) r += __popc(words[k] & ((1u << (i & 31)) - 1u));
    }
    return r;
}

// hits the trace numbers in this batch (the cut-off at the requested hit count)
__device__ __forceinline__ uint32_t batch_take(const RunState *rs, const uint32_t *total) {
    if (rs->reached) return 0u;
    const unsigned long long left = rs->target - rs->hits_done;
    const uint32_t n = *total;
    return uint32_t(n < left ? n : left);
}

// one sorted hit: sun-ray index, element, rank (one 16-byte store); the last numbered one
// marks the cut-off
__device__ __forceinline__ void list_put(uint64_t s0, uint32_t ray, uint32_t e, uint32_t pos, uint32_t rank,
                                         uint32_t take, RunState *rs, HitRec *hits) {
    HitRec h;
    h.sid = s0 + ray;
    h.el = e;
    h.rank = rank;
    hits[pos] = h;
    if (rank + 1 == take) rs->cut_sid = s0 + ray;
}

__global__ void __launch_bounds__(256) k_list_hist(const uint32_t *list_count, const uint32_t *cand_el,
                                                   uint32_t *elem_count) {
    const uint32_t n = *list_count;
    for (uint32_t i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
        const uint32_t h = cand_el[i];
        if (h) atomicAdd(&elem_count[h - 1], 1u);
    }
}
__global__ void __launch_bounds__(256) k_list_scatter(uint64_t s0, ProbeOut o, const uint32_t *offsets,
                                                      const uint32_t *total, RunState *rs, uint32_t *elem_cursor,
                                                      HitRec *hits) {
    const uint32_t n = *o.cand_count;
    const uint32_t take = batch_take(rs, total);
    for (uint32_t i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
        const uint32_t h = o.cand_el[i];
        if (!h) continue;
        const uint32_t pos = atomicAdd(&elem_cursor[h - 1], 1u);
        const uint32_t ray = o.cand[i];
        list_put(s0, ray, h - 1, pos, rank_of(rank_load(offsets, o.hit_mask, ray), ray), take, rs, hits);
    }
}

// The same counting sort for first stages of at most kSortBins elements, with the counts
// kept per block in shared memory: each block takes a contiguous chunk of the list,
// counts its elements there and adds its non-zero counts to the global ones (hist), or
// reserves one range per element in the output with a single global atomic and hands out
// the places in it from shared memory (scatter).  Global atomics: one per block and
// element present, instead of one per hit.
constexpr int kSortBins = 11264;
constexpr int kSortBlock = 1024;
constexpr int kSortUnroll = 4;
// count the elements of list entries [a, b) in h (kSortUnroll loads in flight per thread)
__device__ __forceinline__ void list_count_sh(uint32_t *h, const uint32_t *cand_el, uint32_t a, uint32_t b) {
    for (uint32_t i0 = a + threadIdx.x; i0 < b; i0 += kSortUnroll * kSortBlock) {
        uint32_t x[kSortUnroll];
#pragma unroll
        for (int u = 0; u < kSortUnroll; ++u) {
            const uint32_t i = i0 + u * kSortBlock;
            x[u] = (i < b) ? cand_el[i] : 0u;
        }
#pragma unroll
        for (int u = 0; u < kSortUnroll; ++u)
            if (x[u]) atomicAdd(&h[x[u] - 1], 1u);
    }
}
__global__ void __launch_bounds__(kSortBlock) k_list_hist_sh(const uint32_t *list_count, const uint32_t *cand_el,
                                                             uint32_t n_elem, uint32_t *elem_count) {
    __shared__ uint32_t h[kSortBins];
    const uint32_t n = *list_count;
    const uint32_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const uint32_t a = min(n, blockIdx.x * chunk), b = min(n, a + chunk);
    for (uint32_t e = threadIdx.x; e < n_elem; e += kSortBlock) h[e] = 0;
    __syncthreads();
    list_count_sh(h, cand_el, a, b);
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < n_elem; e += kSortBlock)
        if (h[e]) atomicAdd(&elem_count[e], h[e]);
}
__global__ void __launch_bounds__(kSortBlock) k_list_scatter_sh(uint64_t s0, ProbeOut o, const uint32_t *offsets,
                                                                const uint32_t *total, RunState *rs, uint32_t n_elem,
                                                                uint32_t *elem_cursor, HitRec *hits) {
    __shared__ uint32_t h[kSortBins];
    const uint32_t n = *o.cand_count;
    const uint32_t take = batch_take(rs, total);
    const uint32_t chunk = (n + gridDim.x - 1) / gridDim.x;
    const uint32_t a = min(n, blockIdx.x * chunk), b = min(n, a + chunk);
    for (uint32_t e = threadIdx.x; e < n_elem; e += kSortBlock) h[e] = 0;
    __syncthreads();
    list_count_sh(h, o.cand_el, a, b);
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < n_elem; e += kSortBlock)
        if (h[e]) h[e] = atomicAdd(&elem_cursor[e], h[e]);
    __syncthreads();
    // kSortUnroll entries per thread and step, their loads issued before their uses
    for (uint32_t i0 = a + threadIdx.x; i0 < b; i0 += kSortUnroll * kSortBlock) {
        uint32_t x[kSortUnroll], ray[kSortUnroll];
        RankIn q[kSortUnroll];
#pragma unroll
        for (int u = 0; u < kSortUnroll; ++u) {
            const uint32_t i = i0 + u * kSortBlock;
            x[u] = (i < b) ? o.cand_el[i] : 0u;
        }
#pragma unroll
        for (int u = 0; u < kSortUnroll; ++u) ray[u] = x[u] ? o.cand[i0 + u * kSortBlock] : 0u;
#pragma unroll
        for (int u = 0; u < kSortUnroll; ++u)
            if (x[u]) q[u] = rank_load(offsets, o.hit_mask, ray[u]);
#pragma unroll
        for (int u = 0; u < kSortUnroll; ++u) {
            if (!x[u]) continue;
            const uint32_t pos = atomicAdd(&h[x[u] - 1], 1u);
            list_put(s0, ray[u], x[u] - 1, pos, rank_of(q[u], ray[u]), take, rs, hits);
        }
    }
}

// single thread: apply the cut-off at the requested hit count and advance the run state
__global__ void k_advance(const uint32_t *total, const uint64_t *hit_sid, uint64_t s0, uint32_t n, RunState *rs) {
    rs->cursor = 0;  // the next batch's trace work queue starts empty
    if (rs->reached) return;
    const unsigned long long left = rs->target - rs->hits_done;
    const unsigned long long take = (*total < left) ? *total : left;
    rs->hits_done += take;
    if (rs->hits_done == rs->target && take > 0) {
        rs->reached = 1;
        rs->sun_rays = (hit_sid ? hit_sid[take - 1] : rs->cut_sid) + 1;
    } else {
        rs->sun_rays = s0 + n;
    }
}
#endif  // ST_COMMON_KERNELS

// ------------------------------------------------------------------------------------
// Trace: a wavefront over device-side ray queues.
//
// The per-ray state machine of raytrace.cpp:582-1040 is cut into two steps, each its own
// kernel over a queue of rays: `shade` (the full hit on a known element: interaction,
// random draws, records, flux and counters, then the outgoing ray) and `search` (the
// nearest element of the current stage, or the stage exit).  Rays move between the
// queues until they are absorbed or leave the last stage; the state they carry between
// kernels is what the serial loop keeps in its locals.  Each kernel holds only the code of
// its step, so it keeps few registers and many resident warps, and every warp does the
// same step (a single trace kernel with both steps inlined was latency bound).  After a
// fixed number of rounds a finishing kernel runs the remaining rays to the end one step
// after the other.  Results do not depend on the queue order (per-ray random streams,
// integer atomics, records ordered on the host by ray number and hit index).
// ------------------------------------------------------------------------------------
enum WfStatus : int { kWfDone = 0, kWfShade = 1, kWfSearch = 2 };

struct WfRay {
    uint64_t sid;
    uint32_t raynum, draw;
    int si, hits, last_j, next_j, fe0;
    double p[3], c[3];  // global while hits == 0 in stage si, stage coordinates after
    bool moved;         // p, c changed since loaded
};

struct WfBlockCtr {
    unsigned long long entries[kMaxStages];
    unsigned long long intersections;  // records the reference would write (hits and misses)
    unsigned int max_enter[kMaxStages], max_tt[kMaxStages];
    unsigned int flags;
};

__device__ __forceinline__ void wf_ctr_init(WfBlockCtr &c) {
    if (threadIdx.x < kMaxStages) {
        c.entries[threadIdx.x] = 0;
        c.max_enter[threadIdx.x] = 0;
        c.max_tt[threadIdx.x] = 0;
    }
    if (threadIdx.x == 0) {
        c.flags = 0;
        c.intersections = 0;
    }
    __syncthreads();
}

__device__ __forceinline__ void wf_ctr_flush(WfBlockCtr &c, const SceneDev &S, const TraceOut &O) {
    __syncthreads();
    if (threadIdx.x < S.n_stages) {
        const int s = threadIdx.x;
        if (c.entries[s]) {
            atomicAdd(&O.ctr->stage_entries[s], c.entries[s]);
            atomicMax(&O.ctr->max_enter[s], c.max_enter[s]);
        }
        if (c.max_tt[s]) atomicMax(&O.ctr->max_ttmiss[s], c.max_tt[s]);
    }
    if (threadIdx.x == 0 && c.flags) atomicOr(&O.ctr->flags, c.flags);
    if (threadIdx.x == 0 && c.intersections) atomicAdd(&O.ctr->records, c.intersections);
}

// one more intersection record (counted whether or not records are kept)
__device__ __forceinline__ void wf_count_record(WfBlockCtr &c) {
    const unsigned mask = __activemask();
    if ((threadIdx.x & 31) == __ffs(mask) - 1) atomicAdd(&c.intersections, (unsigned long long)__popc(mask));
}

__device__ __forceinline__ WfRay wf_load(const WfState &W, uint32_t i) {
    WfRay r;
    r.sid = W.sid[i];
    r.raynum = W.raynum[i];
    r.draw = W.draw[i];
    const int4 m = W.meta[i];
    r.si = m.x;
    r.hits = m.y;
    r.last_j = m.z;
    r.next_j = m.w;
    r.fe0 = W.fe0[i];
    for (int q = 0; q < 3; ++q) {
        r.p[q] = W.p[size_t(q) * W.cap + i];
        r.c[q] = W.c[size_t(q) * W.cap + i];
    }
    r.moved = false;
    return r;
}

__device__ __forceinline__ void wf_store(const WfState &W, uint32_t i, const WfRay &r, bool all) {
    if (all) {
        W.sid[i] = r.sid;
        W.raynum[i] = r.raynum;
    }
    W.draw[i] = r.draw;
    W.meta[i] = make_int4(r.si, r.hits, r.last_j, r.next_j);
    W.fe0[i] = r.fe0;
    if (all || r.moved)
        for (int q = 0; q < 3; ++q) {
            W.p[size_t(q) * W.cap + i] = r.p[q];
            W.c[size_t(q) * W.cap + i] = r.c[q];
        }
}

// Block-wide queue appends: every thread with `want_a` appends `slot` to queue A, every
// thread with kb >= 0 to queue kb of the B family (queue k at qb + k * capb, its count at
// cb[k]), with one global atomic per queue and block (a queue's count is a single address
// that every block of the grid updates).  Called by all threads of the block; wf_push_init
// clears the shared counts first.
struct WfPushSh {
    uint32_t na[kTraceBlock / 32];
    uint32_t nb[kSearchKinds];
    uint32_t base_a, base_b[kSearchKinds];
};
__device__ __forceinline__ void wf_push_init(WfPushSh &sh) {
    if (threadIdx.x < kSearchKinds) sh.nb[threadIdx.x] = 0;  // visible after the next __syncthreads
}
__device__ __forceinline__ void wf_block_push(WfPushSh &sh, uint32_t *qa, uint32_t *ca, bool want_a, uint32_t *qb,
                                              uint32_t capb, uint32_t *cb, int kb, uint32_t slot) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const unsigned ba = __ballot_sync(0xffffffffu, want_a);
    const unsigned peers = __match_any_sync(0xffffffffu, kb);
    const int leader = __ffs(peers) - 1;
    uint32_t off = 0;
    if (lane == 0) sh.na[w] = __popc(ba);
    if (kb >= 0 && lane == leader) off = atomicAdd(&sh.nb[kb], uint32_t(__popc(peers)));
    off = __shfl_sync(0xffffffffu, off, leader) + __popc(peers & lt);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t ta = 0;
        for (int k = 0; k < kTraceBlock / 32; ++k) {
            const uint32_t a = sh.na[k];
            sh.na[k] = ta;  // exclusive prefix over the warps
            ta += a;
        }
        sh.base_a = ta ? atomicAdd(ca, ta) : 0u;
    }
    if (threadIdx.x < kSearchKinds) {
        const uint32_t t = sh.nb[threadIdx.x];
        if (t) sh.base_b[threadIdx.x] = atomicAdd(&cb[threadIdx.x], t);
    }
    __syncthreads();
    if (want_a) qa[sh.base_a + sh.na[w] + __popc(ba & lt)] = slot;
    if (kb >= 0) qb[size_t(kb) * capb + sh.base_b[kb] + off] = slot;
    if (threadIdx.x < kSearchKinds) sh.nb[threadIdx.x] = 0;  // read by no thread before the barrier below
    __syncthreads();  // sh is reused by the next call
}

// a ray enters stage si: entry count and largest ray number (raytrace.cpp:617-623)
__device__ __forceinline__ void wf_stage_enter(WfBlockCtr &c, int si, uint32_t raynum) {
    const unsigned mask = __activemask();
    const unsigned peers = __match_any_sync(mask, si);
    const unsigned mx = __reduce_max_sync(peers, raynum);
    if ((threadIdx.x & 31) == __ffs(peers) - 1) {
        atomicAdd(&c.entries[si], (unsigned long long)__popc(peers));
        atomicMax(&c.max_enter[si], mx);
    }
}

// the ray leaves stage si (no further hit there): a miss is recorded with element 0 and
// ends the ray unless the stage is trace-through (raytrace.cpp:800-826; the one miss the
// reference does not record is removed on the host from max_ttmiss); otherwise the ray
// goes on, in global coordinates, to the next stage
// a ray leaving stage 1 or 2 (0-based si 0 or 1) toward the next stage, kept when stage
// data are saved (global position, direction, ray number)
__device__ __forceinline__ void wf_save_ray(const TraceOut &O, const WfRay &r) {
    if (r.si > 1 || !O.save_rows[r.si]) return;
    const unsigned long long slot = atomicAdd(O.save_count[r.si], 1ull);
    if (slot >= O.save_cap) return;
    double *row = O.save_rows[r.si] + 7 * slot;
    for (int q = 0; q < 3; ++q) {
        row[q] = r.p[q];
        row[3 + q] = r.c[q];
    }
    row[6] = double(r.raynum);
}

template <int RECORDS>
__device__ __forceinline__ int wf_exit_stage(const SceneDev &S, const TraceOut &O, WfBlockCtr &c, WfRay &r,
                                             const double ps[3], const double cs[3]) {
    const StageRec &st = S.stages[r.si];
    if (r.hits == 0) {
        if (r.si == 0) return kWfDone;  // cannot happen: first-stage rays are numbered hits
        wf_count_record(c);
        if (RECORDS) {
            const unsigned long long slot = warp_reserve(O.rec_count);
            if (slot < O.rec_cap) {
                RecordDev rec;
                to_local(st.R, st.o, r.p, r.c, rec.pos, rec.cos);
                rec.element = 0;
                rec.stage = r.si + 1;
                rec.raynum = r.raynum;
                rec.seq = 0;
                O.recs[slot] = rec;
            }
        }
        if (!st.tracethrough) return kWfDone;
        atomicMax(&c.max_tt[r.si], r.raynum);
        // global ray unchanged
    } else {
        to_ref(st.R, st.o, ps, cs, r.p, r.c);
        r.moved = true;
    }
    wf_save_ray(O, r);
    if (r.si + 1 >= S.n_stages) return kWfDone;
    r.si += 1;
    r.hits = 0;
    r.last_j = -1;
    r.next_j = -1;
    wf_stage_enter(c, r.si, r.raynum);
    return kWfSearch;
}

// the ray's position/direction in its stage's coordinates
__device__ __forceinline__ void wf_stage_ray(const SceneDev &S, const WfRay &r, double ps[3], double cs[3]) {
    if (r.hits == 0) {
        const StageRec &st = S.stages[r.si];
        to_local(st.R, st.o, r.p, r.c, ps, cs);
    } else {
        for (int q = 0; q < 3; ++q) {
            ps[q] = r.p[q];
            cs[q] = r.c[q];
        }
    }
}

// search step: nearest element of the current stage (raytrace.cpp:698-770), with the code
// of search kind KIND (the kind of the ray's stage; 0 holds every case)
template <int MIXED, int RECORDS, int KIND = 0>
__device__ __forceinline__ int wf_search(const SceneDev &S, const TraceOut &O, WfBlockCtr &c, WfRay &r) {
    double ps[3], cs[3];
    wf_stage_ray(S, r, ps, cs);
    const int j = nearest_kind<MIXED, KIND>(S, S.stages[r.si], ps, cs, r.last_j);
    if (j < 0) return wf_exit_stage<RECORDS>(S, O, c, r, ps, cs);
    r.next_j = j;
    return kWfShade;
}

template <int MIXED, int RECORDS>
__device__ __forceinline__ int wf_shade_hit(const SceneDev &S, const TraceOut &O, WfBlockCtr &c, WfRay &r,
                                            const ElemRec &e, int j, const Hit &h);

// shade step: the hit on element next_j and what the ray does there (raytrace.cpp:830-1000);
// FLAT: the stage holds flat elements only; CLOSED: closed-form surfaces only
template <int MIXED, int RECORDS, int FLAT = 0, int CLOSED = 0>
__device__ __forceinline__ int wf_shade(const SceneDev &S, const TraceOut &O, WfBlockCtr &c, WfRay &r) {
    const int si = r.si;
    const StageRec &st = S.stages[si];
    double ps[3], cs[3];
    wf_stage_ray(S, r, ps, cs);
    const int j = r.next_j;
    r.next_j = -1;
    const ElemRec &e = S.elems[st.first_elem + j];
    Hit h;
    double pl;
    // re-test the chosen element for the full hit (same arithmetic as the search)
    const bool hit = FLAT ? element_test_flat<MIXED>(e, ps, cs, pl, &h) : element_test<MIXED, CLOSED>(S, e, ps, cs, pl, &h);
    if (!hit) return wf_exit_stage<RECORDS>(S, O, c, r, ps, cs);
    return wf_shade_hit<MIXED, RECORDS>(S, O, c, r, e, j, h);
}

// the hit h of the ray on element j of its stage and what the ray does there
// (raytrace.cpp:830-1000)
template <int MIXED, int RECORDS>
__device__ __forceinline__ int wf_shade_hit(const SceneDev &S, const TraceOut &O, WfBlockCtr &c, WfRay &r,
                                            const ElemRec &e, int j, const Hit &h) {
    const int si = r.si;
    const StageRec &st = S.stages[si];
    double ps[3], cs[3];
    const int hits = ++r.hits;
    if (hits == 1) {
        warp_count(O.first_hits, st.first_elem + j);
        if (si == 0) r.fe0 = st.first_elem + j;
    }
    RayRng rng;
    rng.init(S.seed, r.sid, r.draw);
    bool absorbed = false;
    double pout[3], cout[3];
    if (st.virt) {
        for (int q = 0; q < 3; ++q) {
            pout[q] = h.pe[q];
            cout[q] = h.ce[q];
        }
    } else {
        if (e.interaction != 1 && e.interaction != 2) {
            atomicOr(&c.flags, unsigned(kFlagBadInteraction));
            absorbed = true;
        } else {
            const OpticRec &op = S.optics[h.back ? e.opt_back : e.opt_front];
            const double tv = test_value<MIXED>(S, op, e.interaction, h.ce, h.n);
            if (tv <= rng.u()) absorbed = true;
            if (!absorbed) {
                double cin[3] = {h.ce[0], h.ce[1], h.ce[2]};
                if (S.sunshape_on && si == 0 && hits == 1) {
                    double c2[3];
                    error_sample<MIXED>(S, S.sun.shape, S.sun.sigma / 1000.0, cin, rng, false, h.n, c2);
                    for (int q = 0; q < 3; ++q) cin[q] = c2[q];
                }
                double nrm[3] = {h.n[0], h.n[1], h.n[2]};
                if (S.errors_on) {
                    double n2[3];
                    const int d = op.dist;
                    const int dd = (d == 'g' || d == 'G' || d == 'p' || d == 'P') ? d : 0;
                    error_sample<MIXED>(S, dd, op.slope / 1000.0, nrm, rng, false, nrm, n2);
                    for (int q = 0; q < 3; ++q) nrm[q] = n2[q];
                }
                if (e.interaction == 1)
                    refract<MIXED>(op, cin, nrm, rng, cout);
                else
                    reflect(cin, nrm, cout);
                if (S.errors_on) {
                    const bool diffuse = (op.dist == 'f' || op.dist == 'F');
                    double axis[3], c3[3];
                    for (int q = 0; q < 3; ++q) axis[q] = diffuse ? nrm[q] : cout[q];
                    error_sample<MIXED>(S, op.dist, op.spec / 1000.0, axis, rng, e.interaction == 2, nrm, c3);
                    for (int q = 0; q < 3; ++q) cout[q] = c3[q];
                }
                for (int q = 0; q < 3; ++q) pout[q] = h.pe[q];
            }
        }
    }
    r.draw = rng.k;
    wf_count_record(c);
    if (RECORDS) {
        const unsigned long long slot = warp_reserve(O.rec_count);
        if (slot < O.rec_cap) {
            RecordDev rec;
            to_ref(e.R, e.o, h.pe, h.ce, rec.pos, rec.cos);
            rec.element = absorbed ? -(j + 1) : (j + 1);
            rec.stage = si + 1;
            rec.raynum = r.raynum;
            rec.seq = uint32_t(hits - 1);
            O.recs[slot] = rec;
        }
    }
    if (S.n_flux) bin_flux<MIXED>(S, si, j, absorbed, h.pe, r.fe0);
    if (absorbed) {
        warp_count(O.absorbed, st.first_elem + j);
        if (si == S.n_stages - 1 && r.fe0 >= 0) warp_count(O.delivered, r.fe0);
        return kWfDone;
    }
    to_ref(e.R, e.o, pout, cout, ps, cs);
    // A flat element cannot meet the ray leaving it: the next test's 1e-5 nudge moves the
    // origin 1e-5 |cz| off the plane, behind the ray.  Skipped only when that offset exceeds
    // the round-off of the local z (1e-13 of the coordinates, hundreds of ulps), so the
    // skipped test is one that fails.
    r.last_j = (e.stype == kSurfFlat &&
                1e-5 * fabs(cout[2]) >
                    1e-13 * (1.0 + fabs(e.o[0]) + fabs(e.o[1]) + fabs(e.o[2]) + fabs(pout[0]) + fabs(pout[1])))
                   ? j
                   : -1;
    for (int q = 0; q < 3; ++q) {
        r.p[q] = ps[q];
        r.c[q] = cs[q];
    }
    r.moved = true;
    if (!st.multihit) return wf_exit_stage<RECORDS>(S, O, c, r, ps, cs);
    if (hits >= kMaxHitsPerStage) {
        atomicOr(&c.flags, unsigned(kFlagHitCap));
        return wf_exit_stage<RECORDS>(S, O, c, r, ps, cs);
    }
    return kWfSearch;
}

// First kernel: the batch's numbered rays (hit-list entries below the cut-off at the
// requested hit count; k_advance applies the same rule after the trace) enter the first
// stage and are shaded on the element the probe found.
// FLAT 1: the first stage holds flat elements only; 2: besides, its search kind is
// kSearchFlat, and the rays it reflects are searched for blocking in this kernel (their
// results go to round 0's shade queue and to the search queue of the ray's stage).
template <int MIXED, int RECORDS, int FLAT>
__global__ void __launch_bounds__(kTraceBlock, FLAT ? (MIXED ? kWfFirstFlatMinBlocksMixed : kWfFirstFlatMinBlocks)
                                                    : kWfShadeMinBlocks) k_wf_first(
    const __grid_constant__ SceneDev S, const HitRec *hits, const uint32_t *total,
    const RunState *rs, TraceOut O, WfState W, const __grid_constant__ WfQueues Q) {
    __shared__ WfBlockCtr c;
    __shared__ WfPushSh psh;
    wf_push_init(psh);
    wf_ctr_init(c);
    uint32_t n = 0, take = 0, raynum_base = 0;
    if (!rs->reached) {
        const unsigned long long left = rs->target - rs->hits_done;
        n = *total;
        take = uint32_t(n < left ? n : left);
        raynum_base = uint32_t(rs->hits_done);
    }
    const uint32_t stride = gridDim.x * kTraceBlock;
    // whole blocks in the loop (block-wide queue appends)
    const uint32_t n_round = (n + kTraceBlock - 1) / kTraceBlock * kTraceBlock;
    for (uint32_t i = blockIdx.x * kTraceBlock + threadIdx.x; i < n_round; i += stride) {
        bool live = false;
        WfRay r;
        if (i < n) {
            const HitRec hr = hits[i];
            live = hr.rank < take;
            if (live) {
                r.sid = hr.sid;
                r.raynum = raynum_base + hr.rank + 1;
                RayRng rng;
                rng.init(S.seed, r.sid, 0);
                double xs, ys;
                make_ray(S, r.sid, rng, r.p, r.c, xs, ys);
                r.draw = rng.k;
                r.si = 0;
                r.hits = 0;
                r.last_j = -1;
                r.next_j = int(hr.el);
                r.fe0 = -1;
                r.moved = true;
            }
        }
        int kb = -1, status = kWfDone;
        if (live) {
            wf_stage_enter(c, 0, r.raynum);
            // (an entry without a known element is searched in the first round)
            status = (r.next_j >= 0) ? wf_shade<MIXED, RECORDS, FLAT ? 1 : 0>(S, O, c, r) : int(kWfSearch);
            // FLAT 2: the ray still in the first stage is searched here (its blocking search)
            if (FLAT == 2 && status == kWfSearch && r.si == 0) status = wf_search<MIXED, RECORDS, kSearchFlat>(S, O, c, r);
            if (status != kWfDone) {
                wf_store(W, i, r, true);
                if (status == kWfSearch) kb = Q.stage_queue[r.si];
            }
        }
        wf_block_push(psh, Q.shade, Q.counts + Q.n_queues, status == kWfShade, Q.search[0], Q.cap, Q.counts, kb, i);
    }
    wf_ctr_flush(c, S, O);
}

// Replay entry: rays of saved stage data enter the second stage (raytrace.cpp:544-578
// loads them in place of tracing the first stage).  Row i draws from its own stream
// (key: bit 62 set, row index), as the replayed rays' first-stage draws are not known.
template <int MIXED, int RECORDS>
__global__ void __launch_bounds__(kTraceBlock, kWfShadeMinBlocks) k_wf_replay(
    const __grid_constant__ SceneDev S, TraceOut O, WfState W, ReplayIn in, const __grid_constant__ WfQueues Q) {
    __shared__ WfBlockCtr c;
    __shared__ WfPushSh psh;
    wf_push_init(psh);
    wf_ctr_init(c);
    const uint32_t n = in.n;
    const uint32_t stride = gridDim.x * kTraceBlock;
    const uint32_t n_round = (n + kTraceBlock - 1) / kTraceBlock * kTraceBlock;
    for (uint32_t i = blockIdx.x * kTraceBlock + threadIdx.x; i < n_round; i += stride) {
        const bool live = i < n && S.n_stages > 1;
        if (live) {
            WfRay r;
            const double *row = in.rows + 7 * size_t(i);
            for (int q = 0; q < 3; ++q) {
                r.p[q] = row[q];
                r.c[q] = row[3 + q];
            }
            r.raynum = uint32_t(row[6]);
            r.sid = (1ull << 62) | i;
            r.draw = 0;
            r.si = 1;
            r.hits = 0;
            r.last_j = -1;
            r.next_j = -1;
            r.fe0 = in.fe0 ? in.fe0[i] : -1;
            r.moved = true;
            wf_stage_enter(c, 1, r.raynum);
            wf_store(W, i, r, true);
        }
        wf_block_push(psh, nullptr, nullptr, false, Q.search[0], Q.cap, Q.counts, live ? int(Q.stage_queue[1]) : -1,
                      i);
    }
    wf_ctr_flush(c, S, O);
}

// Search kernel of search kind KIND, over queue k of round r: rays that find an element go
// to the round's shade queue, those that move on to another stage to the next round's
// search queue of that stage.
template <int KIND>
struct SearchBounds {
    static constexpr int min_blocks = (KIND & kSearchBrute) ? kWfBruteMinBlocks
                                      : (KIND & kSearchFlat)  ? kWfFlatSearchMinBlocks
                                                              : kWfSearchMinBlocks;
};
template <int MIXED, int RECORDS, int KIND>
__global__ void __launch_bounds__(kTraceBlock, SearchBounds<KIND>::min_blocks) k_wf_search(
    const __grid_constant__ SceneDev S, TraceOut O, WfState W, const __grid_constant__ WfQueues Q, int r, int k) {
    __shared__ WfBlockCtr c;
    __shared__ WfPushSh psh;
    wf_push_init(psh);
    wf_ctr_init(c);
    const int nq = Q.n_queues;
    uint32_t *cnt = Q.counts + r * (nq + 1);
    const uint32_t *q_in = Q.search[r & 1] + size_t(k) * Q.cap;
    const uint32_t n = cnt[k];
    const uint32_t stride = gridDim.x * kTraceBlock;
    const uint32_t n_round = (n + kTraceBlock - 1) / kTraceBlock * kTraceBlock;
    for (uint32_t q = blockIdx.x * kTraceBlock + threadIdx.x; q < n_round; q += stride) {
        int status = kWfDone, kb = -1;
        uint32_t i = 0;
        if (q < n) {
            i = q_in[q];
            WfRay ray = wf_load(W, i);
            status = wf_search<MIXED, RECORDS, KIND>(S, O, c, ray);
            if (status != kWfDone) wf_store(W, i, ray, false);
            if (status == kWfSearch) kb = Q.stage_queue[ray.si];
        }
        wf_block_push(psh, Q.shade, cnt + nq, status == kWfShade, Q.search[(r + 1) & 1], Q.cap, cnt + nq + 1, kb, i);
    }
    wf_ctr_flush(c, S, O);
}

// Shade kernel over round r's shade queue: survivors go to the next round's search queues.
// CLOSED: every stage has closed-form surfaces only.
template <int MIXED, int RECORDS, int CLOSED>
__global__ void __launch_bounds__(kTraceBlock, CLOSED ? (MIXED ? kWfClosedShadeMinBlocksMixed : kWfClosedShadeMinBlocks)
                                                      : kWfShadeMinBlocks) k_wf_shade(const __grid_constant__ SceneDev S, TraceOut O,
                                                                             WfState W, const __grid_constant__ WfQueues Q,
                                                                             int r) {
    __shared__ WfBlockCtr c;
    __shared__ WfPushSh psh;
    wf_push_init(psh);
    wf_ctr_init(c);
    const int nq = Q.n_queues;
    uint32_t *cnt = Q.counts + r * (nq + 1);
    const uint32_t n = cnt[nq];
    const uint32_t stride = gridDim.x * kTraceBlock;
    const uint32_t n_round = (n + kTraceBlock - 1) / kTraceBlock * kTraceBlock;
    for (uint32_t q = blockIdx.x * kTraceBlock + threadIdx.x; q < n_round; q += stride) {
        int kb = -1;
        uint32_t i = 0;
        if (q < n) {
            i = Q.shade[q];
            WfRay ray = wf_load(W, i);
            const int status = wf_shade<MIXED, RECORDS, 0, CLOSED>(S, O, c, ray);
            if (status != kWfDone) {
                wf_store(W, i, ray, false);
                kb = Q.stage_queue[ray.si];
            }
        }
        wf_block_push(psh, nullptr, nullptr, false, Q.search[(r + 1) & 1], Q.cap, cnt + nq + 1, kb, i);
    }
    wf_ctr_flush(c, S, O);
}

// Finishing kernel: every ray still queued (the search queues of round `rounds`) runs to
// its end, one step after the other.
template <int MIXED, int RECORDS>
__global__ void __launch_bounds__(kTraceBlock, kWfShadeMinBlocks) k_wf_finish(const __grid_constant__ SceneDev S, TraceOut O,
                                                                              WfState W, const __grid_constant__ WfQueues Q) {
    __shared__ WfBlockCtr c;
    wf_ctr_init(c);
    const int nq = Q.n_queues, R = Q.rounds;
    const uint32_t *cnt = Q.counts + R * (nq + 1);
    for (int k = 0; k < nq; ++k) {
        const uint32_t n = cnt[k];
        const uint32_t *q_in = Q.search[R & 1] + size_t(k) * Q.cap;
        for (uint32_t q = blockIdx.x * kTraceBlock + threadIdx.x; q < n; q += gridDim.x * kTraceBlock) {
            WfRay r = wf_load(W, q_in[q]);
            int status = (r.next_j >= 0) ? int(kWfShade) : int(kWfSearch);
            while (status != kWfDone)
                status = (status == kWfShade) ? wf_shade<MIXED, RECORDS>(S, O, c, r) : wf_search<MIXED, RECORDS>(S, O, c, r);
        }
    }
    wf_ctr_flush(c, S, O);
}

// Host side of the trace launch (instantiated per precision in its translation unit).
template <int MIXED, int RECORDS, int KIND>
static void wf_launch_search(const SceneDev &S, const TraceOut &O, const WfState &W, const WfQueues &Q, int r, int k,
                             int sms, cudaStream_t st) {
    // persistent grid: every block the kernel can keep resident on every SM
    static int per_sm = 0;
    if (per_sm == 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wf_search<MIXED, RECORDS, KIND>, kTraceBlock, 0);
        per_sm = per_sm > 0 ? per_sm : 1;
    }
    k_wf_search<MIXED, RECORDS, KIND><<<sms * per_sm, kTraceBlock, 0, st>>>(S, O, W, Q, r, k);
}

template <int MIXED, int RECORDS>
static int wf_launch(const SceneDev &S, const HitRec *hits,
                     const uint32_t *total, const RunState *rs, const TraceOut &O, const WfState &W,
                     const WfQueues &Q, const ReplayIn *replay, cudaStream_t st) {
    // persistent grids: every block the kernels can keep resident on every SM
    static int per_sm[6] = {0, 0, 0, 0, 0, 0};
    if (per_sm[0] == 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[0], k_wf_first<MIXED, RECORDS, 0>, kTraceBlock, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[4], k_wf_first<MIXED, RECORDS, 1>, kTraceBlock, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[5], k_wf_first<MIXED, RECORDS, 2>, kTraceBlock, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[1], k_wf_shade<MIXED, RECORDS, 0>, kTraceBlock, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[3], k_wf_shade<MIXED, RECORDS, 1>, kTraceBlock, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[2], k_wf_finish<MIXED, RECORDS>, kTraceBlock, 0);
        for (int &x : per_sm) x = x > 0 ? x : 1;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int R = Q.rounds, nq = Q.n_queues;
    bool all_closed = true;  // every stage's surfaces are closed-form: the shade kernel without the rest
    for (int s = 0; s < S.n_stages; ++s) all_closed = all_closed && S.stages[s].closed_only;
    int launches = 2;
    cudaMemsetAsync(Q.counts, 0, sizeof(uint32_t) * (R + 1) * (nq + 1), st);
    if (replay)
        k_wf_replay<MIXED, RECORDS><<<sms * per_sm[0], kTraceBlock, 0, st>>>(S, O, W, *replay, Q);
    else if (stage_search_kind(S.stages[0]) == kSearchFlat)  // heliostat fields: blocking search fused
        k_wf_first<MIXED, RECORDS, 2><<<sms * per_sm[5], kTraceBlock, 0, st>>>(S, hits, total, rs,
                                                                                 O, W, Q);
    else if (S.stages[0].flat_only)  // a first stage of flat elements only
        k_wf_first<MIXED, RECORDS, 1><<<sms * per_sm[4], kTraceBlock, 0, st>>>(S, hits, total, rs,
                                                                                 O, W, Q);
    else
        k_wf_first<MIXED, RECORDS, 0><<<sms * per_sm[0], kTraceBlock, 0, st>>>(S, hits, total, rs,
                                                                                 O, W, Q);
    for (int r = 0; r < R; ++r) {
        for (int k = 0; k < nq; ++k) {
            switch (Q.queue_kind[k]) {
                case 1: wf_launch_search<MIXED, RECORDS, 1>(S, O, W, Q, r, k, sms, st); break;
                case 2: wf_launch_search<MIXED, RECORDS, 2>(S, O, W, Q, r, k, sms, st); break;
                case 3: wf_launch_search<MIXED, RECORDS, 3>(S, O, W, Q, r, k, sms, st); break;
                case 4: wf_launch_search<MIXED, RECORDS, 4>(S, O, W, Q, r, k, sms, st); break;
                case 6: wf_launch_search<MIXED, RECORDS, 6>(S, O, W, Q, r, k, sms, st); break;
                default: wf_launch_search<MIXED, RECORDS, 0>(S, O, W, Q, r, k, sms, st);
            }
            ++launches;
        }
        if (all_closed)
            k_wf_shade<MIXED, RECORDS, 1><<<sms * per_sm[3], kTraceBlock, 0, st>>>(S, O, W, Q, r);
        else
            k_wf_shade<MIXED, RECORDS, 0><<<sms * per_sm[1], kTraceBlock, 0, st>>>(S, O, W, Q, r);
        ++launches;
    }
    k_wf_finish<MIXED, RECORDS><<<sms * per_sm[2], kTraceBlock, 0, st>>>(S, O, W, Q);
    return launches;
}

}  // namespace stb
