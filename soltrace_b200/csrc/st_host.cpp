// Host side of coretrace_api.so: the SolTrace context and its C API
// (coretrace/stapi.h:68-176), geometry set-up, acceleration structures and the
// readback of the records the device puts in the reference's order (st_run.cu).
//
// The scene model follows coretrace/types.h:85-343; set-up follows
// coretrace/input.cpp (InitGeometries 153-286, TranslateSurfaceParams 288-366,
// ReadSurfaceFile 368-573, CheckInputs 87-150), coretrace/apertureplane.cpp
// and coretrace/suntoprimarystage.cpp, and then flattens everything into the
// device tables of st_scene.h.
#include <algorithm>
#include <array>
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <climits>
#include <limits>
#include <numeric>
#include <string>
#include <strings.h>
#include <thread>
#include <vector>

#include "../../include/st_b200.h"
#include "st_host.h"

namespace {

using namespace stb;
constexpr double kDegToRad = 0.017453292519943295;
constexpr double kPi = 3.141592653589793238462643;

struct Face {
    char dist = 'g';
    int optnum = 1, apgr = 0, order = 0;
    double refl = 0, trans = 0, slope = 0, spec = 0;
    double n[4] = {0, 0, 0, 0};
    double ab12[4] = {0, 0, 0, 0};
    std::vector<double> refl_tab, trans_tab;  // (angle, value) pairs
    bool use_refl = false, use_trans = false;
};
struct OpticSet {
    std::string name;
    Face front, back;
};
struct Elem {
    bool enabled = true;
    double origin[3] = {0, 0, 0}, aim[3] = {0, 0, 0}, zrot = 0;
    char shape = ' ';
    double p[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    char surface = ' ';
    int stype = 0;
    double kappa = 0, alpha[5] = {0, 0, 0, 0, 0}, vcx = 0, vcy = 0, ra = 0, rs = 0, cone = 0, curv = 0;
    int fit_order = 0;
    std::vector<double> bcoef, poly, spl_x, spl_y, spl_y2, vshot;
    int vshot_rows = 0;
    bool fe_surface = false;
    int interaction = 0;
    std::string optic;
    // derived
    double R[9] = {0}, area = 0, zap = 0;
    int optic_idx = -1;
};
struct StageM {
    bool multihit = true, virt = false, tracethrough = false;
    double origin[3] = {0, 0, 0}, aim[3] = {0, 0, 0}, zrot = 0;
    double R[9] = {0};
    std::vector<Elem> elems;
};
struct SunM {
    char shape = ' ';
    double sigma = 0;
    bool point_source = false;
    std::vector<double> ang, inten;  // mirrored table
    double max_angle = 0, max_intensity = 0;
    double origin[3] = {0, 0, 0};
    double xmin = 0, xmax = 0, ymin = 0, ymax = 0;
};
struct FluxMap {
    FluxMapReq req;
    std::vector<unsigned long long> counts;
};

struct Context {
    SunM sun;
    std::vector<OpticSet> optics;
    std::vector<StageM> stages;
    int raycount = 1000, raymax = 100000;
    bool dyn = false, err_sun = true, err_opt = true;
    std::vector<std::string> messages;
    // results
    RecordColumns rec;  // the last run's records in the reference's order (host memory of the workspace)
    uint64_t sun_rays = 0;
    int precision = ST_B200_FP64;
    bool want_records = true;
    int device = 0;
    std::vector<double> ex_pos, ex_cos;
    std::vector<FluxMap> flux;
    st_b200_stats stats;
    std::vector<std::vector<unsigned long long>> elem_first, elem_absorbed, elem_delivered;
    int (*cb)(unsigned long, unsigned long, unsigned long, unsigned long, unsigned long, void *) = nullptr;
    void *cbdata = nullptr;
    double last_hit_rate = 0.0;  // batch planning hint carried between runs of a context
    // stage data (st_b200_set_save_stage_data / st_b200_sim_run_replay, stapi.cpp:680-728)
    bool save_stage_data = false;
    std::vector<double> stage_s0, stage_s1;  // saved: 8 doubles per stage-1 record, 7 per ray
    bool replaying = false;
    std::vector<double> replay_s0, replay_s1;
    // the flattened scene of the last run and the exact key of the inputs it was built from:
    // a run whose inputs are unchanged reuses it (geometry set-up, grids and lists skipped)
    HostScene scene_cache;
    std::string scene_key;
    bool scene_valid = false;
    Workspace *ws = nullptr;     // device buffers reused by every run of this context
    // results of the last batched run (st_b200_sim_run_batch), per sun position
    std::vector<PositionResult> batch;
    std::vector<std::array<double, 4>> batch_box;  // sun box (xmin, xmax, ymin, ymax)
    st_b200_stats batch_stats;
    double sun_grid_cells = 4.0e6;  // cell budget of the sun-plane grid
    uint64_t max_sun64 = 0;  // st_b200_set_max_sun_rays: sun-ray cap beyond st_sim_params' int (0: unused)
    // this context's place in a run over several GPUs (st_b200_set_ranks)
    int rank = 0, nranks = 1;
    int (*allgather)(const unsigned long long *, unsigned long long *, int, void *) = nullptr;
    int (*allreduce)(unsigned long long *, unsigned long long, int, void *) = nullptr;
    void *comm_user = nullptr;
    ~Context() {
        if (ws) workspace_destroy(ws);
    }
    Context() {
        memset(&stats, 0, sizeof stats);
        memset(&batch_stats, 0, sizeof batch_stats);
    }
    void log(const char *fmt, ...) {
        char buf[513];
        va_list a;
        va_start(a, fmt);
        vsnprintf(buf, 512, fmt, a);
        va_end(a);
        messages.push_back(buf);
    }
};

// ---------------- math (mathproc.cpp:175-217, input.cpp:160-176) ----------------
void rot_from_euler(const double e[3], double R[9]) {
    const double ca = cos(e[0]), cb = cos(e[1]), cg = cos(e[2]);
    const double sa = sin(e[0]), sb = sin(e[1]), sg = sin(e[2]);
    R[0] = ca * cg + sa * sb * sg;
    R[1] = -cb * sg;
    R[2] = -sa * cg + ca * sb * sg;
    R[3] = ca * sg - sa * sb * cg;
    R[4] = cb * cg;
    R[5] = -sa * sg - ca * sb * cg;
    R[6] = sa * cb;
    R[7] = sb;
    R[8] = ca * cb;
}
bool euler_of(const double o[3], const double a[3], double zrot, double e[3]) {
    double dx = a[0] - o[0], dy = a[1] - o[1], dz = a[2] - o[2];
    const double d = sqrt(dx * dx + dy * dy + dz * dz);
    if (d == 0.0) return false;
    dx = dx / d;
    dy = dy / d;
    dz = dz / d;
    e[0] = atan2(dx, dz);
    e[1] = asin(dy);
    e[2] = zrot * kDegToRad;
    return true;
}
void mulv(const double R[9], const double v[3], double o[3]) {
    o[0] = R[0] * v[0] + R[1] * v[1] + R[2] * v[2];
    o[1] = R[3] * v[0] + R[4] * v[1] + R[5] * v[2];
    o[2] = R[6] * v[0] + R[7] * v[1] + R[8] * v[2];
}
inline double sq(double x) { return x * x; }

double mono_at(const Elem &e, double x, double y) {
    const int w = e.fit_order + 1;
    double z = 0.0;
    for (int i = 0; i <= e.fit_order; ++i)
        for (int j = 0; j <= i; ++j) {
            const double xx = (j == 0) ? 1.0 : pow(x, j);
            const double yy = (i - j == 0) ? 1.0 : pow(y, i - j);
            z = z + e.bcoef[i * w + j] * xx * yy;
        }
    return z;
}
double poly_at(const Elem &e, double r) {
    double z = 0.0;
    for (int i = 0; i <= e.fit_order; ++i) z = z + e.poly[i] * pow(r, i);
    return z;
}

// natural / end-slope cubic spline second derivatives (tridiagonal sweep)
void spline_y2(const std::vector<double> &x, const std::vector<double> &y, double yp1, double ypn,
               std::vector<double> &y2) {
    const int n = int(x.size());
    std::vector<double> u(n, 0.0);
    y2.assign(n, 0.0);
    if (n < 2) return;
    if (yp1 > 0.99e30) {
        y2[0] = 0.0;
        u[0] = 0.0;
    } else {
        y2[0] = -0.5;
        u[0] = (3.0 / (x[1] - x[0])) * ((y[1] - y[0]) / (x[1] - x[0]) - yp1);
    }
    for (int i = 1; i < n - 1; ++i) {
        const double sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]);
        const double p = sig * y2[i - 1] + 2.0;
        y2[i] = (sig - 1.0) / p;
        u[i] = (y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1]);
        u[i] = (6.0 * u[i] / (x[i + 1] - x[i - 1]) - sig * u[i - 1]) / p;
    }
    double qn = 0.0, un = 0.0;
    if (!(ypn > 0.99e30)) {
        qn = 0.5;
        un = (3.0 / (x[n - 1] - x[n - 2])) * (ypn - (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]));
    }
    y2[n - 1] = (un - qn * u[n - 2]) / (qn * y2[n - 2] + 1.0);
    for (int k = n - 2; k >= 0; --k) y2[k] = y2[k] * y2[k + 1] + u[k];
}

// ---------------- surface translation (input.cpp:288-366) ----------------
bool translate_surface(Context *cx, Elem &e, const double p[8]) {
    const bool line = (e.shape == 'l' || e.shape == 'L');
    switch (e.surface) {
        case 's':
        case 'S':
            e.vcx = p[0];
            e.vcy = line ? 0.0 : e.vcx;
            e.kappa = 1.0;
            e.stype = (e.vcy == 0.0) ? 7 : 1;
            return true;
        case 'p':
        case 'P':
            e.vcx = p[0];
            e.vcy = p[1];
            e.kappa = 0.0;
            e.stype = (e.vcy == 0.0) ? 7 : 1;
            return true;
        case 'o':
        case 'O':
            e.vcx = p[0];
            e.vcy = p[0];
            e.kappa = p[1];
            e.stype = (e.vcy == 0.0) ? 7 : 1;
            return true;
        case 'g':
        case 'G':
            e.vcx = p[0];
            e.vcy = p[1];
            e.kappa = p[2];
            for (int i = 0; i < 5; ++i) e.alpha[i] = p[3 + i];
            e.stype = (e.vcy == 0.0) ? 7 : 1;
            return true;
        case 'f':
        case 'F':
            e.alpha[0] = 0;
            e.alpha[1] = 0;
            e.alpha[2] = 1;
            e.alpha[3] = 0;
            e.alpha[4] = 0;
            e.stype = 3;
            return true;
        case 'c':
        case 'C':
            e.cone = p[0];
            e.stype = 1;
            return true;
        case 't':
        case 'T':
            if (!line || e.p[0] != 0.0 || e.p[1] != 0.0) {
                cx->log("Bad aperture or parameters of element not consistent with cylindrical surface\n");
                return false;
            }
            e.curv = p[0];
            e.vcx = e.curv;
            e.stype = 2;
            return true;
        case 'd':
        case 'D':
            if ((e.shape != 'a' && e.shape != 'A') || e.p[0] != 0.0 || e.p[1] != 0.0) {
                cx->log("Bad aperture or parameters of element not consistent with toroidal surface\n");
                return false;
            }
            e.ra = p[0];
            e.rs = p[1];
            e.stype = 10;
            return true;
        default:
            cx->log("invalid surface index: %c\n", e.surface);
            return false;
    }
}

// ---------------- ZAperture (apertureplane.cpp:57-491) ----------------
void aperture_plane(Elem &e) {
    const char sh = char(tolower(e.shape));
    double maxr = 0.0;
    if (sh == 'i' || sh == 'q') {
        maxr = sqrt(sq(e.p[0]) + sq(e.p[1]));
        maxr = std::max(maxr, sqrt(sq(e.p[2]) + sq(e.p[3])));
        maxr = std::max(maxr, sqrt(sq(e.p[4]) + sq(e.p[5])));
        if (sh == 'q') maxr = std::max(maxr, sqrt(sq(e.p[6]) + sq(e.p[7])));
    }
    // family: 1 circle/hexagon/triangle, 2 rectangle, 3 annulus/line, 4 irregular
    int fam = 0;
    double r2 = 0.0;
    if (sh == 'c' || sh == 'h' || sh == 't') {
        fam = 1;
        r2 = sq(e.p[0] / 2.0);
    } else if (sh == 'r') {
        fam = 2;
        r2 = sq(e.p[0] / 2.0) + sq(e.p[1] / 2.0);
    } else if (sh == 'a' || sh == 'l') {
        fam = 3;
        r2 = (fabs(e.p[1]) >= fabs(e.p[0])) ? sq(e.p[1]) : sq(e.p[0]);
    } else if (sh == 'i' || sh == 'q') {
        fam = 4;
        r2 = sq(maxr);
    }
    switch (tolower(e.surface)) {
        case 'g': {
            if (!fam) break;
            double sum = 0.0;
            if (fam == 1) {
                double rho = 1.0;
                for (int i = 0; i < 5; ++i) {
                    rho = rho * r2;
                    sum += e.alpha[i] * rho;
                }
                e.zap = e.vcx * r2 / (1 + sqrt(1 - e.kappa * e.vcx * e.vcx * r2)) + sum;
            } else {
                if (fam != 4)
                    for (int i = 0; i < 5; ++i) sum += e.alpha[i] * pow(r2, (int)(i + 1));
                e.zap = e.vcx * r2 / (1 + sqrt(1 - e.kappa * sq(e.vcx) * r2)) + sum;
            }
            break;
        }
        case 's':
            if (fam) {
                const double f = 1.0 / (2.0 * e.vcx);
                e.zap = 2.0 * f - sqrt(sq(2.0 * f) - r2);
            }
            break;
        case 'p':
            if (fam) e.zap = r2 / (4.0 * (1.0 / (2.0 * e.vcx)));
            break;
        case 'm':
            if (fam && e.fit_order >= 2) {
                const int w = e.fit_order + 1;
                const double f = (1.0 / (4.0 * e.bcoef[2 * w + 0]) + 1.0 / (4.0 * e.bcoef[2 * w + 2])) / 2.0;
                e.zap = r2 / (4.0 * f);
            }
            break;
        case 'f':
            e.zap = 0.0;
            break;
        case 'o':
            if (fam) e.zap = (1 - sqrt(1 - e.kappa * sq(e.vcx) * r2)) / (e.kappa * e.vcx);
            break;
        case 'c': {
            const double t = tan(e.cone * kDegToRad);
            if (fam == 1)
                e.zap = e.p[0] / (2.0 * t);
            else if (fam == 2 || fam == 4)
                e.zap = sqrt(r2) / (2.0 * t);
            else if (sh == 'a')
                e.zap = e.p[1] / t;
            break;
        }
        case 't':
            e.zap = 2.0 / e.curv;
            break;
        case 'd':
            e.zap = 2.0 * e.rs;
            break;
        case 'r':
            if (fam) e.zap = poly_at(e, fam == 1 ? e.p[0] / 2.0 : sqrt(r2));
            break;
        case 'i':
            if (!e.spl_y.empty()) e.zap = e.spl_y.back();
            break;
        case 'v': {
            double z = 0.0;
            for (int i = 0; i < e.vshot_rows; ++i) z = std::max(z, mono_at(e, e.vshot[5 * i], e.vshot[5 * i + 1]));
            e.zap = z;
            break;
        }
        case 'e': {
            double z = 0.0;  // the reference scans the nodes' second coordinate
            for (size_t i = 0; i + 2 < e.vshot.size(); i += 3) z = std::max(z, e.vshot[i + 1]);
            e.zap = z;
            break;
        }
        default:
            break;
    }
}

bool check_inputs(Context *cx) {  // input.cpp:87-150
    for (size_t i = 0; i < cx->stages.size(); ++i)
        for (size_t j = 0; j < cx->stages[i].elems.size(); ++j) {
            const Elem &e = cx->stages[i].elems[j];
            const bool pp = e.surface == 'p' || e.surface == 'P', ss = e.surface == 's' || e.surface == 'S';
            const bool line = e.shape == 'l' || e.shape == 'L';
            if (pp && line && e.vcy != 0.0) {
                cx->log("Parabolic surface combined with single axis curvature section aperture must have Cy = 0.  Element %d Stage %d.",
                        int(j + 1), int(i + 1));
                return false;
            }
            if (ss && e.vcx == 0.0) {
                cx->log("Spherical surface must have a curvature greater than 0.0.  Consider using a flat surface instead. Element %d, Stage %d.",
                        int(j + 1), int(i + 1));
                return false;
            }
            if (ss && e.vcy != 0.0 && e.vcy != e.vcx) {
                cx->log("Spherical surface must have Cy=0 or Cy=Cx.  Currently, Cy=%lg for Element %d, Stage %d", e.vcy,
                        int(j + 1), int(i + 1));
                return false;
            }
            if ((e.surface == 'o' || e.surface == 'O') && (e.kappa == 1.0 || e.kappa == 0.0)) {
                cx->log("Kappa = 0.0 or 1.0 defines either a parabola or a sphere.  Use the specific surface definition for either of those cases. Element %d, Stage %d.",
                        int(j + 1), int(i + 1));
                return false;
            }
        }
    return true;
}

bool init_geometries(Context *cx) {  // input.cpp:153-286
    for (size_t i = 0; i < cx->stages.size(); ++i) {
        StageM &st = cx->stages[i];
        double eu[3];
        if (!euler_of(st.origin, st.aim, st.zrot, eu)) {
            cx->log("Stage %d geometry as defined not possible.\n", int(i));
            return false;
        }
        rot_from_euler(eu, st.R);
        for (size_t j = 0; j < st.elems.size(); ++j) {
            Elem &e = st.elems[j];
            if (!euler_of(e.origin, e.aim, e.zrot, eu)) {
                cx->log("Stage %d element %d geometry as defined not possible.\n", int(i), int(j));
                return false;
            }
            rot_from_euler(eu, e.R);
            const double *p = e.p;
            switch (e.shape) {
                case 'c':
                case 'C':
                    e.area = kPi * sq(p[0] / 2);
                    break;
                case 'h':
                case 'H':
                    e.area = 5.0 * sq(p[0] / 2.0) * cos(30.0 * kDegToRad) * sin(30.0 * kDegToRad);
                    break;
                case 'r':
                case 'R':
                    e.area = p[0] * p[1];
                    break;
                case 't':
                case 'T':
                    e.area = 0.25 * sq(p[0] * cos(30.0 * kDegToRad)) * sqrt(3.0);
                    break;
                case 'a':
                case 'A':
                    e.area = p[2] * kDegToRad * (p[1] - p[0]);
                    break;
                case 'l':
                case 'L':
                    e.area = (p[1] - p[0]) * p[2];
                    break;
                case 'i':
                case 'I': {
                    const double v11 = p[0] - p[2], v12 = p[1] - p[3], v21 = p[4] - p[2], v22 = p[5] - p[3];
                    const double a = sqrt(v11 * v11 + v12 * v12), b = sqrt(v21 * v21 + v22 * v22);
                    e.area = 0.5 * a * b * sin(acos((v11 * v21 + v12 * v22) / (a * b)));
                    break;
                }
                case 'q':
                case 'Q': {
                    const double v11 = p[0] - p[2], v12 = p[1] - p[3], v21 = p[4] - p[2], v22 = p[5] - p[3];
                    const double v31 = p[4] - p[6], v32 = p[5] - p[7], v41 = p[0] - p[6], v42 = p[1] - p[7];
                    const double a = sqrt(v11 * v11 + v12 * v12), b = sqrt(v21 * v21 + v22 * v22);
                    const double c = sqrt(v31 * v31 + v32 * v32), d = sqrt(v41 * v41 + v42 * v42);
                    e.area = 0.5 * (a * b * sin(acos((v11 * v21 + v12 * v22) / (a * b))) +
                                    c * d * sin(acos((v31 * v41 + v32 * v42) / (c * d))));
                    break;
                }
                default:
                    cx->log("invalid shape '%c' for aperture, element %d\n", e.shape, int(j));
                    return false;
            }
            if (!st.virt) {
                int found = -1;
                for (size_t k = 0; k < cx->optics.size(); ++k)
                    if (strcasecmp(cx->optics[k].name.c_str(), e.optic.c_str()) == 0) found = int(k);
                if (found < 0) {
                    cx->log("Stage %d element %d invalid optical property set name: '%s'\n", int(i), int(j),
                            e.optic.c_str());
                    return false;
                }
                e.optic_idx = found;
                OpticSet &set = cx->optics[found];
                set.front.n[2] = set.back.n[0];
                set.front.n[3] = set.back.n[1];
                set.back.n[2] = set.front.n[0];
                set.back.n[3] = set.front.n[1];
            } else {
                e.optic_idx = -1;
            }
            aperture_plane(e);
        }
    }
    return check_inputs(cx);
}

// Radius about the element origin that contains every hit the trace can accept,
// or -1 when no finite bound is known for the surface (those elements are tested
// for every ray).  Used to build the sun-plane grid and the stage BVHs.
double accept_radius(const Elem &e) {
    const char sh = char(tolower(e.shape));
    double rap;
    switch (sh) {
        case 'c':
        case 'h':
            rap = e.p[0] / 2.0;
            break;
        case 't':
            rap = e.p[0] / 2.0;
            break;
        case 'r':
            rap = 0.5 * sqrt(sq(e.p[0]) + sq(e.p[1]));
            break;
        case 'a':
            rap = std::max(fabs(e.p[0]), fabs(e.p[1]));
            break;
        case 'l':
            // x1 = x2 = 0 leaves x unbounded (intersect.cpp applies no x limit then): only the
            // closed cylinder and torus below stay bounded
            if (e.p[0] == 0.0 && e.p[1] == 0.0 && e.stype != 2 && e.stype != 10) return -1.0;
            rap = sqrt(sq(std::max(fabs(e.p[0]), fabs(e.p[1]))) + sq(e.p[2] / 2.0));
            break;
        case 'i':
        case 'q': {
            rap = 0;
            for (int k = 0; k < (sh == 'q' ? 8 : 6); k += 2) rap = std::max(rap, sqrt(sq(e.p[k]) + sq(e.p[k + 1])));
            break;
        }
        default:
            return -1.0;
    }
    const int s = tolower(e.surface);
    double zext;
    if (e.stype == 3) {
        zext = 0.0;
    } else if (s == 'p' && e.stype != 2) {
        // z = (Cx x^2 + Cy y^2)/2 on the surface, for (x, y) inside the aperture
        zext = 0.5 * std::max(fabs(e.vcx), fabs(e.vcy)) * rap * rap;
    } else if (e.stype == 2) {
        // cylinder about the local y axis through (0, y, r): |x| <= r, 0 <= z <= 2r
        const double r = fabs(1.0 / e.curv);
        return sqrt(sq(r) + sq(e.p[2] / 2.0) + sq(2.0 * r)) * (1.0 + 1e-9) + 1e-6;
    } else if (e.stype == 10) {
        return sqrt(sq(fabs(e.ra) + fabs(e.rs)) + sq(2.0 * fabs(e.rs))) * (1.0 + 1e-9) + 1e-6;
    } else if (s == 's' && e.vcx > 0.0) {
        // accepted hits satisfy z <= ZAperture on the lower cap (0 <= z)
        zext = std::max(fabs(e.zap), 0.0);
    } else {
        return -1.0;
    }
    return sqrt(rap * rap + zext * zext) * (1.0 + 1e-9) + 1e-6;
}

// Element-local box [x0,x1] x [y0,y1] x [-hz,hz] holding every hit the trace can accept,
// for elements whose accepted hits lie on a surface of bounded sag over the aperture
// (flat, parabolic and spherical-cap sections); false otherwise.
bool local_box(const Elem &e, double &x0, double &x1, double &y0, double &y1, double &hz) {
    const double rb = accept_radius(e);
    if (rb < 0) return false;
    if (e.stype == 2 || e.stype == 10) return false;  // cylinder, torus: the radius bound only
    const char sh = char(tolower(e.shape));
    switch (sh) {
        case 'r':
            x0 = -e.p[0] / 2.0;
            x1 = e.p[0] / 2.0;
            y0 = -e.p[1] / 2.0;
            y1 = e.p[1] / 2.0;
            break;
        case 'l':
            x0 = std::min(e.p[0], e.p[1]);
            x1 = std::max(e.p[0], e.p[1]);
            y0 = -fabs(e.p[2]) / 2.0;
            y1 = fabs(e.p[2]) / 2.0;
            break;
        case 'i':
        case 'q':
            x0 = y0 = 1e300;
            x1 = y1 = -1e300;
            for (int k = 0; k < (sh == 'q' ? 8 : 6); k += 2) {
                x0 = std::min(x0, e.p[k]);
                x1 = std::max(x1, e.p[k]);
                y0 = std::min(y0, e.p[k + 1]);
                y1 = std::max(y1, e.p[k + 1]);
            }
            break;
        case 'a': {
            const double ra = std::max(fabs(e.p[0]), fabs(e.p[1]));
            x0 = y0 = -ra;
            x1 = y1 = ra;
            break;
        }
        default: {  // 'c', 'h', 't': inside the circle of diameter p0
            const double ra = fabs(e.p[0]) / 2.0;
            x0 = y0 = -ra;
            x1 = y1 = ra;
        }
    }
    // sag over the aperture, as accept_radius bounds it: 0 for flat elements, the paraboloid's
    // z at the farthest aperture corner, ZAperture for spherical caps
    const double rxy2 = std::max(sq(x0), sq(x1)) + std::max(sq(y0), sq(y1));
    if (e.stype == 3)
        hz = 0.0;
    else if (tolower(e.surface) == 'p')
        hz = 0.5 * std::max(fabs(e.vcx), fabs(e.vcy)) * rxy2 * (1.0 + 1e-9) + 1e-9;
    else
        hz = std::max(fabs(e.zap), 0.0) * (1.0 + 1e-9) + 1e-9;
    return true;
}

// Ground grid of a stage whose elements are spread over its x-y plane in a thin z band
// (z extent at most a quarter of the x-y extent, every element bounded).  Cells are about
// one element radius wide; an enabled element is listed in every cell its bounding disc,
// padded by 1e-3 of a cell plus 1e-6 of the coordinates (float traversal), overlaps, with
// its float bounding sphere beside it so that the walk reads one entry per element.  The z
// band and the grid box carry the same padding.  Returns false (grid off) otherwise.
bool build_ground_grid(const std::vector<Elem> &els, const float4 *sphere, StageRec &sr, std::vector<int2> &cells,
                       std::vector<float4> &ent_sphere, std::vector<int> &ent_elem) {
    const size_t n = els.size();
    std::vector<double> rad(n);
    double xlo = 1e300, xhi = -1e300, ylo = 1e300, yhi = -1e300, zlo = 1e300, zhi = -1e300;
    for (size_t j = 0; j < n; ++j) {
        const double r = accept_radius(els[j]);
        if (r < 0) return false;
        rad[j] = r;
        const double *c = els[j].origin;
        xlo = std::min(xlo, c[0] - r);
        xhi = std::max(xhi, c[0] + r);
        ylo = std::min(ylo, c[1] - r);
        yhi = std::max(yhi, c[1] + r);
        zlo = std::min(zlo, c[2] - r);
        zhi = std::max(zhi, c[2] + r);
    }
    const double ext = std::max(xhi - xlo, yhi - ylo);
    if (!(ext > 0) || (zhi - zlo) > 0.25 * ext) return false;
    std::vector<double> rs = rad;
    std::nth_element(rs.begin(), rs.begin() + n / 2, rs.end());
    double cell = std::max(rs[n / 2], ext / 4096.0);
    if (!(cell > 0)) return false;
    const double big = std::max(std::max(fabs(xlo), fabs(xhi)), std::max(fabs(ylo), fabs(yhi)));
    double gx0, gy0;
    int nx, ny;
    for (;;) {
        const double m = 1e-3 * cell + 1e-6 * big + 1e-6 + 0.5 * cell;  // margin around the padded discs
        gx0 = xlo - m;
        gy0 = ylo - m;
        nx = int(ceil((xhi - xlo + 2 * m) / cell)) + 1;
        ny = int(ceil((yhi - ylo + 2 * m) / cell)) + 1;
        if (double(nx) * ny <= 1.0e6) break;
        cell *= 1.5;
    }
    std::vector<std::vector<int>> lists(size_t(nx) * ny);
    for (size_t j = 0; j < n; ++j) {
        if (!els[j].enabled) continue;
        const double *c = els[j].origin;
        const double pad = rad[j] * (1.0 + 1e-6) + 1e-3 * cell + 1e-6 * big + 1e-6;
        const int x0 = std::max(0, int(floor((c[0] - pad - gx0) / cell)));
        const int x1 = std::min(nx - 1, int(floor((c[0] + pad - gx0) / cell)));
        const int y0 = std::max(0, int(floor((c[1] - pad - gy0) / cell)));
        const int y1 = std::min(ny - 1, int(floor((c[1] + pad - gy0) / cell)));
        for (int gy = y0; gy <= y1; ++gy)
            for (int gx = x0; gx <= x1; ++gx) {
                const double ax = gx0 + gx * cell, bx = ax + cell, ay = gy0 + gy * cell, by = ay + cell;
                const double dx = std::max(std::max(ax - c[0], 0.0), c[0] - bx);
                const double dy = std::max(std::max(ay - c[1], 0.0), c[1] - by);
                if (dx * dx + dy * dy <= pad * pad) lists[size_t(gy) * nx + gx].push_back(int(j));
            }
    }
    const double zpad = 1e-3 * (zhi - zlo) + 1e-3 + 1e-6 * std::max(fabs(zlo), fabs(zhi));
    sr.grid_on = 1;
    sr.gnx = nx;
    sr.gny = ny;
    sr.gcell_off = int(cells.size());
    sr.gx0 = float(gx0);
    sr.gy0 = float(gy0);
    sr.gcell = float(cell);
    sr.ginv = float(1.0 / cell);
    sr.gzlo = float(zlo - zpad);
    sr.gzhi = float(zhi + zpad);
    for (const auto &l : lists) {
        const int a = int(ent_elem.size());
        for (int j : l) {
            ent_elem.push_back(j);
            ent_sphere.push_back(sphere[j]);
        }
        cells.push_back(int2{a, int(ent_elem.size())});
    }
    return true;
}

// Zone table of a finite-element surface for the device (st_device.cuh fe_eval), the
// neighbourhoods the reference's st_hash_tree gives its nodes (input.cpp:538-556,
// treemesh.cpp:353-535): the nodes' bounding box halved floor(log2(extent / zone)) >= 1
// times per axis, zone = 1.5 sqrt(area per node); a query in zone (ix, iy) considers the
// nodes of that zone, then of its 8 neighbours (x offset outer, y inner).  Layout, in
// doubles: N, levels x, levels y, xmin, xmax, ymin, ymax, zone count Z, Z + 1 list starts,
// the lists (node indices), the nodes (x, y, z).
void fe_table(const std::vector<double> &nodes, std::vector<double> &out) {
    const size_t n = nodes.size() / 3;
    double xmin = std::numeric_limits<double>::max(), ymin = xmin, xmax = -xmin, ymax = -xmin;
    for (size_t i = 0; i < n; ++i) {
        const double x = nodes[3 * i], y = nodes[3 * i + 1];
        xmax = x > xmax ? x : xmax;
        ymax = y > ymax ? y : ymax;
        xmin = x < xmin ? x : xmin;
        ymin = y < ymin ? y : ymin;
    }
    const double zone = 1.5 * sqrt(((xmax - xmin) * (ymax - ymin)) / (double)std::max<size_t>(n, 1));
    const double inv_ln2 = 1. / log(2.);
    const int lx = std::max(1, (int)floor(log((xmax - xmin) / zone) * inv_ln2));
    const int ly = std::max(1, (int)floor(log((ymax - ymin) / zone) * inv_ln2));
    const int nx = 1 << std::min(lx, 12), ny = 1 << std::min(ly, 12);
    auto zone_of = [&](double x, double y) {
        double x0 = xmin, x1 = xmax, y0 = ymin, y1 = ymax;
        int ix = 0, iy = 0;
        for (int k = 0; k < lx && k < 12; ++k) {
            const double c = (x0 + x1) * 0.5;
            if (x > c) x0 = c, ix = 2 * ix + 1;
            else x1 = c, ix = 2 * ix;
        }
        for (int k = 0; k < ly && k < 12; ++k) {
            const double c = (y0 + y1) * 0.5;
            if (y > c) y0 = c, iy = 2 * iy + 1;
            else y1 = c, iy = 2 * iy;
        }
        return iy * nx + ix;
    };
    std::vector<std::vector<int>> own(size_t(nx) * ny);
    for (size_t i = 0; i < n; ++i) own[zone_of(nodes[3 * i], nodes[3 * i + 1])].push_back(int(i));
    std::vector<double> starts, items;
    for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
            starts.push_back(double(items.size()));
            for (int i : own[size_t(iy) * nx + ix]) items.push_back(i);
            for (int dx = -1; dx < 2; ++dx)
                for (int dy = -1; dy < 2; ++dy) {
                    const int jx = ix + dx, jy = iy + dy;
                    if ((dx == 0 && dy == 0) || jx < 0 || jx >= nx || jy < 0 || jy >= ny) continue;
                    for (int i : own[size_t(jy) * nx + jx]) items.push_back(i);
                }
        }
    starts.push_back(double(items.size()));
    const double head[8] = {double(n), double(std::min(lx, 12)), double(std::min(ly, 12)), xmin, xmax, ymin, ymax,
                            double(nx) * ny};
    out.insert(out.end(), head, head + 8);
    out.insert(out.end(), starts.begin(), starts.end());
    out.insert(out.end(), items.begin(), items.end());
    out.insert(out.end(), nodes.begin(), nodes.begin() + 3 * n);
}

// Outgoing-beam candidate lists of the first stage's flat elements (heliostat fields).
//
// A sun ray reflected by a flat element leaves it close to the mirror image of the sun
// direction about the element's normal: sunshape, slope and specularity errors move it by
// tens of milliradians at most.  For every flat element j of a first stage with a ground
// grid and a directional sun, the list holds every element k whose padded bounding sphere
// meets the volume swept by rays that start inside j's bounding sphere with a direction
// within kBeamHalfAngle of that axis, up to where such rays leave the stage's z band.  A ray
// leaving j inside the cone (checked per ray, in float with 1e-3 rad of margin in the
// lists) is searched against the list; any other ray walks the ground grid.  Lists longer
// than kBeamMaxList are not kept.
constexpr double kBeamHalfAngle = 0.1;  // rad
constexpr size_t kBeamMaxList = 256;

void build_beam_lists(Context *cx, HostScene &hs) {
    const size_t ne = hs.elems.size();
    hs.beam_axis.assign(ne, float4{0.f, 0.f, 0.f, 2.f});
    hs.beam_range.assign(ne, int2{0, 0});
    hs.beam_elem.clear();
    StageRec &sr = hs.dev.stages[0];
    if (cx->sun.point_source || !sr.grid_on || !sr.multihit) return;
    const StageM &st = cx->stages[0];
    const double *Rs = hs.dev.sun.Rsun;
    const double din[3] = {Rs[6], Rs[7], Rs[8]};  // sun-ray direction in the stage frame
    const double th = kBeamHalfAngle + 1e-3, tan_th = tan(th);
    const double zlo = sr.gzlo, zhi = sr.gzhi;
    const size_t n = st.elems.size();
    std::vector<double> rad(n);
    for (size_t k = 0; k < n; ++k) {
        const double r = accept_radius(st.elems[k]);
        const double *c = st.elems[k].origin;
        rad[k] = r < 0 ? -1.0 : r * (1.0 + 1e-6) + 1e-3 + 1e-6 * (fabs(c[0]) + fabs(c[1]) + fabs(c[2]));
    }
    // centres binned on an x-y grid, so that each list only examines elements within its
    // reach; elements without a finite bound are examined by every list
    double rmax = 0, xlo = 1e300, ylo = 1e300, xhi = -1e300, yhi = -1e300;
    std::vector<int> unbounded;
    for (size_t k = 0; k < n; ++k) {
        if (rad[k] < 0) {
            unbounded.push_back(int(k));
            continue;
        }
        rmax = std::max(rmax, rad[k]);
        xlo = std::min(xlo, st.elems[k].origin[0]);
        xhi = std::max(xhi, st.elems[k].origin[0]);
        ylo = std::min(ylo, st.elems[k].origin[1]);
        yhi = std::max(yhi, st.elems[k].origin[1]);
    }
    const double bin = std::max(4.0 * rmax, std::max(xhi - xlo, yhi - ylo) / 1024.0) + 1e-9;
    const int bnx = xhi >= xlo ? int((xhi - xlo) / bin) + 1 : 1, bny = yhi >= ylo ? int((yhi - ylo) / bin) + 1 : 1;
    std::vector<std::vector<int>> bins(size_t(bnx) * bny);
    for (size_t k = 0; k < n; ++k)
        if (rad[k] >= 0)
            bins[size_t(int((st.elems[k].origin[1] - ylo) / bin)) * bnx + int((st.elems[k].origin[0] - xlo) / bin)]
                .push_back(int(k));
    std::vector<int> list, cand;
    for (size_t j = 0; j < n; ++j) {
        const Elem &e = st.elems[j];
        if (e.stype != 3 || !e.enabled || rad[j] < 0) continue;
        const double nrm[3] = {e.R[6], e.R[7], e.R[8]};
        const double dn = din[0] * nrm[0] + din[1] * nrm[1] + din[2] * nrm[2];
        double a[3] = {din[0] - 2.0 * dn * nrm[0], din[1] - 2.0 * dn * nrm[1], din[2] - 2.0 * dn * nrm[2]};
        const double la = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        if (!(la > 0)) continue;
        for (double &v : a) v /= la;
        // how far along the beam a ray can still be inside the z band
        const double elev = asin(std::max(-1.0, std::min(1.0, a[2])));
        const double *cj = e.origin;
        double s_max = 1e300;
        if (elev - th > 0) s_max = (zhi - (cj[2] - rad[j])) / sin(elev - th);
        else if (elev + th < 0) s_max = ((cj[2] + rad[j]) - zlo) / sin(-(elev + th));
        // elements whose centre is within reach of the beam's in-band part
        cand.assign(unbounded.begin(), unbounded.end());
        const double reach = s_max + 2.0 * rad[j] + rmax;
        if (reach >= 1e299 || reach / bin > bnx + bny) {
            for (size_t k = 0; k < n; ++k)
                if (rad[k] >= 0) cand.push_back(int(k));
        } else {
            const int x0 = std::max(0, int((cj[0] - reach - xlo) / bin)), x1 = std::min(bnx - 1, int((cj[0] + reach - xlo) / bin));
            const int y0 = std::max(0, int((cj[1] - reach - ylo) / bin)), y1 = std::min(bny - 1, int((cj[1] + reach - ylo) / bin));
            for (int by = y0; by <= y1; ++by)
                for (int bx = x0; bx <= x1; ++bx)
                    for (int k : bins[size_t(by) * bnx + bx]) cand.push_back(k);
        }
        list.clear();
        bool too_long = false;
        for (size_t q = 0; q < cand.size() && !too_long; ++q) {
            const size_t k = size_t(cand[q]);
            if (k == j || !st.elems[k].enabled) continue;
            const double rk = rad[k] < 0 ? 1e300 : rad[k];
            const double *ck = st.elems[k].origin;
            const double v[3] = {ck[0] - cj[0], ck[1] - cj[1], ck[2] - cj[2]};
            const double t = v[0] * a[0] + v[1] * a[1] + v[2] * a[2];
            if (t < -(rad[j] + rk) || t - rk > rad[j] + s_max) continue;
            const double w[3] = {v[0] - t * a[0], v[1] - t * a[1], v[2] - t * a[2]};
            const double p = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
            if (p > rk + rad[j] + (std::max(t, 0.0) + rk + rad[j]) * tan_th) continue;
            list.push_back(int(k));
            too_long = list.size() > kBeamMaxList;
        }
        if (too_long) continue;
        const size_t g = size_t(sr.first_elem) + j;
        hs.beam_axis[g] = float4{float(a[0]), float(a[1]), float(a[2]), float(cos(kBeamHalfAngle))};
        hs.beam_range[g] = int2{int(hs.beam_elem.size()), int(hs.beam_elem.size() + list.size())};
        hs.beam_elem.insert(hs.beam_elem.end(), list.begin(), list.end());
    }
}

// Median-split BVH over element bounding spheres (stage coordinates).
void build_bvh(const std::vector<Elem> &els, std::vector<BvhNode> &nodes, std::vector<int> &items) {
    struct Item {
        int j;
        double c[3], r;
    };
    std::vector<Item> its;
    for (size_t j = 0; j < els.size(); ++j) {
        const double r = accept_radius(els[j]);
        Item it;
        it.j = int(j);
        for (int q = 0; q < 3; ++q) it.c[q] = els[j].origin[q];
        it.r = (r < 0) ? 1e30 : r;  // unbounded elements get an all-space box
        its.push_back(it);
    }
    const size_t base = nodes.size();
    (void)base;
    struct Task {
        int node, lo, hi;
    };
    auto box = [&](int lo, int hi, BvhNode &nd) {
        double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
        for (int k = lo; k < hi; ++k)
            for (int q = 0; q < 3; ++q) {
                mn[q] = std::min(mn[q], its[k].c[q] - its[k].r);
                mx[q] = std::max(mx[q], its[k].c[q] + its[k].r);
            }
        for (int q = 0; q < 3; ++q) {
            // pad for the float traversal: 1 mm plus 1e-6 of the coordinate
            const double pl = 1e-3 + 1e-6 * fabs(mn[q]), ph = 1e-3 + 1e-6 * fabs(mx[q]);
            nd.lo[q] = float(std::max(mn[q] - pl, -3.0e38));
            nd.hi[q] = float(std::min(mx[q] + ph, 3.0e38));
            nd.lo[q] = std::nextafter(nd.lo[q], -INFINITY);
            nd.hi[q] = std::nextafter(nd.hi[q], INFINITY);
        }
    };
    std::vector<BvhNode> out(1);
    std::vector<Task> todo{{0, 0, int(its.size())}};
    while (!todo.empty()) {
        Task t = todo.back();
        todo.pop_back();
        BvhNode nd;
        box(t.lo, t.hi, nd);
        if (t.hi - t.lo <= 4) {
            nd.first = t.lo;
            nd.count = t.hi - t.lo;
            out[t.node] = nd;
            continue;
        }
        double cmn[3] = {1e300, 1e300, 1e300}, cmx[3] = {-1e300, -1e300, -1e300};
        for (int k = t.lo; k < t.hi; ++k)
            for (int q = 0; q < 3; ++q) {
                cmn[q] = std::min(cmn[q], its[k].c[q]);
                cmx[q] = std::max(cmx[q], its[k].c[q]);
            }
        int ax = 0;
        for (int q = 1; q < 3; ++q)
            if (cmx[q] - cmn[q] > cmx[ax] - cmn[ax]) ax = q;
        const int mid = (t.lo + t.hi) / 2;
        std::nth_element(its.begin() + t.lo, its.begin() + mid, its.begin() + t.hi,
                         [ax](const Item &a, const Item &b) { return a.c[ax] < b.c[ax]; });
        const int left = int(out.size());
        out.push_back(BvhNode());
        out.push_back(BvhNode());
        nd.first = left;
        nd.count = 0;
        out[t.node] = nd;
        todo.push_back({left + 1, mid, t.hi});
        todo.push_back({left, t.lo, mid});
    }
    nodes.insert(nodes.end(), out.begin(), out.end());
    for (auto &it : its) items.push_back(it.j);
}

// ---------------- the sun frame and sun box (suntoprimarystage.cpp:59-293) ----------------
bool sun_setup(Context *cx, HostScene &hs) {
    StageM &st = cx->stages[0];
    SunM &sun = cx->sun;
    const double dx = 0.0 - sun.origin[0], dy = 0.0 - sun.origin[1], dz = 0.0 - sun.origin[2];
    const double dt = sqrt(dx * dx + dy * dy + dz * dz);
    if (dt == 0.0) {
        cx->log("error calculating sun position in primary stage, dtot = 0.0\n");
        return false;
    }
    const double cg[3] = {dx / dt, dy / dt, dz / dt};
    double cs[3];
    mulv(st.R, cg, cs);
    const double se[3] = {atan2(cs[0], cs[2]), asin(cs[1]), 0.0};
    double Rs[9];
    rot_from_euler(se, Rs);
    sun.xmax = -1.0e20;
    sun.xmin = 1.0e20;
    sun.ymax = -1.0e20;
    sun.ymin = 1.0e20;
    const double cd[3] = {0, 0, 1};
    (void)cd;
    size_t n = 0;
    for (const Elem &e : st.elems) {
        if (!e.enabled) continue;
        double pl[3];
        mulv(Rs, e.origin, pl);
        double ext = 0.0;
        const double *p = e.p;
        switch (e.shape) {
            case 'c':
            case 'C':
            case 'h':
            case 'H':
                ext = p[0] / 2.0;
                break;
            case 'r':
            case 'R':
                ext = sqrt((p[0] * p[0] + p[1] * p[1]) / 4.0);
                break;
            case 't':
            case 'T':
                ext = p[0] / (2.0 * cos(30.0 * kDegToRad));
                break;
            case 'a':
            case 'A':
                ext = p[1];
                break;
            case 'l':
            case 'L': {
                const double leg = (fabs(p[1]) >= fabs(p[0])) ? p[1] : p[0];
                ext = sqrt(leg * leg + 0.25 * p[2] * p[2]);
                break;
            }
            case 'i':
            case 'I':
            case 'q':
            case 'Q': {
                double m = sqrt(p[0] * p[0] + p[1] * p[1]);
                m = std::max(m, sqrt(p[2] * p[2] + p[3] * p[3]));
                m = std::max(m, sqrt(p[4] * p[4] + p[5] * p[5]));
                if (e.shape == 'q' || e.shape == 'Q') m = std::max(m, sqrt(p[6] * p[6] + p[7] * p[7]));
                ext = m;
                break;
            }
            default:
                break;
        }
        if (pl[0] - ext < sun.xmin) sun.xmin = pl[0] - ext;
        if (pl[0] + ext > sun.xmax) sun.xmax = pl[0] + ext;
        if (pl[1] - ext < sun.ymin) sun.ymin = pl[1] - ext;
        if (pl[1] + ext > sun.ymax) sun.ymax = pl[1] + ext;
        n++;
    }
    if (n == 0) {
        cx->log("error calculating sun position in primary stage because no elements were enabled");
        return false;
    }
    SunDev &sd = hs.dev.sun;
    sd.xmin = sun.xmin;
    sd.xmax = sun.xmax;
    sd.ymin = sun.ymin;
    sd.ymax = sun.ymax;
    for (int k = 0; k < 9; ++k) sd.Rsun[k] = Rs[k];
    for (int k = 0; k < 3; ++k) {
        sd.pos_sun_stage[k] = 0.0;  // the sun frame is centred on the first stage's origin
        sd.origin[k] = sun.origin[k];
    }
    sd.shape = sun.shape;
    sd.point_source = sun.point_source ? 1 : 0;
    sd.sigma = sun.sigma;

    // Inverse CDF of p(theta) ~ theta * I(theta) on [0, MaxAngle] for table sunshapes:
    // trapezoid CDF on kSunCdfCells cells, then theta(u) tabulated at kSunInvCells + 1
    // equally spaced probabilities so that a sample costs one interpolation.
    hs.inv_cdf.clear();
    if (sun.ang.size() >= 3 && sun.max_angle > 0) {
        auto intensity = [&](double th) {
            size_t i = 0;
            while (i < sun.ang.size() - 1 && sun.ang[i] < th) i++;
            if (i == 0) return sun.inten[0];
            return sun.inten[i - 1] + (sun.inten[i] - sun.inten[i - 1]) * (th - sun.ang[i - 1]) / (sun.ang[i] - sun.ang[i - 1]);
        };
        const int K = kSunCdfCells, KI = kSunInvCells;
        std::vector<double> th(K + 1, 0.0), cdf(K + 1, 0.0);
        const double dth = sun.max_angle / K;
        double prev = 0.0;
        for (int j = 0; j <= K; ++j) {
            th[j] = dth * j;
            const double pdf = th[j] * intensity(th[j]);
            if (j > 0) cdf[j] = cdf[j - 1] + 0.5 * (prev + pdf) * dth;
            prev = pdf;
        }
        const double tot = cdf[K];
        for (int j = 0; j <= K; ++j) cdf[j] = tot > 0 ? cdf[j] / tot : 0.0;
        hs.inv_cdf.assign(KI + 1, 0.0);
        for (int j = 0; j <= KI; ++j) {
            const double u = double(j) / KI;
            int lo = 0, hi = K;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (cdf[mid] <= u)
                    lo = mid;
                else
                    hi = mid;
            }
            const double f = (cdf[hi] > cdf[lo]) ? (u - cdf[lo]) / (cdf[hi] - cdf[lo]) : 0.0;
            hs.inv_cdf[j] = th[lo] + f * (th[hi] - th[lo]);
        }
    }

    // sun-plane grid over the first stage: every element whose bounding disc (centre
    // = projected origin, radius = accept radius) overlaps a cell is listed there
    sd.grid_on = 0;
    sd.exact_flat = 0;
    hs.cell_start.assign(2, 0);
    hs.cell_disc.clear();
    hs.cell_par.clear();
    hs.cell_xa.clear();
    hs.cell_xb.clear();
    hs.cell_xc.clear();
    if (!sun.point_source && st.elems.size() >= 4) {
        bool bounded = true;
        double rmax = 0;
        std::vector<double> rad(st.elems.size()), cx_(st.elems.size()), cy_(st.elems.size());
        for (size_t j = 0; j < st.elems.size(); ++j) {
            const double r = accept_radius(st.elems[j]);
            if (r < 0) {
                bounded = false;
                break;
            }
            double pl[3];
            mulv(Rs, st.elems[j].origin, pl);
            rad[j] = r;
            cx_[j] = pl[0];
            cy_[j] = pl[1];
            rmax = std::max(rmax, r);
        }
        if (bounded && rmax > 0) {
            const double W = sun.xmax - sun.xmin, H = sun.ymax - sun.ymin;
            double cell = std::max(rmax * 0.5, 1e-6);
            // keep the grid within the context's cell budget (~4M cells for a single run)
            while ((W / cell + 1) * (H / cell + 1) > cx->sun_grid_cells) cell *= 1.5;
            const int nx = std::max(1, int(ceil(W / cell))), ny = std::max(1, int(ceil(H / cell)));
            std::vector<std::vector<int>> cells(size_t(nx) * ny);
            for (size_t j = 0; j < st.elems.size(); ++j) {
                const double pad = rad[j] * (1.0 + 1e-9) + 1e-6 * (1.0 + fabs(cx_[j]) + fabs(cy_[j]));
                const int x0 = std::max(0, int(floor((cx_[j] - pad - sun.xmin) / cell)));
                const int x1 = std::min(nx - 1, int(floor((cx_[j] + pad - sun.xmin) / cell)));
                const int y0 = std::max(0, int(floor((cy_[j] - pad - sun.ymin) / cell)));
                const int y1 = std::min(ny - 1, int(floor((cy_[j] + pad - sun.ymin) / cell)));
                for (int gy = y0; gy <= y1; ++gy)
                    for (int gx = x0; gx <= x1; ++gx) {
                        // distance from the disc centre to the cell rectangle
                        const double ax = sun.xmin + gx * cell, bx = ax + cell;
                        const double ay = sun.ymin + gy * cell, by = ay + cell;
                        const double ddx = std::max(std::max(ax - cx_[j], 0.0), cx_[j] - bx);
                        const double ddy = std::max(std::max(ay - cy_[j], 0.0), cy_[j] - by);
                        if (ddx * ddx + ddy * ddy <= pad * pad) cells[size_t(gy) * nx + gx].push_back(int(j));
                    }
            }
            // Per element a float disc (centre, radius) and a parallelogram about the same
            // centre for the probe's pre-tests; both contain every sun-plane point whose ray can
            // be accepted by the element.
            //
            // Parallelogram: the projection (along the sun's z) of the element's local box lies
            // inside the parallelogram spanned from the projected box centre by the projected
            // half-axes ax = hx P(X), ay = hy P(Y), widened by the projected half sag
            // az = hz P(Z): with (u, v) = [ax ay]^-1 q, a point q of the footprint has
            // |u| <= 1 + |uz| and |v| <= 1 + |vz| where (uz, vz) = [ax ay]^-1 az.  Near edge-on
            // elements, and surfaces without a box, keep the disc alone (rows all zero).
            //
            // Disc: the radius is widened by the float rounding of centre and ray coordinates
            // (~1e-7 relative) and by the distance from the projected origin to the centre.
            std::vector<float4> disc(st.elems.size()), par(st.elems.size(), float4{0.f, 0.f, 0.f, 0.f});
            const double box_ext = fabs(sun.xmin) + fabs(sun.xmax) + fabs(sun.ymin) + fabs(sun.ymax);
            for (size_t j = 0; j < st.elems.size(); ++j) {
                const Elem &e = st.elems[j];
                double ccx = cx_[j], ccy = cy_[j];
                double x0, x1, y0, y1, hz;
                if (local_box(e, x0, x1, y0, y1, hz)) {
                    const double pad = 1e-3 + 2e-6 * (1.0 + fabs(cx_[j]) + fabs(cy_[j]) + box_ext + rad[j]);
                    const double hx = (x1 - x0) / 2.0 + pad, hy = (y1 - y0) / 2.0 + pad, hzz = hz + pad;
                    const double lx = (x0 + x1) / 2.0, ly = (y0 + y1) / 2.0;
                    double c3[3], ax3[3], ay3[3], az3[3], c2[3], a2[3], b2[3], z2[3];
                    for (int q = 0; q < 3; ++q) {
                        c3[q] = e.origin[q] + lx * e.R[q] + ly * e.R[3 + q];
                        ax3[q] = hx * e.R[q];
                        ay3[q] = hy * e.R[3 + q];
                        az3[q] = hzz * e.R[6 + q];
                    }
                    mulv(Rs, c3, c2);
                    mulv(Rs, ax3, a2);
                    mulv(Rs, ay3, b2);
                    mulv(Rs, az3, z2);
                    const double det = a2[0] * b2[1] - a2[1] * b2[0];
                    const double la = sqrt(sq(a2[0]) + sq(a2[1])), lb = sqrt(sq(b2[0]) + sq(b2[1]));
                    if (fabs(det) > 1e-3 * la * lb) {  // not within ~0.06 deg of edge-on
                        const double i00 = b2[1] / det, i01 = -b2[0] / det, i10 = -a2[1] / det, i11 = a2[0] / det;
                        const double uz = i00 * z2[0] + i01 * z2[1], vz = i10 * z2[0] + i11 * z2[1];
                        // limits widened for the float evaluation of (u, v): 1e-5, plus 1e-6 of the
                        // largest term a row can produce over the parallelogram (skewed footprints)
                        const double Q = 2.0 * (la + lb + sqrt(sq(z2[0]) + sq(z2[1]))) + 1.0;
                        const double lu = (1.0 + fabs(uz)) * (1.0 + 1e-5) + 1e-6 * (fabs(i00) + fabs(i01)) * Q;
                        const double lv = (1.0 + fabs(vz)) * (1.0 + 1e-5) + 1e-6 * (fabs(i10) + fabs(i11)) * Q;
                        par[j] = float4{float(i00 / lu), float(i01 / lu), float(i10 / lv), float(i11 / lv)};
                        ccx = c2[0];
                        ccy = c2[1];
                    }
                }
                const double shift = sqrt(sq(ccx - cx_[j]) + sq(ccy - cy_[j]));
                const double pad = rad[j] * (1.0 + 1e-9) + 1e-6 * (1.0 + fabs(cx_[j]) + fabs(cy_[j])) + shift;
                const double fr = pad + 4e-7 * (fabs(ccx) + fabs(ccy) + box_ext + pad);
                int bits;
                const int jj = int(j);
                memcpy(&bits, &jj, 4);
                float w;
                memcpy(&w, &bits, 4);
                disc[j] = float4{float(ccx), float(ccy), float(fr), w};
            }
            // Exact footprints for first stages of flat rectangles (the mixed-precision probe
            // decides hit and nearest element in float and defers to double within its
            // rounding margins): a sun-frame ray (x, y) meets the plane of element j at depth
            // z0 + gx qx + gy qy, q = (x, y) - centre, inside the rectangle when
            // |i00 qx + i01 qy| <= 1 and |i10 qx + i11 qy| <= 1 (the rectangle's half-axes
            // projected along the sun's z, inverted).  Coordinates are taken relative to the
            // lower corner of the entry's cell, so that floats hold them to ~1e-6 m.
            bool exact = true;
            for (const Elem &e : st.elems)
                if (e.stype != 3 || char(tolower(e.shape)) != 'r') exact = false;
            std::vector<float4> xb(exact ? st.elems.size() : 0), xc(exact ? st.elems.size() : 0);
            std::vector<double> ecx(exact ? st.elems.size() : 0), ecy(exact ? st.elems.size() : 0);
            if (exact) {
                for (size_t j = 0; j < st.elems.size(); ++j) {
                    const Elem &e = st.elems[j];
                    double c2[3], a2[3], b2[3], n2[3], ax3[3], ay3[3], nz3[3];
                    for (int q = 0; q < 3; ++q) {
                        ax3[q] = e.p[0] / 2.0 * e.R[q];
                        ay3[q] = e.p[1] / 2.0 * e.R[3 + q];
                        nz3[q] = e.R[6 + q];
                    }
                    mulv(Rs, e.origin, c2);
                    mulv(Rs, ax3, a2);
                    mulv(Rs, ay3, b2);
                    mulv(Rs, nz3, n2);
                    const double det = a2[0] * b2[1] - a2[1] * b2[0];
                    const double la = sqrt(sq(a2[0]) + sq(a2[1])), lb = sqrt(sq(b2[0]) + sq(b2[1]));
                    ecx[j] = c2[0];
                    ecy[j] = c2[1];
                    xb[j] = float4{0.f, 0.f, 0.f, 0.f};
                    if (!e.enabled || !(0.0 <= e.zap)) {
                        xc[j] = float4{0.f, 0.f, INFINITY, 0.f};  // never accepted (element_test_flat)
                    } else if (!(fabs(det) > 1e-3 * la * lb) || !(fabs(n2[2]) > 1e-3)) {
                        xc[j] = float4{0.f, 0.f, NAN, 0.f};  // near edge-on: always decided in double
                    } else {
                        xb[j] = float4{float(b2[1] / det), float(-b2[0] / det), float(-a2[1] / det),
                                       float(a2[0] / det)};
                        xc[j] = float4{float(-n2[0] / n2[2]), float(-n2[1] / n2[2]), float(c2[2]), 0.f};
                    }
                }
            }
            // (start, end) pair per cell: cell c at [2c, 2c + 1], read on the device as one int2
            hs.cell_start.assign(2 * size_t(nx) * ny, 0);
            int at = 0;
            for (size_t c = 0; c < cells.size(); ++c) {
                hs.cell_start[2 * c] = at;
                const int gxc = int(c % size_t(nx)), gyc = int(c / size_t(nx));
                const double x0c = sun.xmin + gxc * cell, y0c = sun.ymin + gyc * cell;
                for (int j : cells[c]) {
                    hs.cell_disc.push_back(disc[j]);
                    hs.cell_par.push_back(par[j]);
                    if (exact) {
                        const float r = disc[j].z;
                        hs.cell_xa.push_back(float4{float(ecx[j] - x0c), float(ecy[j] - y0c), r * r, disc[j].w});
                        hs.cell_xb.push_back(xb[j]);
                        hs.cell_xc.push_back(xc[j]);
                    }
                }
                at += int(cells[c].size());
                hs.cell_start[2 * c + 1] = at;
            }
            sd.exact_flat = exact ? 1 : 0;
            sd.grid_on = 1;
            sd.gnx = nx;
            sd.gny = ny;
            sd.gx0 = sun.xmin;
            sd.gy0 = sun.ymin;
            sd.ginv = 1.0 / cell;
            sd.gcell = cell;
        }
    }
    return true;
}

bool flatten(Context *cx, HostScene &hs) {
    hs = HostScene();
    memset(&hs.dev, 0, sizeof hs.dev);
    if (cx->stages.size() > size_t(kMaxStages)) {
        cx->log("at most %d stages are supported", kMaxStages);
        return false;
    }
    // optics: two OpticRec per set (front, back)
    for (const OpticSet &os : cx->optics) {
        for (int fb = 0; fb < 2; ++fb) {
            const Face &f = fb ? os.back : os.front;
            OpticRec r;
            memset(&r, 0, sizeof r);
            r.refl = f.refl;
            r.trans = f.trans;
            r.slope = f.slope;
            r.spec = f.spec;
            r.n_in = f.n[0];
            r.n_out = f.n[2];
            r.dist = f.dist;
            r.refl_tab_off = int(hs.tables.size());
            r.refl_tab_n = f.use_refl ? int(f.refl_tab.size() / 2) : 0;
            if (f.use_refl) hs.tables.insert(hs.tables.end(), f.refl_tab.begin(), f.refl_tab.end());
            r.trans_tab_off = int(hs.tables.size());
            r.trans_tab_n = f.use_trans ? int(f.trans_tab.size() / 2) : 0;
            if (f.use_trans) hs.tables.insert(hs.tables.end(), f.trans_tab.begin(), f.trans_tab.end());
            hs.optics.push_back(r);
        }
    }
    hs.dev.n_stages = int(cx->stages.size());
    for (size_t si = 0; si < cx->stages.size(); ++si) {
        const StageM &st = cx->stages[si];
        StageRec &sr = hs.dev.stages[si];
        for (int k = 0; k < 9; ++k) sr.R[k] = st.R[k];
        for (int k = 0; k < 3; ++k) sr.o[k] = st.origin[k];
        sr.first_elem = int(hs.elems.size());
        sr.n_elem = int(st.elems.size());
        sr.virt = st.virt;
        sr.multihit = st.multihit;
        sr.tracethrough = st.tracethrough;
        sr.bvh_off = -1;
        for (const Elem &e : st.elems) {
            ElemRec r;
            memset(&r, 0, sizeof r);
            for (int k = 0; k < 9; ++k) r.R[k] = e.R[k];
            for (int k = 0; k < 3; ++k) r.o[k] = e.origin[k];
            for (int k = 0; k < 8; ++k) r.ap[k] = e.p[k];
            r.zap = e.zap;
            r.kappa = e.kappa;
            r.vcx = e.vcx;
            r.vcy = e.vcy;
            r.curv_rev = e.curv;
            r.cone_deg = e.cone;
            r.ra = e.ra;
            r.rs = e.rs;
            r.area = e.area;
            r.bound_r = accept_radius(e);
            {
                // float bounding sphere for the BVH leaf pre-test: 1 mm plus 1e-6 of the centre's
                // coordinates on top of the exact radius; unbounded elements always pass
                const double cmax = std::max(fabs(e.origin[0]), std::max(fabs(e.origin[1]), fabs(e.origin[2])));
                const float w = r.bound_r < 0 ? 3.0e38f : float(r.bound_r * (1.0 + 1e-6) + 1e-3 + 1e-6 * cmax);
                hs.elem_sphere.push_back(make_float4(float(e.origin[0]), float(e.origin[1]), float(e.origin[2]), w));
            }
            r.shape = tolower(e.shape);
            r.surf = e.surface;
            r.stype = e.stype;
            r.interaction = e.interaction;
            r.opt_front = e.optic_idx >= 0 ? 2 * e.optic_idx : -1;
            r.opt_back = e.optic_idx >= 0 ? 2 * e.optic_idx + 1 : -1;
            r.enabled = e.enabled;
            r.fit_order = e.fit_order;
            r.data_off = int(hs.surf_data.size());
            switch (e.stype) {
                case kSurfZernike:
                    hs.surf_data.insert(hs.surf_data.end(), e.bcoef.begin(), e.bcoef.end());
                    break;
                case kSurfVshot:
                    hs.surf_data.insert(hs.surf_data.end(), e.bcoef.begin(), e.bcoef.end());
                    hs.surf_data.insert(hs.surf_data.end(), e.vshot.begin(), e.vshot.end());
                    r.data_n = e.vshot_rows;
                    break;
                case kSurfPoly:
                    hs.surf_data.insert(hs.surf_data.end(), e.poly.begin(), e.poly.end());
                    break;
                case kSurfSpline:
                    hs.surf_data.insert(hs.surf_data.end(), e.spl_x.begin(), e.spl_x.end());
                    hs.surf_data.insert(hs.surf_data.end(), e.spl_y.begin(), e.spl_y.end());
                    hs.surf_data.insert(hs.surf_data.end(), e.spl_y2.begin(), e.spl_y2.end());
                    r.spl_n = int(e.spl_x.size());
                    break;
                case kSurfFE:
                    fe_table(e.vshot, hs.surf_data);
                    break;
                default:
                    break;
            }
            hs.elems.push_back(r);
        }
        sr.flat_only = 1;
        for (const Elem &e : st.elems) sr.flat_only &= (e.stype == 3) ? 1 : 0;
        sr.closed_only = 1;
        for (int k = sr.first_elem; k < sr.first_elem + sr.n_elem; ++k)
            sr.closed_only &= closed_form_surface(hs.elems[k].stype, hs.elems[k].surf) ? 1 : 0;
        sr.grid_on = 0;
        if (st.elems.size() >= 64)
            build_ground_grid(st.elems, hs.elem_sphere.data() + sr.first_elem, sr, hs.stage_cells, hs.grid_sphere,
                              hs.grid_elem);
        if (st.elems.size() >= 16) {
            sr.bvh_off = int(hs.bvh.size());
            sr.bvh_items_off = int(hs.bvh_items.size());
            build_bvh(st.elems, hs.bvh, hs.bvh_items);
            // child indices are relative to the stage's first node
        }
    }
    if (!sun_setup(cx, hs)) return false;
    build_beam_lists(cx, hs);
    hs.dev.sunshape_on = cx->err_sun;
    hs.dev.errors_on = cx->err_opt;
    return true;
}

// Saved second-stage input as the reference leaves it (raytrace.cpp:1064-1078): the stage's
// ray array at the end of stage 2 holds, in ray order, the rays that left stage 2 in its
// first positions (written back in place as they were produced) and the rays that entered
// it in the rest.  `in` and `out` are unordered rows of 7 doubles (ray number last).
std::vector<double> saved_second_stage(std::vector<double> in, std::vector<double> out) {
    auto by_ray = [](std::vector<double> &rows) {
        const size_t n = rows.size() / 7;
        std::vector<size_t> idx(n);
        std::iota(idx.begin(), idx.end(), size_t(0));
        std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return rows[7 * a + 6] < rows[7 * b + 6]; });
        std::vector<double> o(rows.size());
        for (size_t k = 0; k < n; ++k) std::copy(rows.begin() + 7 * idx[k], rows.begin() + 7 * idx[k] + 7, o.begin() + 7 * k);
        rows.swap(o);
    };
    by_ray(in);
    by_ray(out);
    const size_t n = in.size() / 7, w = std::min(out.size() / 7, n);
    std::vector<double> s1(in);
    std::copy(out.begin(), out.begin() + 7 * w, s1.begin());
    return s1;
}

// Exact key of every input the flattened scene is built from: optics, stages and elements
// (with their surface data), the sun and the error switches, serialised byte for byte.  A
// run reuses the cached scene only when the key equals the stored one, so no input change
// can go unseen (a front end that re-sends an unchanged scene before every run, as
// pysoltrace does, still reuses it).
struct SceneKey {
    std::string k;
    void bytes(const void *p, size_t n) { k.append(static_cast<const char *>(p), n); }
    template <typename T>
    void pod(const T &v) {
        bytes(&v, sizeof v);
    }
    void vec(const std::vector<double> &v) {
        pod(v.size());
        if (!v.empty()) bytes(v.data(), v.size() * sizeof(double));
    }
    void str(const std::string &s) {
        pod(s.size());
        bytes(s.data(), s.size());
    }
};

std::string scene_key(const Context *cx) {
    SceneKey g;
    g.k.reserve(cx->scene_key.size() + 64);
    g.pod(cx->err_sun);
    g.pod(cx->err_opt);
    const SunM &s = cx->sun;
    g.pod(s.shape);
    g.pod(s.sigma);
    g.pod(s.point_source);
    g.vec(s.ang);
    g.vec(s.inten);
    g.bytes(s.origin, sizeof s.origin);
    g.pod(cx->optics.size());
    for (const OpticSet &o : cx->optics) {
        g.str(o.name);
        for (const Face *f : {&o.front, &o.back}) {
            g.pod(f->dist);
            g.pod(f->optnum);
            g.pod(f->apgr);
            g.pod(f->order);
            g.pod(f->refl);
            g.pod(f->trans);
            g.pod(f->slope);
            g.pod(f->spec);
            g.bytes(f->n, sizeof f->n);
            g.bytes(f->ab12, sizeof f->ab12);
            g.vec(f->refl_tab);
            g.vec(f->trans_tab);
            g.pod(f->use_refl);
            g.pod(f->use_trans);
        }
    }
    g.pod(cx->stages.size());
    for (const StageM &st : cx->stages) {
        g.pod(st.multihit);
        g.pod(st.virt);
        g.pod(st.tracethrough);
        g.bytes(st.origin, sizeof st.origin);
        g.bytes(st.aim, sizeof st.aim);
        g.pod(st.zrot);
        g.pod(st.elems.size());
        for (const Elem &e : st.elems) {
            g.pod(e.enabled);
            g.bytes(e.origin, sizeof e.origin);
            g.bytes(e.aim, sizeof e.aim);
            g.pod(e.zrot);
            g.pod(e.shape);
            g.bytes(e.p, sizeof e.p);
            g.pod(e.surface);
            g.pod(e.stype);
            g.pod(e.kappa);
            g.bytes(e.alpha, sizeof e.alpha);
            g.pod(e.vcx);
            g.pod(e.vcy);
            g.pod(e.ra);
            g.pod(e.rs);
            g.pod(e.cone);
            g.pod(e.curv);
            g.pod(e.fit_order);
            g.vec(e.bcoef);
            g.vec(e.poly);
            g.vec(e.spl_x);
            g.vec(e.spl_y);
            g.vec(e.spl_y2);
            g.vec(e.vshot);
            g.pod(e.vshot_rows);
            g.pod(e.fe_surface);
            g.pod(e.interaction);
            g.str(e.optic);
        }
    }
    return std::move(g.k);
}

// the flattened scene of the context's current inputs (rebuilt only when they changed)
bool ensure_scene(Context *cx) {
    std::string key = scene_key(cx);
    if (!cx->scene_valid || cx->scene_key != key) {
        cx->scene_valid = false;
        if (!init_geometries(cx)) return false;
        cx->scene_cache = HostScene();
        if (!flatten(cx, cx->scene_cache)) return false;
        // the set-up fills derived fields; the next run starts from this state
        cx->scene_key = scene_key(cx);
        cx->scene_valid = true;
    }
    return true;
}

int run(Context *cx, unsigned seed) {
    cx->rec = RecordColumns{};
    memset(&cx->stats, 0, sizeof cx->stats);
    cx->stage_s0.clear();
    cx->stage_s1.clear();
    if (cx->save_stage_data && !cx->want_records) {
        cx->log("saving stage data needs the intersection records (st_b200_set_records)");
        return -1;
    }
    if (cx->ex_pos.empty() && !cx->replaying && cx->raycount < 1) {
        cx->log("invalid number of rays: %d", cx->raycount);
        return -1;
    }
    if (cx->stages.empty()) {
        cx->log("no stages defined.");
        return -1;
    }
    const auto t0 = std::chrono::steady_clock::now();
    if (!ensure_scene(cx)) return -1;
    const HostScene &hs = cx->scene_cache;
    RunRequest rq;
    rq.n_hits = uint64_t(cx->raycount);
    rq.max_sun = cx->max_sun64 ? cx->max_sun64 : uint64_t(std::max(cx->raymax, 0));
    rq.seed = seed;
    rq.precision = cx->precision;
    rq.records = cx->want_records;
    rq.device = cx->device;
    rq.ex_pos = cx->ex_pos;
    rq.ex_cos = cx->ex_cos;
    for (auto &f : cx->flux) rq.flux.push_back(f.req);
    rq.callback = cx->cb;
    rq.cbdata = cx->cbdata;
    rq.hit_rate_hint = cx->last_hit_rate;
    rq.save_stage_data = cx->save_stage_data;
    rq.rank = cx->rank;
    rq.nranks = cx->nranks;
    rq.allgather = cx->allgather;
    rq.allreduce = cx->allreduce;
    rq.comm_user = cx->comm_user;
    if (cx->nranks > 1) rq.hit_rate_hint = 0.0;  // every rank must plan from the same numbers
    if (cx->replaying) {
        // rays enter stage 2 from the saved rows; each row's first first-stage element from
        // the saved stage-1 records of its ray number (the first one), for the per-element
        // delivered counts
        rq.replay = true;
        rq.replay_rows = cx->replay_s1;
        const size_t n0 = cx->replay_s0.size() / 8, n1 = cx->replay_s1.size() / 7;
        std::vector<std::pair<double, int>> first;  // (ray number, element) of each ray's first record
        for (size_t k = 0; k < n0; ++k) {
            const double rn = cx->replay_s0[8 * k + 7];
            if (first.empty() || first.back().first != rn) first.push_back({rn, int(fabs(cx->replay_s0[8 * k + 6]))});
        }
        std::sort(first.begin(), first.end(), [](const std::pair<double, int> &a, const std::pair<double, int> &b) {
            return a.first < b.first;
        });
        rq.replay_fe0.assign(n1, -1);
        const int f0 = hs.dev.stages[0].first_elem, m0 = hs.dev.stages[0].n_elem;
        for (size_t k = 0; k < n1; ++k) {
            const double rn = cx->replay_s1[7 * k + 6];
            auto it = std::lower_bound(first.begin(), first.end(), std::make_pair(rn, INT_MIN));
            if (it != first.end() && it->first == rn && it->second >= 1 && it->second <= m0)
                rq.replay_fe0[k] = f0 + it->second - 1;
        }
        rq.replay_sun_rays = n0 ? uint64_t(cx->replay_s0[8 * (n0 - 1) + 7]) : 0;
        // the saved stage-1 records are the replay's stage-1 records (raytrace.cpp:554-565)
        if (rq.records) {
            double last = -1;
            uint32_t seq = 0;
            rq.pre_records.reserve(n0);
            for (size_t k = 0; k < n0; ++k) {
                const double *row = cx->replay_s0.data() + 8 * k;
                RecordDev r;
                memset(&r, 0, sizeof r);
                for (int q = 0; q < 3; ++q) {
                    r.pos[q] = row[q];
                    r.cos[q] = row[3 + q];
                }
                r.element = int(row[6]);
                r.stage = 1;
                r.raynum = uint32_t(row[7]);
                seq = (row[7] == last) ? seq + 1 : 0;
                last = row[7];
                r.seq = seq;
                rq.pre_records.push_back(r);
            }
        }
    }
    RunResult rr;
    const double host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (!cx->ws) cx->ws = workspace_create();
    const bool ok = gpu_run(hs, rq, rr, *cx->ws);
    if (!ok) {
        cx->log("%s", rr.error.c_str());
        return -1;
    }
    cx->sun_rays = rr.sun_rays;
    if (rr.sun_rays > 0 && cx->ex_pos.empty()) cx->last_hit_rate = double(rr.ray_hits) / double(rr.sun_rays);
    const int nst = int(cx->stages.size());
    const uint32_t N = uint32_t(rr.ray_hits);
    const bool drop_later = !cx->replaying && nst > 1 && rr.stage_entries[1] == 1 && rr.max_enter[1] == N;
    // flux maps and per-element counts
    for (size_t m = 0; m < cx->flux.size(); ++m) {
        cx->flux[m].counts = rr.flux[m];
        if (drop_later && cx->flux[m].req.stage >= 1) std::fill(cx->flux[m].counts.begin(), cx->flux[m].counts.end(), 0ull);
    }
    cx->elem_first.assign(nst, {});
    cx->elem_absorbed.assign(nst, {});
    cx->elem_delivered.assign(nst, {});
    for (int s = 0; s < nst; ++s) {
        const int f = hs.dev.stages[s].first_elem, n = hs.dev.stages[s].n_elem;
        cx->elem_first[s].assign(rr.first_hits.begin() + f, rr.first_hits.begin() + f + n);
        cx->elem_absorbed[s].assign(rr.absorbed.begin() + f, rr.absorbed.begin() + f + n);
        cx->elem_delivered[s].assign(rr.delivered.begin() + f, rr.delivered.begin() + f + n);
        if (drop_later && s >= 1) {
            std::fill(cx->elem_first[s].begin(), cx->elem_first[s].end(), 0ull);
            std::fill(cx->elem_absorbed[s].begin(), cx->elem_absorbed[s].end(), 0ull);
        }
    }
    if (drop_later) std::fill(cx->elem_delivered[0].begin(), cx->elem_delivered[0].end(), 0ull);
    st_b200_stats &S = cx->stats;
    S.sun_rays = rr.sun_rays;
    S.ray_hits = rr.ray_hits;
    S.ray_stage_units = rr.sun_rays;
    for (int s = 0; s < nst && s < 16; ++s) {
        S.stage_entries[s] = (drop_later && s >= 1) ? 0 : rr.stage_entries[s];
        if (s >= 1) S.ray_stage_units += S.stage_entries[s];
    }
    S.probe_ms = rr.probe_ms;
    S.trace_ms = rr.trace_ms;
    S.kernel_ms = rr.device_ms;
    S.setup_ms = rr.setup_ms + host_ms;
    S.batches = rr.batches;
    S.gpu_launches = rr.gpu_launches;
    S.h2d_bytes = rr.h2d_bytes;
    S.d2h_bytes = rr.d2h_bytes;
    S.probe_variant = rr.probe_variant;
    S.trace_variant = rr.trace_variant;
    if (rr.flags & 1u) cx->log("warning: a ray reached the limit of intersections per stage; it was stopped there");
    const auto ta = std::chrono::steady_clock::now();
    cx->rec = rr.rec;  // ordered on the device (gpu_run)
    const RecordColumns &R = cx->rec;
    if (cx->save_stage_data) {
        // stage-1 records in ray order (the records of stage 1 keep that order in the merged
        // readback) and the second stage's input as the reference saves it
        for (size_t i = 0; i < R.n; ++i)
            if (R.stage[i] == 1) {
                const double row[8] = {R.x[i], R.y[i], R.z[i], R.cx[i], R.cy[i], R.cz[i], double(R.element[i]),
                                       double(R.raynum[i])};
                cx->stage_s0.insert(cx->stage_s0.end(), row, row + 8);
            }
        if (nst >= 2) cx->stage_s1 = saved_second_stage(rr.saved[0], rr.saved[1]);
    }
    S.readback_ms = rr.readback_ms + std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - ta).count();
    S.records = R.n;
    // over several ranks the records are this rank's, the counts the whole run's
    S.intersections = (cx->want_records && cx->nranks <= 1) ? uint64_t(R.n) : rr.intersections;
    return int(R.n);
}

// Batched runs keep every position's sun-plane grid on the device at once (per chunk of
// kBatchChunk positions), so their grids get a smaller cell budget than a single run's.
constexpr double kBatchSunGridCells = 2.5e5;
constexpr size_t kBatchChunk = 64;

// The sun-dependent tables of one position of a batched run: the context's sun moved to
// `sun_xyz` and, with `target`, every first-stage element re-aimed so that its normal bisects
// the sun direction and the direction to the target (a heliostat tracking the sun; the aim
// point is origin + 100 n, zrot kept, rotation by input.cpp:160-176).
bool build_position(const Context *cx, const HostScene &hs, const double sun_xyz[3], const double *target,
                    SunPosition &out, std::string &err) {
    Context c;
    c.sun = cx->sun;
    c.sun_grid_cells = kBatchSunGridCells;
    for (int q = 0; q < 3; ++q) c.sun.origin[q] = sun_xyz[q];
    c.err_sun = cx->err_sun;
    c.err_opt = cx->err_opt;
    c.stages.push_back(cx->stages[0]);
    StageM &st0 = c.stages[0];
    if (target) {
        const double sn = sqrt(sq(sun_xyz[0]) + sq(sun_xyz[1]) + sq(sun_xyz[2]));
        if (!(sn > 0)) {
            err = "sun position at the origin";
            return false;
        }
        const double s[3] = {sun_xyz[0] / sn, sun_xyz[1] / sn, sun_xyz[2] / sn};
        for (Elem &e : st0.elems) {
            double t[3] = {target[0] - e.origin[0], target[1] - e.origin[1], target[2] - e.origin[2]};
            const double tn = sqrt(sq(t[0]) + sq(t[1]) + sq(t[2]));
            double n[3];
            for (int q = 0; q < 3; ++q) n[q] = s[q] + (tn > 0 ? t[q] / tn : 0.0);
            const double nn = sqrt(sq(n[0]) + sq(n[1]) + sq(n[2]));
            if (!(nn > 0)) {
                err = "a tracking element cannot bisect the sun and target directions";
                return false;
            }
            for (int q = 0; q < 3; ++q) e.aim[q] = e.origin[q] + 100.0 * (n[q] / nn);
            double eu[3];
            if (!euler_of(e.origin, e.aim, e.zrot, eu)) {
                err = "a tracking element's geometry is not possible";
                return false;
            }
            rot_from_euler(eu, e.R);
        }
    }
    HostScene h;
    h.dev = hs.dev;
    if (!sun_setup(&c, h)) {
        err = c.messages.empty() ? std::string("sun set-up failed") : c.messages.back();
        return false;
    }
    out.sun = h.dev.sun;
    out.cell_start.swap(h.cell_start);
    out.cell_disc.swap(h.cell_disc);
    out.cell_par.swap(h.cell_par);
    out.cell_xa.swap(h.cell_xa);
    out.cell_xb.swap(h.cell_xb);
    out.cell_xc.swap(h.cell_xc);
    if (target) {
        const StageRec &sr = hs.dev.stages[0];
        out.rot.resize(size_t(sr.n_elem) * 9);
        for (int k = 0; k < sr.n_elem; ++k)
            for (int q = 0; q < 9; ++q) out.rot[size_t(k) * 9 + q] = st0.elems[size_t(k)].R[q];
    }
    return true;
}

int run_batch(Context *cx, unsigned seed, int n_pos, const double *sun_xyz, const st_uint_t *hits,
              const double *target) {
    cx->batch.clear();
    cx->batch_box.clear();
    memset(&cx->batch_stats, 0, sizeof cx->batch_stats);
    if (n_pos < 1 || !sun_xyz || !hits) {
        cx->log("st_b200_sim_run_batch: at least one sun position with its hit count is needed");
        return -1;
    }
    if (!cx->ex_pos.empty()) {
        cx->log("st_b200_sim_run_batch: the context traces explicit rays; batched runs trace sun rays");
        return -1;
    }
    if (cx->stages.empty()) {
        cx->log("no stages defined.");
        return -1;
    }
    const auto t0 = std::chrono::steady_clock::now();
    if (!ensure_scene(cx)) return -1;
    const HostScene &hs = cx->scene_cache;
    const size_t np = static_cast<size_t>(n_pos);
    RunRequest rq;
    rq.max_sun = uint64_t(std::max(cx->raymax, 0));
    rq.precision = cx->precision;
    rq.device = cx->device;
    for (auto &f : cx->flux) rq.flux.push_back(f.req);
    // positions go to the device in chunks; the host builds the next chunk's tables while
    // the device runs the current one
    auto build_chunk = [cx, &hs, sun_xyz, hits, target, seed](size_t a, size_t b, std::vector<SunPosition> &pos,
                                                               std::string &err) -> bool {
        const size_t n = b - a;
        pos.assign(n, SunPosition());
        std::vector<std::string> errs(n);
        std::vector<char> ok(n, 0);
        const size_t nth = std::max<size_t>(1, std::min<size_t>(n, std::thread::hardware_concurrency()));
        std::vector<std::thread> th;
        for (size_t t = 0; t < nth; ++t)
            th.emplace_back([&, t]() {
                for (size_t i = t; i < n; i += nth) {
                    const size_t p = a + i;
                    ok[i] = build_position(cx, hs, sun_xyz + 3 * p, target, pos[i], errs[i]);
                    pos[i].n_hits = uint64_t(hits[p]);
                    pos[i].seed = seed + unsigned(p);
                }
            });
        for (auto &x : th) x.join();
        for (size_t i = 0; i < n; ++i)
            if (!ok[i]) {
                err = "sun position " + std::to_string(a + i) + ": " + errs[i];
                return false;
            }
        return true;
    };
    if (!cx->ws) cx->ws = workspace_create();
    if (!workspace_bind(*cx->ws, rq.device)) {
        cx->log("st_b200_sim_run_batch: cannot use CUDA device %d", rq.device);
        return -1;
    }
    double host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    BatchResult tot;
    std::vector<SunPosition> cur, nxt;
    std::string err, err_next;
    const auto tb = std::chrono::steady_clock::now();
    if (!build_chunk(0, std::min(np, kBatchChunk), cur, err)) {
        cx->log("st_b200_sim_run_batch: %s", err.c_str());
        return -1;
    }
    int slot = 0;  // the staging area holding `cur`; the next chunk is staged in the other
    stage_positions(*cx->ws, slot, cur, rq.device);
    host_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tb).count();
    for (size_t a = 0; a < np; a += kBatchChunk) {
        const size_t b = std::min(np, a + kBatchChunk);
        bool next_ok = true;
        std::thread builder;
        if (b < np)
            builder = std::thread([&]() {
                next_ok = build_chunk(b, std::min(np, b + kBatchChunk), nxt, err_next);
                if (next_ok) stage_positions(*cx->ws, slot ^ 1, nxt, rq.device);
            });
        BatchResult br;
        const bool ran = gpu_run_batch(hs, cur, rq, br, *cx->ws, slot);
        if (builder.joinable()) builder.join();
        if (!ran) {
            cx->log("%s", br.error.c_str());
            return -1;
        }
        if (!next_ok) {
            cx->log("st_b200_sim_run_batch: %s", err_next.c_str());
            return -1;
        }
        for (const SunPosition &sp : cur) cx->batch_box.push_back({sp.sun.xmin, sp.sun.xmax, sp.sun.ymin, sp.sun.ymax});
        for (auto &r : br.pos) tot.pos.push_back(std::move(r));
        tot.device_ms += br.device_ms;
        tot.probe_ms += br.probe_ms;
        tot.trace_ms += br.trace_ms;
        tot.setup_ms += br.setup_ms;
        tot.batches += br.batches;
        tot.waves += br.waves;
        tot.gpu_launches += br.gpu_launches;
        tot.h2d_bytes += br.h2d_bytes;
        tot.d2h_bytes += br.d2h_bytes;
        tot.probe_variant = br.probe_variant;
        cur.swap(nxt);
        nxt.clear();
        slot ^= 1;
    }
    BatchResult &br = tot;
    cx->batch.swap(br.pos);
    st_b200_stats &S = cx->batch_stats;
    for (const PositionResult &r : cx->batch) {
        S.sun_rays += r.sun_rays;
        S.ray_hits += r.ray_hits;
        S.ray_stage_units += r.sun_rays;
        for (size_t k = 0; k < r.stage_entries.size() && k < 16; ++k) {
            S.stage_entries[k] += r.stage_entries[k];
            if (k >= 1) S.ray_stage_units += r.stage_entries[k];
        }
        S.intersections += r.intersections;
    }
    S.kernel_ms = br.device_ms;
    S.probe_ms = br.probe_ms;
    S.trace_ms = br.trace_ms;
    S.setup_ms = br.setup_ms + host_ms;
    S.batches = br.batches;
    S.gpu_launches = br.gpu_launches;
    S.h2d_bytes = br.h2d_bytes;
    S.d2h_bytes = br.d2h_bytes;
    S.probe_variant = br.probe_variant;
    return 1;
}

Context *C(st_context_t p) { return reinterpret_cast<Context *>(p); }

}  // namespace

namespace stb {
bool context_device(void *ctx, int &device, bool &sun_rays) {
    Context *cx = C(ctx);
    if (!cx) return false;
    device = cx->device;
    sun_rays = cx->ex_pos.empty() && !cx->replaying;
    return true;
}

// Geometry set-up and flattening of a context's scene for callers outside this file;
// on failure the reason is appended to the context's messages and false is returned.
bool prepare_scene(void *ctx, HostScene &hs) {
    Context *cx = C(ctx);
    if (!cx) return false;
    if (cx->stages.empty()) {
        cx->log("no stages defined.");
        return false;
    }
    if (!init_geometries(cx)) return false;
    if (!flatten(cx, hs)) return false;
    return true;
}
void report(void *ctx, const std::string &msg) {
    if (C(ctx)) C(ctx)->log("%s", msg.c_str());
}
}  // namespace stb

// message hook of the .stinput reader (st_stinput.cpp); not exported
extern "C" __attribute__((visibility("hidden"))) void st_input_report(void *ctx, const char *msg) {
    stb::report(ctx, msg ? msg : "");
}

namespace {
StageM *stage_of(Context *cx, st_uint_t i) { return i < cx->stages.size() ? &cx->stages[i] : nullptr; }
Elem *elem_of(Context *cx, st_uint_t s, st_uint_t i) {
    StageM *st = stage_of(cx, s);
    return (st && i < st->elems.size()) ? &st->elems[i] : nullptr;
}

bool read_surface_file(Context *cx, Elem &e, const char *file) {  // input.cpp:368-573
    const char *dot = strrchr(file, '.');
    if (!dot) {
        cx->log("Could not determine surface file type: '%s'\n", file);
        return false;
    }
    std::string ext(dot + 1);
    for (auto &c : ext) c = char(tolower(c));
    FILE *fp = fopen(file, "r");
    if (!fp) {
        cx->log("Could not open surface file for read: %s\n", file);
        return false;
    }
    char line[1024];
    auto rd = [&]() {
        if (!fgets(line, sizeof line, fp)) line[0] = 0;
    };
    bool ok = true;
    if (ext == "mon") {
        rd();
        const int order = atoi(line);
        e.bcoef.assign(size_t(order + 1) * (order + 1), 0.0);
        for (int k = 0; k <= order; ++k)
            for (int m = 0; m <= k; ++m) {
                rd();
                e.bcoef[size_t(k) * (order + 1) + m] = atof(line);
            }
        e.fit_order = order;
        e.surface = 'm';
        e.stype = 6;
    } else if (ext == "sht") {
        rd();
        rd();
        rd();
        int idum = 0, order = 0, np = 0;
        sscanf(line, "%d %d %d", &idum, &order, &np);
        rd();
        e.fit_order = order;
        e.bcoef.assign(size_t(order + 1) * (order + 1), 0.0);
        for (int k = 0; k <= order; ++k)
            for (int m = 0; m <= k; ++m) {
                rd();
                e.bcoef[size_t(k) * (order + 1) + m] = atof(line);
            }
        e.vshot.assign(size_t(5) * np, 0.0);
        e.vshot_rows = np;
        for (int k = 0; k < np; ++k) {
            rd();
            double *v = &e.vshot[size_t(5) * k];
            sscanf(line, "%lg %lg %lg %lg %lg", v, v + 1, v + 2, v + 3, v + 4);
        }
        e.surface = 'v';
        e.stype = 5;
    } else if (ext == "ply") {
        rd();
        const int order = atoi(line);
        e.poly.assign(size_t(order + 1), 0.0);
        for (int k = 0; k <= order; ++k) {
            rd();
            e.poly[k] = atof(line);
        }
        e.fit_order = order;
        e.surface = 'r';
        e.stype = 8;
    } else if (ext == "csi") {
        rd();
        const int np = atoi(line);
        e.spl_x.assign(np, 0.0);
        e.spl_y.assign(np, 0.0);
        for (int k = 0; k < np; ++k) {
            rd();
            sscanf(line, "%lg %lg", &e.spl_x[k], &e.spl_y[k]);
        }
        double a = 0, b = 0;
        rd();
        sscanf(line, "%lg %lg", &a, &b);
        spline_y2(e.spl_x, e.spl_y, a, b, e.spl_y2);
        if (np < 2 || (e.shape != 'a' && e.shape != 'A' && e.shape != 'l' && e.shape != 'L') || e.p[0] < e.spl_x[0] ||
            e.p[1] > e.spl_x.back()) {
            cx->log("Error: Element uses cubic spline interpolation:"
                    "\tMake sure aperture is type 'a' or 'l' and that "
                    "1st and 2nd parameters are not < and not > the "
                    "1st and last X values in file respectively.\n");
            ok = false;
        } else {
            e.surface = 'i';
            e.stype = 9;
        }
    } else if (ext == "fed") {
        // accepted so that scenes load; st_sim_run reports that this surface is not traced
        rd();
        rd();
        const int np = atoi(line);
        e.vshot.assign(size_t(3) * std::max(np, 0), 0.0);
        for (int k = 0; k < np; ++k) {
            rd();
            sscanf(line, "%lg %lg %lg", &e.vshot[3 * k], &e.vshot[3 * k + 1], &e.vshot[3 * k + 2]);
        }
        e.fe_surface = true;
        e.surface = 'e';
        e.stype = 4;
    } else {
        cx->log("Surface file type extension unknown: '%s'\n", ext.c_str());
        ok = false;
    }
    fclose(fp);
    return ok;
}

}  // namespace

// ======================================================================================
// C API
// ======================================================================================
#define CTX(p, r)        \
    Context *cx = C(p);  \
    if (!cx) return r;

extern "C" {

st_context_t st_create_context(void) { return new Context; }
int st_free_context(st_context_t p) {
    CTX(p, -1);
    delete cx;
    return 1;
}
int st_num_messages(st_context_t p) {
    CTX(p, -1);
    return int(cx->messages.size());
}
const char *st_message(st_context_t p, st_uint_t i) {
    CTX(p, nullptr);
    return i < cx->messages.size() ? cx->messages[i].c_str() : nullptr;
}
void st_clear_messages(st_context_t p) {
    if (C(p)) C(p)->messages.clear();
}
int st_num_optics(st_context_t p) {
    CTX(p, -1);
    return int(cx->optics.size());
}
int st_add_optic(st_context_t p, const char *name) {
    CTX(p, -1);
    cx->optics.push_back(OpticSet());
    cx->optics.back().name = name ? name : "";
    return int(cx->optics.size()) - 1;
}
int st_delete_optic(st_context_t p, st_uint_t i) {
    CTX(p, -1);
    if (i >= cx->optics.size()) return -1;
    cx->optics.erase(cx->optics.begin() + i);
    return 1;
}
int st_clear_optics(st_context_t p) {
    CTX(p, -1);
    cx->optics.clear();
    return 1;
}
int st_optic(st_context_t p, st_uint_t idx, int fb, char dist, int optnum, int apgr, int order, double rreal,
             double rimag, double ref, double tra, double gratingab12[3], double rmsslope, double rmsspec,
             int userefltable, int refl_npoints, double *refl_angles, double *refls, int usetranstable,
             int trans_npoints, double *trans_angles, double *transs) {
    CTX(p, -1);
    if (idx >= cx->optics.size()) return -1;
    Face &f = (fb == 2) ? cx->optics[idx].back : cx->optics[idx].front;
    f.dist = dist;
    f.optnum = optnum;
    f.apgr = apgr;
    f.order = order;
    f.n[0] = rreal;
    f.n[1] = rimag;
    f.refl = ref;
    f.trans = tra;
    // the reference reads four grating coefficients (stapi.cpp:188-189)
    if (gratingab12)
        for (int i = 0; i < 4; ++i) f.ab12[i] = gratingab12[i];
    f.slope = rmsslope;
    f.spec = rmsspec;
    if (userefltable && refl_npoints > 0 && refl_angles && refls) {
        f.use_refl = true;
        f.refl_tab.clear();
        for (int i = 0; i < refl_npoints; ++i) {
            f.refl_tab.push_back(refl_angles[i]);
            f.refl_tab.push_back(refls[i]);
        }
    }
    if (usetranstable && trans_npoints > 0 && trans_angles && transs) {
        f.use_trans = true;
        f.trans_tab.clear();
        for (int i = 0; i < trans_npoints; ++i) {
            f.trans_tab.push_back(trans_angles[i]);
            f.trans_tab.push_back(transs[i]);
        }
    }
    return 1;
}
int st_num_stages(st_context_t p) {
    CTX(p, -1);
    return int(cx->stages.size());
}
int st_add_stage(st_context_t p) {
    CTX(p, -1);
    cx->stages.push_back(StageM());
    return int(cx->stages.size()) - 1;
}
int st_add_stages(st_context_t p, st_uint_t n) {
    CTX(p, -1);
    for (st_uint_t i = 0; i < n; ++i) cx->stages.push_back(StageM());
    return int(n);
}
int st_delete_stage(st_context_t p, st_uint_t i) {
    CTX(p, -1);
    if (i >= cx->stages.size()) return -1;
    cx->stages.erase(cx->stages.begin() + i);
    return 1;
}
int st_clear_stages(st_context_t p) {
    CTX(p, -1);
    cx->stages.clear();
    return 1;
}
#define STAGE_SET(body)                     \
    CTX(p, -1);                             \
    StageM *st = stage_of(cx, i);           \
    if (!st) return -1;                     \
    body;                                   \
    return 1;
int st_stage_xyz(st_context_t p, st_uint_t i, double x, double y, double z) {
    STAGE_SET(st->origin[0] = x; st->origin[1] = y; st->origin[2] = z)
}
int st_stage_aim(st_context_t p, st_uint_t i, double x, double y, double z) {
    STAGE_SET(st->aim[0] = x; st->aim[1] = y; st->aim[2] = z)
}
int st_stage_zrot(st_context_t p, st_uint_t i, double z) { STAGE_SET(st->zrot = z) }
int st_stage_flags(st_context_t p, st_uint_t i, int virt, int multihit, int tracethrough) {
    STAGE_SET(st->virt = virt != 0; st->multihit = multihit != 0; st->tracethrough = tracethrough != 0)
}
int st_num_elements(st_context_t p, st_uint_t s) {
    CTX(p, -1);
    StageM *st = stage_of(cx, s);
    return st ? int(st->elems.size()) : -1;
}
int st_add_element(st_context_t p, st_uint_t s) {
    CTX(p, -1);
    StageM *st = stage_of(cx, s);
    if (!st) return -1;
    st->elems.push_back(Elem());
    return int(st->elems.size()) - 1;
}
int st_add_elements(st_context_t p, st_uint_t s, st_uint_t n) {
    CTX(p, -1);
    if (n < 1) return -1;
    StageM *st = stage_of(cx, s);
    if (!st) return -1;
    st->elems.resize(st->elems.size() + n);
    return int(n);
}
int st_delete_element(st_context_t p, st_uint_t s, st_uint_t i) {
    CTX(p, -1);
    StageM *st = stage_of(cx, s);
    if (!st || i >= st->elems.size()) return -1;
    st->elems.erase(st->elems.begin() + i);
    return 1;
}
int st_clear_elements(st_context_t p, st_uint_t s) {
    CTX(p, -1);
    StageM *st = stage_of(cx, s);
    if (!st) return -1;
    st->elems.clear();
    return 1;
}
#define ELEM_SET(body)                      \
    CTX(p, -1);                             \
    Elem *e = elem_of(cx, s, i);            \
    if (!e) return -1;                      \
    body;                                   \
    return 1;
int st_element_enabled(st_context_t p, st_uint_t s, st_uint_t i, int en) { ELEM_SET(e->enabled = en != 0) }
int st_element_xyz(st_context_t p, st_uint_t s, st_uint_t i, double x, double y, double z) {
    ELEM_SET(e->origin[0] = x; e->origin[1] = y; e->origin[2] = z)
}
int st_element_aim(st_context_t p, st_uint_t s, st_uint_t i, double x, double y, double z) {
    ELEM_SET(e->aim[0] = x; e->aim[1] = y; e->aim[2] = z)
}
int st_element_zrot(st_context_t p, st_uint_t s, st_uint_t i, double z) { ELEM_SET(e->zrot = z) }
int st_element_aperture(st_context_t p, st_uint_t s, st_uint_t i, char ap) { ELEM_SET(e->shape = ap) }
int st_element_aperture_params(st_context_t p, st_uint_t s, st_uint_t i, double prm[8]) {
    ELEM_SET(for (int k = 0; k < 8; ++k) e->p[k] = prm[k])
}
int st_element_surface(st_context_t p, st_uint_t s, st_uint_t i, char sf) { ELEM_SET(e->surface = sf) }
int st_element_surface_params(st_context_t p, st_uint_t s, st_uint_t i, double prm[8]) {
    CTX(p, -1);
    Elem *e = elem_of(cx, s, i);
    if (!e) return -1;
    return translate_surface(cx, *e, prm) ? 1 : -1;
}
int st_element_surface_file(st_context_t p, st_uint_t s, st_uint_t i, const char *file) {
    CTX(p, -1);
    Elem *e = elem_of(cx, s, i);
    if (!e || !file) return -1;
    return read_surface_file(cx, *e, file) ? 1 : -1;
}
int st_element_interaction(st_context_t p, st_uint_t s, st_uint_t i, int t) { ELEM_SET(e->interaction = t) }
int st_element_optic(st_context_t p, st_uint_t s, st_uint_t i, const char *name) {
    ELEM_SET(e->optic = name ? name : "")
}
int st_sun(st_context_t p, int ps, char shape, double sigma) {
    CTX(p, -1);
    cx->sun.point_source = ps != 0;
    cx->sun.shape = shape;
    cx->sun.sigma = sigma;
    return 1;
}
int st_sun_xyz(st_context_t p, double x, double y, double z) {
    CTX(p, -1);
    cx->sun.origin[0] = x;
    cx->sun.origin[1] = y;
    cx->sun.origin[2] = z;
    return 1;
}
// solar position formula of stapi.cpp:485-527 (x west, y zenith, z north)
// Degrees to radians as the reference writes it, v * pi / 180 evaluated left to right (not
// v * (pi / 180)), so that the sun vector agrees with the reference's bit for bit.
static inline double rad(double v) { return v * kPi / 180; }
static inline double rad_l(double v) { return kPi / 180 * v; }  // the reference's M_PI / 180 * v
int st_sun_position(st_context_t, double lat, double day, double hour, double *x, double *y, double *z) {
    const double decl = 180 / kPi * asin(0.39795 * cos(0.98563 * kPi / 180 * (day - 173)));
    const double ha = 15 * (hour - 12);
    const double el = 180 / kPi * asin(sin(rad(decl)) * sin(rad(lat)) + cos(rad(decl)) * cos(rad(ha)) * cos(rad(lat)));
    double az = 180 / kPi *
                acos((sin(rad_l(decl)) * cos(rad_l(lat)) - cos(rad_l(decl)) * sin(rad_l(lat)) * cos(rad_l(ha))) /
                         cos(rad_l(el)) +
                     0.0000000001);
    if (sin(rad(ha)) > 0.0) az = 360 - az;
    if (x) *x = -sin(rad(az)) * cos(rad(el));
    if (y) *y = sin(rad(el));
    if (z) *z = cos(rad(az)) * cos(rad(el));
    return 1;
}
int st_sun_userdata(st_context_t p, st_uint_t n, double angle[], double intensity[]) {
    CTX(p, -1);
    if (n <= 2) return -1;
    SunM &s = cx->sun;
    s.max_angle = 0;
    s.max_intensity = 0;
    s.ang.assign(2 * n - 1, 0.0);
    s.inten.assign(2 * n - 1, 0.0);
    for (st_uint_t i = 0; i < n; ++i) {
        s.ang[n + i - 1] = angle[i];
        s.inten[n + i - 1] = intensity[i];
        s.max_angle = std::max(s.max_angle, angle[i]);
        s.max_intensity = std::max(s.max_intensity, intensity[i]);
    }
    for (st_uint_t i = 0; i + 1 < n; ++i) {
        s.ang[i] = -angle[n - i - 1];
        s.inten[i] = intensity[n - i - 1];
    }
    return int(n);
}
// readback (stapi.cpp:570-647): the caller's arrays hold st_num_intersections() entries;
// each is one copy of a column of the ordered records
int st_num_intersections(st_context_t p) {
    CTX(p, -1);
    return int(cx->rec.n);
}
static void copy_col(void *dst, const void *src, size_t bytes) {
    if (dst && src && bytes) memcpy(dst, src, bytes);
}
int st_locations(st_context_t p, double *x, double *y, double *z) {
    CTX(p, -1);
    const size_t b = cx->rec.n * sizeof(double);
    copy_col(x, cx->rec.x, b);
    copy_col(y, cx->rec.y, b);
    copy_col(z, cx->rec.z, b);
    return 1;
}
int st_cosines(st_context_t p, double *x, double *y, double *z) {
    CTX(p, -1);
    const size_t b = cx->rec.n * sizeof(double);
    copy_col(x, cx->rec.cx, b);
    copy_col(y, cx->rec.cy, b);
    copy_col(z, cx->rec.cz, b);
    return 1;
}
int st_elementmap(st_context_t p, int *m) {
    CTX(p, -1);
    copy_col(m, cx->rec.element, cx->rec.n * sizeof(int));
    return 1;
}
int st_stagemap(st_context_t p, int *m) {
    CTX(p, -1);
    copy_col(m, cx->rec.stage, cx->rec.n * sizeof(int));
    return 1;
}
int st_raynumbers(st_context_t p, int *m) {
    CTX(p, -1);
    copy_col(m, cx->rec.raynum, cx->rec.n * sizeof(int));
    return 1;
}
int st_sun_stats(st_context_t p, double *xmin, double *xmax, double *ymin, double *ymax, int *nsun) {
    CTX(p, -1);
    if (xmin) *xmin = cx->sun.xmin;
    if (xmax) *xmax = cx->sun.xmax;
    if (ymin) *ymin = cx->sun.ymin;
    if (ymax) *ymax = cx->sun.ymax;
    if (nsun) *nsun = int(cx->sun_rays);
    return 1;
}
int st_sim_params(st_context_t p, int raycount, int maxcount, int dyn) {
    CTX(p, -1);
    cx->raycount = raycount;
    cx->raymax = maxcount;
    cx->dyn = dyn != 0;
    return 1;
}
int st_sim_errors(st_context_t p, int sun, int opt) {
    CTX(p, -1);
    cx->err_sun = sun != 0;
    cx->err_opt = opt != 0;
    return 1;
}
int st_sim_run(st_context_t p, unsigned int seed,
               int (*cb)(st_uint_t, st_uint_t, st_uint_t, st_uint_t, st_uint_t, void *), void *data) {
    CTX(p, -1);
    cx->cb = cb;
    cx->cbdata = data;
    return run(cx, seed);
}

// transform utilities (stapi.cpp:737-778)
void st_calc_euler_angles(double origin[3], double aimpoint[3], double zrot, double euler[3]) {
    euler[0] = euler[1] = euler[2] = 0;
    euler_of(origin, aimpoint, zrot, euler);
}
void st_transform_to_local(double posref[3], double cosref[3], double origin[3], double R[3][3], double posloc[3],
                           double cosloc[3]) {
    const double d[3] = {posref[0] - origin[0], posref[1] - origin[1], posref[2] - origin[2]};
    mulv(&R[0][0], d, posloc);
    mulv(&R[0][0], cosref, cosloc);
}
void st_transform_to_reference(double posloc[3], double cosloc[3], double origin[3], double R[3][3], double posref[3],
                               double cosref[3]) {
    double d[3];
    mulv(&R[0][0], posloc, d);
    mulv(&R[0][0], cosloc, cosref);
    for (int i = 0; i < 3; ++i) posref[i] = d[i] + origin[i];
}
void st_matrix_vector_mult(double m[3][3], double v[3], double mxv[3]) { mulv(&m[0][0], v, mxv); }
void st_calc_transform_matrices(double euler[3], double rreftoloc[3][3], double rloctoref[3][3]) {
    rot_from_euler(euler, &rreftoloc[0][0]);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) rloctoref[i][j] = rreftoloc[j][i];
}
void st_matrix_transpose(double in[3][3], double out[3][3]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) out[i][j] = in[j][i];
}

// ---------------- B200 extensions ----------------
int st_b200_set_precision(st_context_t p, int mode) {
    CTX(p, -1);
    if (mode != ST_B200_FP64 && mode != ST_B200_MIXED) return -1;
    cx->precision = mode;
    return 1;
}
int st_b200_set_records(st_context_t p, int on) {
    CTX(p, -1);
    cx->want_records = on != 0;
    return 1;
}
int st_b200_set_device(st_context_t p, int device) {
    CTX(p, -1);
    if (device < 0) return -1;
    cx->device = device;
    return 1;
}
int st_b200_explicit_rays(st_context_t p, st_uint_t n, const double *pos, const double *cos) {
    CTX(p, -1);
    if (n && (!pos || !cos)) return -1;
    cx->ex_pos.assign(pos, pos + 3 * n);
    cx->ex_cos.assign(cos, cos + 3 * n);
    return int(n);
}
static int add_flux_map(Context *cx, int stage, int element, int kind, int nx, int ny, double x0, double x1,
                        double y0, double y1, int absorbed_only, int per_source) {
    if (cx->flux.size() >= size_t(kMaxFluxMaps) || nx <= 0 || ny <= 0 || stage < 1 || element < 1 || kind < 0 ||
        kind > 4 || !(x1 > x0 || kind == 1 || kind >= 3) || !(y1 > y0) || (kind != 0 && kind != 2 && !(x1 > 0))) {
        cx->log("invalid flux map request");
        return -1;
    }
    FluxMap m;
    m.req = FluxMapReq{stage - 1, element - 1, kind, nx, ny, absorbed_only ? 1 : 0, x0, x1, y0, y1, per_source};
    cx->flux.push_back(m);
    return int(cx->flux.size()) - 1;
}
int st_b200_add_flux_map(st_context_t p, int stage, int element, int kind, int nx, int ny, double x0, double x1,
                         double y0, double y1, int absorbed_only) {
    CTX(p, -1);
    return add_flux_map(cx, stage, element, kind, nx, ny, x0, x1, y0, y1, absorbed_only, 0);
}
int st_b200_add_source_flux_map(st_context_t p, int stage, int element, int kind, int nx, int ny, double x0,
                                double x1, double y0, double y1, int absorbed_only) {
    CTX(p, -1);
    return add_flux_map(cx, stage, element, kind, nx, ny, x0, x1, y0, y1, absorbed_only, 1);
}
int st_b200_clear_flux_maps(st_context_t p) {
    CTX(p, -1);
    cx->flux.clear();
    return 1;
}
int st_b200_flux_counts(st_context_t p, int map, unsigned long long *counts) {
    CTX(p, -1);
    if (map < 0 || size_t(map) >= cx->flux.size() || !counts) return -1;
    const auto &c = cx->flux[map].counts;
    size_t n = size_t(cx->flux[map].req.nx) * cx->flux[map].req.ny;
    if (cx->flux[map].req.per_source) n *= cx->stages.empty() ? 0 : cx->stages[0].elems.size();
    for (size_t i = 0; i < n; ++i) counts[i] = i < c.size() ? c[i] : 0ull;
    return 1;
}
// Flux statistics of a map, as the GUI computes them for an element
// (app/src/project.cpp:1139-1288): power per ray from the sun box and SunRayCount, flux =
// count x power per ray / bin area, peak and minimum (first bin in x-major order on ties),
// mean, population standard deviation, uniformity = sigma / mean, and the Monte-Carlo
// uncertainties 100/sqrt(rays in the peak bin) and 100/sqrt(intersections of the run), %.
int st_b200_flux_stats(st_context_t p, int map, double dni, st_b200_flux_stats_t *out) {
    CTX(p, -1);
    if (map < 0 || size_t(map) >= cx->flux.size() || !out) return -1;
    const FluxMap &fm = cx->flux[map];
    const FluxMapReq &q = fm.req;
    const size_t nb = size_t(q.nx) * q.ny;
    if (q.per_source) {
        cx->log("flux statistics are computed for whole-element maps, not per-source maps");
        return -1;
    }
    if (fm.counts.size() != nb || cx->sun_rays == 0) {
        cx->log("flux statistics need a completed run");
        return -1;
    }
    const double two_pi = 2.0 * 3.14159265358979323846;
    const double bx = (q.kind == 1 || q.kind >= 3) ? two_pi * q.x1 / q.nx : (q.x1 - q.x0) / q.nx;
    const double by = (q.y1 - q.y0) / q.ny;
    st_b200_flux_stats_t r;
    memset(&r, 0, sizeof r);
    r.power_per_ray = dni * (cx->sun.xmax - cx->sun.xmin) * (cx->sun.ymax - cx->sun.ymin) / double(cx->sun_rays);
    r.bin_area = bx * by;
    const double zs = r.power_per_ray / r.bin_area;
    double sum = 0, sum2 = 0, peak = 0, mn = 1e99;
    unsigned long long npeak = 0, nmin = 0, binned = 0;
    bool have_peak = false;
    for (int ix = 0; ix < q.nx; ++ix)
        for (int iy = 0; iy < q.ny; ++iy) {
            const unsigned long long c = fm.counts[size_t(iy) * q.nx + ix];
            const double z = double(c) * zs;
            binned += c;
            sum += z;
            sum2 += z * z;
            if (z > peak) {
                peak = z;
                npeak = c;
                have_peak = true;
            }
            if (z < mn) {
                mn = z;
                nmin = c;
            }
        }
    const double n = double(nb);
    r.peak_flux = peak;
    r.min_flux = mn;
    r.ave_flux = sum / n;
    r.sigma_flux = sqrt((n * sum2 - sum * sum) / (n * n));
    r.uniformity = r.sigma_flux / r.ave_flux;
    r.peak_flux_uncertainty = have_peak ? 100.0 / sqrt(double(npeak)) : INFINITY;
    r.ave_flux_uncertainty = cx->stats.intersections ? 100.0 / sqrt(double(cx->stats.intersections)) : INFINITY;
    r.rays_binned = binned;
    r.rays_in_peak_bin = npeak;
    r.rays_in_min_bin = nmin;
    *out = r;
    return 1;
}
int st_b200_set_save_stage_data(st_context_t p, int on) {
    CTX(p, -1);
    cx->save_stage_data = on != 0;
    return 1;
}
int st_b200_stage_data_sizes(st_context_t p, st_uint_t *n0, st_uint_t *n1) {
    CTX(p, -1);
    if (n0) *n0 = st_uint_t(cx->stage_s0.size() / 8);
    if (n1) *n1 = st_uint_t(cx->stage_s1.size() / 7);
    return 1;
}
int st_b200_stage_data(st_context_t p, double *s0, double *s1) {
    CTX(p, -1);
    if (s0) std::copy(cx->stage_s0.begin(), cx->stage_s0.end(), s0);
    if (s1) std::copy(cx->stage_s1.begin(), cx->stage_s1.end(), s1);
    return 1;
}
int st_b200_sim_run_replay(st_context_t p, unsigned int seed, st_uint_t n0, const double *s0, st_uint_t n1,
                           const double *s1, int (*cb)(st_uint_t, st_uint_t, st_uint_t, st_uint_t, st_uint_t, void *),
                           void *data) {
    CTX(p, -1);
    if ((n0 && !s0) || (n1 && !s1)) return -1;
    if (n0 == 0 || n1 == 0) {
        // the reference loads saved data only when both parts are non-empty; otherwise it
        // traces from the sun, for as many rays as s1 has rows when it has any
        // (stapi.cpp:700-703, raytrace.cpp:159-163)
        const int keep = cx->raycount;
        if (n1) cx->raycount = int(n1);
        cx->cb = cb;
        cx->cbdata = data;
        const int rc = run(cx, seed);
        cx->raycount = keep;
        return rc;
    }
    if (cx->stages.size() < 2) {
        cx->log("a replay needs at least two stages");
        return -1;
    }
    cx->replay_s0.assign(s0, s0 + 8 * n0);
    cx->replay_s1.assign(s1, s1 + 7 * n1);
    for (st_uint_t k = 0; k < n1; ++k)
        if (!(s1[7 * k + 6] >= 1 && s1[7 * k + 6] < 4294967296.0)) {
            cx->log("replay ray %lu has an invalid ray number", (unsigned long)k);
            return -1;
        }
    cx->cb = cb;
    cx->cbdata = data;
    cx->replaying = true;
    const int rc = run(cx, seed);
    cx->replaying = false;
    cx->replay_s0.clear();
    cx->replay_s1.clear();
    return rc;
}
int st_b200_run_stats(st_context_t p, st_b200_stats *out) {
    CTX(p, -1);
    if (!out) return -1;
    *out = cx->stats;
    return 1;
}
int st_b200_element_counts(st_context_t p, int stage, unsigned long long *first_hits, unsigned long long *absorbed,
                           unsigned long long *delivered) {
    CTX(p, -1);
    if (stage < 1 || size_t(stage) > cx->elem_first.size()) return -1;
    const size_t s = size_t(stage - 1);
    for (size_t i = 0; i < cx->elem_first[s].size(); ++i) {
        if (first_hits) first_hits[i] = cx->elem_first[s][i];
        if (absorbed) absorbed[i] = cx->elem_absorbed[s][i];
        if (delivered) delivered[i] = cx->elem_delivered[s][i];
    }
    return 1;
}

int st_b200_set_max_sun_rays(st_context_t p, unsigned long long n) {
    CTX(p, -1);
    cx->max_sun64 = n;
    return 1;
}
int st_b200_set_ranks(st_context_t p, int rank, int nranks, st_b200_allgather_t allgather,
                      st_b200_allreduce_t allreduce, void *user) {
    CTX(p, -1);
    if (nranks < 1 || rank < 0 || rank >= nranks || (nranks > 1 && (!allgather || !allreduce))) {
        cx->log("st_b200_set_ranks: rank must be in [0, nranks) and both exchange callbacks given for nranks > 1");
        return -1;
    }
    cx->rank = rank;
    cx->nranks = nranks;
    cx->allgather = allgather;
    cx->allreduce = allreduce;
    cx->comm_user = user;
    return 1;
}
int st_b200_sim_run_batch(st_context_t p, unsigned int seed, int n_positions, const double *sun_xyz,
                          const st_uint_t *hits, const double *track_target) {
    CTX(p, -1);
    return run_batch(cx, seed, n_positions, sun_xyz, hits, track_target);
}
int st_b200_batch_stats(st_context_t p, int position, st_b200_stats *out) {
    CTX(p, -1);
    if (!out) return -1;
    if (position < 0) {
        *out = cx->batch_stats;
        return 1;
    }
    if (size_t(position) >= cx->batch.size()) return -1;
    const PositionResult &r = cx->batch[size_t(position)];
    memset(out, 0, sizeof *out);
    out->sun_rays = r.sun_rays;
    out->ray_hits = r.ray_hits;
    out->ray_stage_units = r.sun_rays;
    for (size_t k = 0; k < r.stage_entries.size() && k < 16; ++k) {
        out->stage_entries[k] = r.stage_entries[k];
        if (k >= 1) out->ray_stage_units += r.stage_entries[k];
    }
    out->intersections = r.intersections;
    return 1;
}
int st_b200_batch_flux_counts(st_context_t p, int map, int position, unsigned long long *counts) {
    CTX(p, -1);
    if (!counts || position < 0 || size_t(position) >= cx->batch.size()) return -1;
    const PositionResult &r = cx->batch[size_t(position)];
    if (map < 0 || size_t(map) >= r.flux.size()) return -1;
    std::copy(r.flux[size_t(map)].begin(), r.flux[size_t(map)].end(), counts);
    return 1;
}
int st_b200_batch_absorbed(st_context_t p, int position, int stage, unsigned long long *absorbed) {
    CTX(p, -1);
    if (!absorbed || position < 0 || size_t(position) >= cx->batch.size() || stage < 1 ||
        size_t(stage) > cx->stages.size() || !cx->scene_valid)
        return -1;
    const StageRec &sr = cx->scene_cache.dev.stages[stage - 1];
    const PositionResult &r = cx->batch[size_t(position)];
    std::copy(r.absorbed.begin() + sr.first_elem, r.absorbed.begin() + sr.first_elem + sr.n_elem, absorbed);
    return 1;
}
int st_b200_batch_sun_box(st_context_t p, int position, double *xmin, double *xmax, double *ymin, double *ymax) {
    CTX(p, -1);
    if (position < 0 || size_t(position) >= cx->batch_box.size()) return -1;
    const auto &b = cx->batch_box[size_t(position)];
    if (xmin) *xmin = b[0];
    if (xmax) *xmax = b[1];
    if (ymin) *ymin = b[2];
    if (ymax) *ymax = b[3];
    return 1;
}

}  // extern "C"
