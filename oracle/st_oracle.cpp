// CPU ORACLE — test infrastructure only.
//
// A restatement, in plain C++, of SolTrace coretrace's Monte-Carlo trace behind
// st_sim_run (coretrace/stapi.cpp:680-734 -> coretrace/raytrace.cpp:137-1113).
// Only tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
// this library, and only as the checker; the CUDA product never calls it.
//
// It exports the same flat C API as coretrace/stapi.h (so one scene builder can
// drive the reference, this oracle and the product alike) plus a few st_oracle_*
// extras:
//   * st_oracle_set_rng(ctx, mode): mode 0 replays the reference's libstdc++ stream
//     (minstd_rand0 + polar normals, rejection-sampled sunshapes) so that a run
//     reproduces the reference's records bit for bit; mode 1 uses the per-ray
//     Philox streams and inverse-CDF samplers that the CUDA product uses, so that
//     the GPU trace can be compared ray by ray.
//   * st_oracle_explicit_rays: trace caller-supplied stage-1 rays instead of sun rays.
//   * st_oracle_flux: integer flux bins from the element-local hit positions.
//
// Parity is pinned against the reference compiled from its own sources
// (oracle/Makefile target "ref"): see tests/test_oracle.py and the digests in
// tests/golden/reference_runs.json.
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <strings.h>
#include <vector>
#include <algorithm>

#include "st_oracle_rng.h"

using st_uint_t = unsigned long;
using namespace st_oracle_rng;

namespace {

constexpr double kDegToRad = 0.017453292519943295;  // acos(-1)/180 (types.h:64)
constexpr double kPi = 3.141592653589793238462643;

// ------------------------------------------------------------------------------------
// Scene model (coretrace/types.h:85-343)
// ------------------------------------------------------------------------------------
struct Optics {
    char dist = 'g';
    int optnum = 1, apgr = 0, order = 0;
    double refl = 0, trans = 0, slope = 0, spec = 0;
    double rindex[4] = {0, 0, 0, 0};
    double ab12[4] = {0, 0, 0, 0};
    bool use_refl_table = false, use_trans_table = false;
    std::vector<double> refl_ang, refl_val, trans_ang, trans_val;
};

struct OpticSet {
    std::string name;
    Optics front, back;
};

struct Element {
    bool enabled = true;
    double origin[3] = {0, 0, 0}, aim[3] = {0, 0, 0}, zrot = 0;
    double euler[3] = {0, 0, 0};
    double r_to_loc[3][3] = {{0}}, r_to_ref[3][3] = {{0}};
    char shape = ' ';
    double p[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // aperture parameters A..H
    double aperture_area = 0, z_aperture = 0;
    char surface = ' ';
    int surface_type = 0;
    double kappa = 0, alpha[5] = {0, 0, 0, 0, 0};
    double vcx = 0, vcy = 0, annular_r = 0, cross_r = 0, cone_half_angle = 0, curv_rev = 0;
    int fit_order = 0;
    std::vector<double> bcoef;  // (order+1)^2 row-major, B(i,j) at i*(order+1)+j
    std::vector<double> poly;
    std::vector<double> spl_x, spl_y, spl_y2;
    std::vector<double> vshot;  // rows of 5
    // finite-element surface (.fed): nodes (x, y, z) and the zone grid the reference's
    // st_hash_tree builds over them (treemesh.cpp:353-535): 2^fe_nx x 2^fe_ny zones over
    // the nodes' bounding box; per zone, the nodes of the 3 x 3 zones around it
    std::vector<double> fe_nodes;
    int fe_nx = 0, fe_ny = 0;
    double fe_lim[4] = {0, 0, 0, 0};
    std::vector<int> fe_start, fe_items;
    int vshot_rows = 0;
    int interaction = 0;
    std::string optic_name;
    OpticSet *optics = nullptr;
};

struct Stage {
    bool multihit = true, virt = false, tracethrough = false;
    double origin[3] = {0, 0, 0}, aim[3] = {0, 0, 0}, zrot = 0;
    double euler[3] = {0, 0, 0};
    double r_to_loc[3][3] = {{0}}, r_to_ref[3][3] = {{0}};
    std::vector<Element *> elements;
    ~Stage() {
        for (auto *e : elements) delete e;
    }
};

struct Sun {
    char shape = ' ';
    double sigma = 0;
    bool point_source = false;
    std::vector<double> ang, inten;  // mirrored table (stapi.cpp:529-560)
    double max_angle = 0, max_intensity = 0;
    double origin[3] = {0, 0, 0};
    double euler[3] = {0, 0, 0};
    double r_to_loc[3][3] = {{0}}, r_to_ref[3][3] = {{0}};
    double xmin = 0, xmax = 0, ymin = 0, ymax = 0;
    // inverse-CDF table for the per-ray stream (theta in mrad, cdf in [0,1])
    std::vector<double> cdf_theta, cdf;
};

struct Record {
    double pos[3], cos[3];
    int element, stage;
    unsigned raynum;
    double loc[3];  // element-local hit position (for flux binning)
};

struct Context {
    Sun sun;
    std::vector<OpticSet *> optics;
    std::vector<Stage *> stages;
    int raycount = 1000, raymax = 100000;
    bool dyn_group = false, err_sun = true, err_opt = true;
    std::vector<std::string> messages;
    std::vector<Record> all;  // merged, reference order
    unsigned long sun_ray_count = 0;
    int rng_mode = 0;
    std::vector<double> explicit_pos, explicit_cos;
    std::vector<std::vector<Record>> stage_records;
    ~Context() {
        for (auto *o : optics) delete o;
        for (auto *s : stages) delete s;
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

// ------------------------------------------------------------------------------------
// Linear algebra (coretrace/mathproc.cpp:58-217)
// ------------------------------------------------------------------------------------
inline void mat_vec(const double m[3][3], const double v[3], double o[3]) {
    o[0] = m[0][0] * v[0] + m[0][1] * v[1] + m[0][2] * v[2];
    o[1] = m[1][0] * v[0] + m[1][1] * v[1] + m[1][2] * v[2];
    o[2] = m[2][0] * v[0] + m[2][1] * v[1] + m[2][2] * v[2];
}
inline double dot3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// reference -> local: pos' = R (pos - origin), dir' = R dir   (mathproc.cpp:115-141)
inline void to_local(const double pr[3], const double cr[3], const double org[3], const double R[3][3],
                     double pl[3], double cl[3]) {
    double d[3] = {pr[0] - org[0], pr[1] - org[1], pr[2] - org[2]};
    mat_vec(R, d, pl);
    mat_vec(R, cr, cl);
}
// local -> reference: pos = R^T pos' + origin, dir = R^T dir'   (mathproc.cpp:145-173)
inline void to_ref(const double pl[3], const double cl[3], const double org[3], const double Rt[3][3],
                   double pr[3], double cr[3]) {
    double d[3];
    mat_vec(Rt, pl, d);
    mat_vec(Rt, cl, cr);
    for (int i = 0; i < 3; ++i) pr[i] = d[i] + org[i];
}

// Spencer & Murty eq. 2 rotation from Euler angles (mathproc.cpp:175-217)
void euler_matrices(const double e[3], double R[3][3], double Rt[3][3]) {
    const double ca = cos(e[0]), cb = cos(e[1]), cg = cos(e[2]);
    const double sa = sin(e[0]), sb = sin(e[1]), sg = sin(e[2]);
    R[0][0] = ca * cg + sa * sb * sg;
    R[0][1] = -cb * sg;
    R[0][2] = -sa * cg + ca * sb * sg;
    R[1][0] = ca * sg - sa * sb * cg;
    R[1][1] = cb * cg;
    R[1][2] = -sa * sg - ca * sb * cg;
    R[2][0] = sa * cb;
    R[2][1] = sb;
    R[2][2] = ca * cb;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Rt[i][j] = R[j][i];
}

// origin/aim/zrot -> Euler angles (input.cpp:160-176, stapi.cpp:737-753)
bool aim_euler(const double o[3], const double a[3], double zrot, double e[3]) {
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

// ------------------------------------------------------------------------------------
// Surface helpers (mathproc.cpp:220-330, vshot.cpp:59-139)
// ------------------------------------------------------------------------------------
double eval_poly(double ax, double ay, const std::vector<double> &c, int order) {
    double z = 0.0;
    const double r = sqrt(ax * ax + ay * ay);
    for (int i = 0; i <= order; ++i) z = z + c[i] * pow(r, i);
    return z;
}
void poly_slope(const std::vector<double> &c, int order, double ax, double ay, double *dx, double *dy) {
    double dzdr = 0.0;
    const double r = sqrt(ax * ax + ay * ay);
    const double drdx = ax / r, drdy = ay / r;
    for (int i = 1; i <= order; ++i) dzdr = dzdr + i * c[i] * pow(r, i - 1);
    *dx = dzdr * drdx;
    *dy = dzdr * drdy;
}
inline double bco(const Element *e, int i, int j) { return e->bcoef[i * (e->fit_order + 1) + j]; }
double eval_mono(const Element *e, double x, double y) {
    double z = 0.0;
    for (int i = 0; i <= e->fit_order; ++i)
        for (int j = 0; j <= i; ++j) {
            const double xx = (j == 0) ? 1.0 : pow(x, j);
            const double yy = (i - j == 0) ? 1.0 : pow(y, i - j);
            z = z + bco(e, i, j) * xx * yy;
        }
    return z;
}
void mono_slope(const Element *e, double sx, double sy, double *dzdx, double *dzdy) {
    if (sx == 0.0) sx = sx + 1.0e-10;
    if (sy == 0.0) sy = sy + 1.0e-10;
    *dzdx = 0.0;
    *dzdy = 0.0;
    for (int i = 1; i <= e->fit_order; ++i)
        for (int j = 0; j <= i; ++j) {
            *dzdx = *dzdx + j * bco(e, i, j) * pow(sx, (j - 1)) * pow(sy, (i - j));
            *dzdy = *dzdy + (i - j) * bco(e, i, j) * pow(sx, j) * pow(sy, (i - j - 1));
        }
}
bool splint(const std::vector<double> &xa, const std::vector<double> &ya, const std::vector<double> &y2a,
            double x, double *y, double *dydx) {
    int klo = 0, khi = int(xa.size()) - 1;
    while (khi - klo > 1) {
        const int k = (khi + klo) / 2;
        if (xa[k] > x)
            khi = k;
        else
            klo = k;
    }
    const double h = xa[khi] - xa[klo];
    if (h == 0.0) return false;
    const double a = (xa[khi] - x) / h, b = (x - xa[klo]) / h;
    *y = a * ya[klo] + b * ya[khi] + ((a * a * a - a) * y2a[klo] + (b * b * b - b) * y2a[khi]) * (h * h) / 6.0;
    *dydx = (ya[khi] - ya[klo]) / (xa[khi] - xa[klo]) - (3.0 * a * a - 1.0) * (xa[khi] - xa[klo]) * y2a[klo] / 6.0 +
            (3.0 * b * b - 1.0) * (xa[khi] - xa[klo]) * y2a[khi] / 6.0;
    return true;
}
// natural/clamped cubic spline second derivatives (mathproc.cpp:287-330)
void spline_setup(const std::vector<double> &x, const std::vector<double> &y, double yp1, double ypn,
                  std::vector<double> &y2) {
    const int n = int(x.size());
    std::vector<double> u(n);
    y2.assign(n, 0.0);
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
    double qn, un;
    if (ypn > 0.99e30) {
        qn = 0.0;
        un = 0.0;
    } else {
        qn = 0.5;
        un = (3.0 / (x[n - 1] - x[n - 2])) * (ypn - (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]));
    }
    y2[n - 1] = (un - qn * u[n - 2]) / (qn * y2[n - 2] + 1.0);
    for (int k = n - 2; k >= 0; --k) y2[k] = y2[k] * y2[k + 1] + u[k];
}

// modified Shepard interpolation of VSHOT slopes (vshot.cpp:290-367)
void vshot_slopes(const Element *e, double x, double y, double density, double *zx, double *zy) {
    const double roi2 = 30.0 / density / 3.14159;
    double s = 0.0, wx = 0.0, wy = 0.0;
    for (int i = 0; i < e->vshot_rows; ++i) {
        const double *v = &e->vshot[5 * i];
        const double xx = v[0] - x, yy = v[1] - y;
        if (xx == 0.0 && yy == 0.0) {
            *zx = v[2];
            *zy = v[3];
            return;
        }
        const double r2 = xx * xx + yy * yy;
        if (r2 < roi2) {
            s = s + 1.0 / r2;
            wx = wx + v[2] / r2;
            wy = wy + v[3] / r2;
        }
    }
    if (s == 0.0) {
        *zx = 0.0;
        *zy = 0.0;
        return;
    }
    *zx = wx / s;
    *zy = wy / s;
}

// ------------------------------------------------------------------------------------
// Finite-element surface (vshot.cpp:166-242, interpolate.cpp:5-238, treemesh.cpp)
// ------------------------------------------------------------------------------------
// zone index of (x, y): repeated halving of the bounding box, upper half when strictly
// above the midpoint (st_hash_tree::pos_to_binary, treemesh.cpp:757-800)
static int fe_zone(const Element *e, double x, double y) {
    double x0 = e->fe_lim[0], x1 = e->fe_lim[1], y0 = e->fe_lim[2], y1 = e->fe_lim[3];
    int ix = 0, iy = 0;
    for (int k = 0; k < e->fe_nx; ++k) {
        const double c = (x0 + x1) * 0.5;
        if (x > c) {
            x0 = c;
            ix = 2 * ix + 1;
        } else {
            x1 = c;
            ix = 2 * ix;
        }
    }
    for (int k = 0; k < e->fe_ny; ++k) {
        const double c = (y0 + y1) * 0.5;
        if (y > c) {
            y0 = c;
            iy = 2 * iy + 1;
        } else {
            y1 = c;
            iy = 2 * iy;
        }
    }
    return iy * (1 << e->fe_nx) + ix;
}

// Build the zone grid of the nodes (input.cpp:510-557 -> st_hash_tree): zone size from
// 1.5 sqrt(area per node), levels floor(log2(extent / size)) >= 1 per axis.  A zone's
// candidate list: its own nodes, then those of its 8 neighbours (x offset outer loop, y
// inner, treemesh.cpp:448-485); zones with no node in their 3 x 3 block have none.
static void fe_build(Element *e) {
    const size_t n = e->fe_nodes.size() / 3;
    double xmin = 1.79769313486231570e308, ymin = xmin, xmax = -xmin, ymax = -xmin;
    for (size_t i = 0; i < n; ++i) {
        const double x = e->fe_nodes[3 * i], y = e->fe_nodes[3 * i + 1];
        xmax = x > xmax ? x : xmax;
        ymax = y > ymax ? y : ymax;
        xmin = x < xmin ? x : xmin;
        ymin = y < ymin ? y : ymin;
    }
    e->fe_lim[0] = xmin;
    e->fe_lim[1] = xmax;
    e->fe_lim[2] = ymin;
    e->fe_lim[3] = ymax;
    const double rap = 1.5 * sqrt(((xmax - xmin) * (ymax - ymin)) / (double)n);
    const double l2i = 1. / log(2.);
    e->fe_nx = (int)floor(log((xmax - xmin) / rap) * l2i);
    e->fe_nx = e->fe_nx < 1 ? 1 : e->fe_nx;
    e->fe_ny = (int)floor(log((ymax - ymin) / rap) * l2i);
    e->fe_ny = e->fe_ny < 1 ? 1 : e->fe_ny;
    const int nx = 1 << e->fe_nx, ny = 1 << e->fe_ny;
    std::vector<std::vector<int>> zone(size_t(nx) * ny);
    for (size_t i = 0; i < n; ++i) zone[fe_zone(e, e->fe_nodes[3 * i], e->fe_nodes[3 * i + 1])].push_back(int(i));
    e->fe_start.assign(size_t(nx) * ny + 1, 0);
    e->fe_items.clear();
    for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
            const int z = iy * nx + ix;
            e->fe_start[z] = int(e->fe_items.size());
            e->fe_items.insert(e->fe_items.end(), zone[z].begin(), zone[z].end());
            for (int i = -1; i < 2; ++i)
                for (int j = -1; j < 2; ++j) {
                    if (i == 0 && j == 0) continue;
                    const int jx = ix + i, jy = iy + j;
                    if (jx < 0 || jx >= nx || jy < 0 || jy >= ny) continue;
                    const auto &l = zone[size_t(jy) * nx + jx];
                    e->fe_items.insert(e->fe_items.end(), l.begin(), l.end());
                }
        }
    e->fe_start[size_t(nx) * ny] = int(e->fe_items.size());  // zone z: [fe_start[z], fe_start[z + 1])
}

// Kriging with a power-law variogram (Numerical Recipes 3rd ed. section 3.7.4, the Krig
// and Powvargram structures, with an LU decomposition with implicit partial pivoting, section
// 2.3), in the reference's arithmetic order (interpolate.cpp:5-238).
struct FeKrig {
    int n = 0;
    double x[7][2], alph = 0, bet = 1.999;
    double lu[8][8];
    int indx[8];
    double yvi[8];
    double pvg(double r) const { return 0.0 + alph * pow(r, bet); }
    static double sq(double a) { return a * a; }
    double rdist(const double *a, const double *b) const {
        double d = 0.;
        for (int k = 0; k < 2; ++k) d += sq(a[k] - b[k]);
        return sqrt(d);
    }
    void setup(const double (*px)[2], const double *py, int npt) {
        n = npt;
        for (int i = 0; i < n; ++i) {
            x[i][0] = px[i][0];
            x[i][1] = px[i][1];
        }
        double num = 0., denom = 0.;
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++) {
                double rb = 0.;
                for (int k = 0; k < 2; k++) rb += sq(x[i][k] - x[j][k]);
                rb = pow(rb, 0.5 * bet);
                num += rb * (0.5 * sq(py[i] - py[j]) - 0.0);
                denom += sq(rb);
            }
        alph = num / denom;
        const int m = n + 1;
        for (int i = 0; i < n; i++) {
            for (int j = i; j < n; j++) lu[i][j] = lu[j][i] = pvg(rdist(x[i], x[j]));
            lu[i][n] = lu[n][i] = 1.;
        }
        lu[n][n] = 0.;
        double y[8];
        for (int i = 0; i < n; ++i) y[i] = py[i];
        y[n] = 0.;
        // decomposition
        double vv[8];
        for (int i = 0; i < m; i++) {
            double big = 0.0, t;
            for (int j = 0; j < m; j++)
                if ((t = fabs(lu[i][j])) > big) big = t;
            vv[i] = 1.0 / big;
        }
        for (int k = 0; k < m; k++) {
            double big = 0.0, t;
            int imax = k;
            for (int i = k; i < m; i++) {
                t = vv[i] * fabs(lu[i][k]);
                if (t > big) {
                    big = t;
                    imax = i;
                }
            }
            if (k != imax) {
                for (int j = 0; j < m; j++) {
                    t = lu[imax][j];
                    lu[imax][j] = lu[k][j];
                    lu[k][j] = t;
                }
                vv[imax] = vv[k];
            }
            indx[k] = imax;
            if (lu[k][k] == 0.0) lu[k][k] = 1.0e-40;
            for (int i = k + 1; i < m; i++) {
                t = lu[i][k] /= lu[k][k];
                for (int j = k + 1; j < m; j++) lu[i][j] -= t * lu[k][j];
            }
        }
        // solve for the weights
        int ii = 0;
        for (int i = 0; i < m; i++) yvi[i] = y[i];
        for (int i = 0; i < m; i++) {
            const int ip = indx[i];
            double sum = yvi[ip];
            yvi[ip] = yvi[i];
            if (ii != 0)
                for (int j = ii - 1; j < i; j++) sum -= lu[i][j] * yvi[j];
            else if (sum != 0.0)
                ii = i + 1;
            yvi[i] = sum;
        }
        for (int i = m - 1; i >= 0; i--) {
            double sum = yvi[i];
            for (int j = i + 1; j < m; j++) sum -= lu[i][j] * yvi[j];
            yvi[i] = sum / lu[i][i];
        }
    }
    double interp(const double *xs) const {
        double v = 0.;
        for (int i = 0; i < n; i++) v += yvi[i] * pvg(rdist(xs, x[i]));
        v += yvi[n] * 1.;
        return v;
    }
};

static bool g_fe_failed = false;  // a finite-element query found fewer than 3 nodes

// surface z and its finite-difference slopes at (X, Y): kriging on the 7 nearest candidate
// nodes (FEInterpKD, vshot.cpp:166-215); false when fewer than 3 candidates
static bool fe_interp(const Element *e, double X, double Y, double step, double *zr, double *zx, double *zy) {
    const int z = fe_zone(e, X, Y);
    const int a = e->fe_start[z], b = e->fe_start[z + 1];
    if (b - a < 3) return false;
    std::vector<std::pair<double, int>> nd;
    for (int k = a; k < b; ++k) {
        const double *v = &e->fe_nodes[3 * size_t(e->fe_items[k])];
        nd.push_back({sqrt(pow(X - v[0], 2) + pow(Y - v[1], 2)), e->fe_items[k]});
    }
    std::sort(nd.begin(), nd.end(),
              [](const std::pair<double, int> &p, const std::pair<double, int> &q) { return p.first < q.first; });
    const int m = (int)nd.size() > 7 ? 7 : (int)nd.size();
    double px[7][2], py[7];
    for (int i = 0; i < m; ++i) {
        const double *v = &e->fe_nodes[3 * size_t(nd[i].second)];
        px[i][0] = v[0];
        px[i][1] = v[1];
        py[i] = v[2];
    }
    FeKrig gm;
    gm.setup(px, py, m);
    double xy[2] = {X, Y};
    *zr = gm.interp(xy);
    xy[0] += step;
    const double za = gm.interp(xy);
    xy[0] -= step;
    xy[1] += step;
    const double zb = gm.interp(xy);
    *zx = (*zr - za) / step;
    *zy = (*zr - zb) / step;
    return true;
}

// ------------------------------------------------------------------------------------
// Implicit surface F and grad F (surface.cpp:57-413); returns error flag.
// May overwrite pos[2] with the surface z for data surfaces (surface.cpp:193,246,266,292,332).
// ------------------------------------------------------------------------------------
int surface_eval(double pos[3], const Element *e, double *F, double dF[3]) {
    const double X = pos[0], Y = pos[1], Z = pos[2];
    double dfx = 0, dfy = 0, dfz = 0;
    int err = 0;
    switch (e->surface_type) {
        case 1:
        case 7: {
            const double rho2 = (e->surface_type == 1) ? X * X + Y * Y : X * X;
            if (e->cone_half_angle != 0.0) {
                *F = Z - sqrt(rho2) / tan(e->cone_half_angle * kDegToRad);
                dfx = -X / (sqrt(rho2) * tan(e->cone_half_angle * kDegToRad));
                dfy = -Y / (sqrt(rho2) * tan(e->cone_half_angle * kDegToRad));
                dfz = 1.0;
                break;
            }
            const double sum1 = 0.0, sum2 = 0.0;
            const double q = e->vcx * e->vcx * X * X + e->vcy * e->vcy * Y * Y;
            if (1.0 - e->kappa * q < 0) err = 1;
            const double term = sqrt(1.0 - e->kappa * q);
            *F = Z - (e->vcx * X * X + e->vcy * Y * Y) / (1.0 + term) - sum2;
            dfx = -X * (e->vcx / term + 2.0 * sum1);
            dfy = -Y * (e->vcy / term + 2.0 * sum1);
            dfz = 1.0;
            break;
        }
        case 3:
            dfx = e->alpha[0];
            dfy = e->alpha[1];
            dfz = e->alpha[2];
            *F = dfx * X + dfy * Y + dfz * Z - e->alpha[3];
            break;
        case 4: {  // finite-element data (surface.cpp:217-241)
            if (X * X + Y * Y == 0.0) {
                *F = Z;
                dfz = 1;
                break;
            }
            const double density = (double)(e->fe_nodes.size() / 3) / e->aperture_area;
            const double delta = 0.001 / sqrt(density);
            double zr = 0, zx = 0, zy = 0;
            if (!fe_interp(e, X, Y, delta, &zr, &zx, &zy)) {
                // the reference throws here and the run does not return
                g_fe_failed = true;
                err = 1;
                break;
            }
            pos[2] = zr;
            *F = Z - zr;
            dfx = zx;
            dfy = zy;
            dfz = 1.0;
            break;
        }
        case 5: {
            if (X * X + Y * Y == 0.0) {
                *F = Z;
                dfx = dfy = 0.0;
                dfz = 1.0;
                break;
            }
            const double zm = eval_mono(e, X, Y);
            const double density = e->vshot_rows / e->aperture_area;
            double zx, zy;
            vshot_slopes(e, X, Y, density, &zx, &zy);
            pos[2] = zm;
            *F = Z - zm;
            dfx = -tan(zx);
            dfy = -tan(zy);
            dfz = 1.0;
            break;
        }
        case 6: {
            const double zz = eval_mono(e, X, Y);
            double sx, sy;
            mono_slope(e, X, Y, &sx, &sy);
            pos[2] = zz;
            *F = Z - zz;
            dfx = -sx;
            dfy = -sy;
            dfz = 1.0;
            break;
        }
        case 8: {
            const double yv = (e->shape == 'l' || e->shape == 'L') ? 0.0 : Y;
            const double zz = eval_poly(X, yv, e->poly, e->fit_order);
            double sx, sy;
            poly_slope(e->poly, e->fit_order, X, yv, &sx, &sy);
            pos[2] = zz;
            *F = Z - zz;
            dfx = -sx;
            dfy = -sy;
            dfz = 1.0;
            break;
        }
        case 9: {
            double rho = sqrt(X * X + Y * Y), drx = X / rho, dry = Y / rho;
            if (e->shape == 'l' || e->shape == 'L') {
                rho = X;
                drx = 1.0;
                dry = 0.0;
            }
            double zz, dz;
            if (!splint(e->spl_x, e->spl_y, e->spl_y2, rho, &zz, &dz)) return 3;
            pos[2] = zz;
            *F = Z - zz;
            dfx = -(dz * drx);
            dfy = -(dz * dry);
            dfz = 1.0;
            break;
        }
        default:
            // type 4 (finite-element data surface) is not restated
            return 4;
    }
    dF[0] = dfx;
    dF[1] = dfy;
    dF[2] = dfz;
    return err;
}

// surface z at (x,y) for the Newton start-plane choice (surfacezatxypair.cpp:56-280)
double surface_z_at(const double pos[3], const Element *e) {
    const double X = pos[0], Y = pos[1];
    switch (e->surface_type) {
        case 1:
        case 7: {
            const double rho2 = (e->surface_type == 1) ? X * X + Y * Y : X * X;
            if (e->cone_half_angle != 0.0) return sqrt(rho2) / tan(e->cone_half_angle * kDegToRad);
            const double q = e->vcx * e->vcx * X * X + e->vcy * e->vcy * Y * Y;
            if (e->kappa * q > 1.0) return 0.0;
            return (e->vcx * X * X + e->vcy * Y * Y) / (1.0 + sqrt(1.0 - e->kappa * q));
        }
        case 5:
            if (X * X + Y * Y == 0.0) return 0.0;
            return eval_mono(e, X, Y);
        case 6:
            return eval_mono(e, X, Y);
        case 8: {
            const double yv = (e->shape == 'l' || e->shape == 'L') ? 0.0 : Y;
            return eval_poly(X, yv, e->poly, e->fit_order);
        }
        default:
            return 0.0;
    }
}

// ------------------------------------------------------------------------------------
// Aperture membership (determineelementintersectionnew.cpp:109-624, intersect.cpp:119-138,270-547)
// ------------------------------------------------------------------------------------
inline int sgn_nonneg(double v) { return v >= 0; }
int in_tri(double x1, double y1, double x2, double y2, double x3, double y3, double xt, double yt) {
    const double a = (x1 - xt) * (y2 - yt) - (x2 - xt) * (y1 - yt);
    const double b = (x2 - xt) * (y3 - yt) - (x3 - xt) * (y2 - yt);
    const double c = (x3 - xt) * (y1 - yt) - (x1 - xt) * (y3 - yt);
    return sgn_nonneg(a) == sgn_nonneg(b) && sgn_nonneg(b) == sgn_nonneg(c);
}
int in_quad(const double *p, double x, double y) {
    return in_tri(p[0], p[1], p[2], p[3], p[4], p[5], x, y) || in_tri(p[0], p[1], p[4], p[5], p[6], p[7], x, y);
}

constexpr double kSlope60 = 1.7320508075688767;

// 1 inside, 0 outside, -1 "no section matched" (hexagon/triangle fall-through).
// 'start_plane' selects the rectangle rule of intersect.cpp:402-412, whose conditions
// can never be true (so every point counts as inside).
int aperture_contains(const Element *e, double x, double y, bool start_plane) {
    const double r = sqrt(x * x + y * y);
    switch (e->shape) {
        case 'c':
        case 'C':
            return r > e->p[0] / 2.0 ? 0 : 1;
        case 'h':
        case 'H': {
            const double ro = e->p[0] / 2.0;
            if (r > ro) return 0;
            const double ri = ro * cos(30.0 * kDegToRad);
            if (r <= ri) return 1;
            const double xl = sqrt(ro * ro - ri * ri);
            if (x <= ro && x > xl) {
                const double y1 = kSlope60 * (x - ro);
                return (y >= y1 && y <= -y1) ? 1 : 0;
            }
            if (x <= xl && x >= -xl) return (y >= -ri && y <= ri) ? 1 : 0;
            if (x < -xl && x >= -ro) {
                const double y3 = kSlope60 * (x + ro);
                return (y >= -y3 && y <= y3) ? 1 : 0;
            }
            return -1;
        }
        case 't':
        case 'T': {
            const double ro = e->p[0] / 2.0;
            if (r > ro) return 0;
            const double ri = ro * sin(30.0 * kDegToRad);
            if (r <= ri) return 1;
            if (x <= ro && x > 0.0) {
                const double y1 = -kSlope60 * (x - ri / cos(30.0 * kDegToRad));
                return (y <= y1 && y >= -ri) ? 1 : 0;
            }
            if (x >= -ro && x <= 0.0) {
                const double y3 = kSlope60 * (x + ri / cos(30.0 * kDegToRad));
                return (y >= -ri && y <= y3) ? 1 : 0;
            }
            return -1;
        }
        case 'r':
        case 'R':
            if (start_plane) return 1;
            if (x > e->p[0] / 2.0 || x < -e->p[0] / 2.0) return 0;
            if (y > e->p[1] / 2.0 || y < -e->p[1] / 2.0) return 0;
            return 1;
        case 'a':
        case 'A': {
            if (!(start_plane == false && e->p[0] == 0.0 && e->p[1] == 0.0))
                if (r < e->p[0] || r > e->p[1]) return 0;
            const double half = e->p[2] * kDegToRad / 2.0;
            if (x >= 0.0) return (asin(y / r) > half || asin(y / r) < -half) ? 0 : 1;
            if (y >= 0 && (acos(y / r) + kPi / 2.0) > half) return 0;
            if (y < 0 && (-acos(-y / r) - kPi / 2.0) < -half) return 0;
            return 1;
        }
        case 'l':
        case 'L':
            if (!(e->p[0] == 0.0 && e->p[1] == 0.0))
                if (x < e->p[0] || x > e->p[1]) return 0;
            if (y < -e->p[2] / 2.0 || y > e->p[2] / 2.0) return 0;
            return 1;
        case 'i':
        case 'I':
            return in_tri(e->p[0], e->p[1], e->p[2], e->p[3], e->p[4], e->p[5], x, y) ? 1 : 0;
        case 'q':
        case 'Q':
            return in_quad(e->p, x, y) ? 1 : 0;
        default:
            return -1;
    }
}

// ------------------------------------------------------------------------------------
// Closed forms (quadricsurfaceclosedform.cpp:58-308, torusclosedform.cpp:57-188, root432.cpp)
// ------------------------------------------------------------------------------------
// The reference spells squares as an unparenthesised macro, sqr(x) -> (x*x); the
// normal's terms therefore evaluate as ((((2*K*d)/a2)*2)*K*d)/a2.
inline double sq_macro(double twoK, double d, double a2) { return (((twoK * d) / a2) * twoK * d) / a2; }

int quadric_closed(const Element *e, const double P[3], const double D[3], double out[3], double n[3], double *plen) {
    double xc = 0, yc = 0, zc = 0, kx = 0, ky = 0, kz = 0, r2 = 0, a2 = 0, b2 = 0, c2 = 0, A = 0, B = 0, C = 0;
    const char s = e->surface;
    if (s == 's' || s == 'S') {
        a2 = b2 = c2 = 1;
        kx = 1;
        ky = (e->surface_type == 7) ? 0 : 1;
        kz = 1;
        const double r = 1.0 / e->vcx;
        r2 = r * r;
        zc = r;
        const double xd = P[0] - xc, yd = P[1] - yc, zd = P[2] - zc;
        A = D[0] * D[0] * kx / a2 + D[1] * D[1] * ky / b2 + D[2] * D[2] * kz / c2;
        B = 2.0 * (kx * xd * D[0] / a2 + ky * yd * D[1] / b2 + kz * zd * D[2] / c2);
        C = kx * xd * xd / a2 + ky * yd * yd / b2 + kz * zd * zd / c2 - r2;
    } else if (s == 'p' || s == 'P') {
        a2 = 2.0 / e->vcx;
        b2 = e->vcy > 0.0 ? 2.0 / e->vcy : 1e10;
        c2 = 1.0;
        kx = 1;
        ky = (e->surface_type == 7) ? 0 : 1;
        kz = 0;
        const double xd = P[0] - xc, yd = P[1] - yc, zd = P[2] - zc;
        A = D[0] * D[0] * kx / a2 + D[1] * D[1] * ky / b2;
        B = 2.0 * (kx * xd * D[0] / a2 + ky * yd * D[1] / b2) - D[2] / c2;
        C = kx * xd * xd / a2 + ky * yd * yd / b2 - zd / c2;
    } else if (s == 'o' || s == 'O') {
        a2 = b2 = c2 = 1;
        kx = ky = 1;
        kz = e->kappa;
        zc = 1.0 / e->kappa / e->vcx;
        const double xd = P[0] - xc, yd = P[1] - yc, zd = P[2] - zc;
        A = D[0] * D[0] * kx / a2 + D[1] * D[1] * ky / b2 + D[2] * D[2] * kz / c2;
        B = 2.0 * (kx * xd * D[0] / a2 + ky * yd * D[1] / b2 + kz * zd * D[2] / c2);
        C = kx * xd * xd / a2 + ky * yd * yd / b2 + kz * zd * zd / c2 - 1.0 / e->kappa / (e->vcx * e->vcx);
    } else if (s == 't' || s == 'T') {
        a2 = b2 = c2 = 1;
        kx = 1;
        ky = 0;
        kz = 1;
        const double r = 1.0 / e->curv_rev;
        r2 = r * r;
        zc = r;
        const double xd = P[0] - xc, yd = P[1] - yc, zd = P[2] - zc;
        A = D[0] * D[0] * kx / a2 + D[1] * D[1] * ky / b2 + D[2] * D[2] * kz / c2;
        B = 2.0 * (kx * xd * D[0] / a2 + ky * yd * D[1] / b2 + kz * zd * D[2] / c2);
        C = kx * xd * xd / a2 + ky * yd * yd / a2 + kz * zd * zd / c2 - r2;
    }
    double t;
    if (fabs(A) < 1e-12) {
        const double t1 = -C / B;
        if (t1 > 0) {
            t = t1;
        } else {
            *plen = 0.0;
            return 1;
        }
    } else if (B * B > 4.0 * A * C) {
        const double t1 = (-B + sqrt(B * B - 4.0 * A * C)) / (2.0 * A);
        const double t2 = (-B - sqrt(B * B - 4.0 * A * C)) / (2.0 * A);
        if (t2 > 0) {
            t = t2;
            double z2 = P[2] + t2 * D[2];
            if (z2 > e->z_aperture) t = t1;
            const bool finite_len = (s == 't' || s == 'T') || ((s == 's' || s == 'S') && e->surface_type == 7);
            if (finite_len) {
                const double yt = P[1] + t * D[1];
                if (yt < -e->p[2] / 2.0 || yt > e->p[2] / 2.0) t = t1;
            }
        } else if (t2 == 0) {
            t = t1;
        } else if (t2 < 0 && t1 > 0) {
            t = t1;
        } else {
            *plen = t1;
            return 1;
        }
    } else {
        *plen = 0.0;
        return 1;
    }
    out[0] = P[0] + t * D[0];
    out[1] = P[1] + t * D[1];
    out[2] = P[2] + t * D[2];
    *plen = t;
    double sm;
    if (s == 'p' || s == 'P') {
        sm = sqrt(sq_macro(2.0 * kx, out[0] - xc, a2) + sq_macro(2.0 * ky, out[1] - yc, b2) + 1.0);
        n[0] = -(2.0 * kx * (out[0] - xc) / a2) / sm;
        n[1] = -(2.0 * ky * (out[1] - yc) / b2) / sm;
        n[2] = 1.0 / sm;
    } else {
        sm = sqrt(sq_macro(2.0 * kx, out[0] - xc, a2) + sq_macro(2.0 * ky, out[1] - yc, b2) +
                  sq_macro(2.0 * kz, out[2] - zc, c2));
        n[0] = -(2.0 * kx * (out[0] - xc) / a2) / sm;
        n[1] = -(2.0 * ky * (out[1] - yc) / b2) / sm;
        n[2] = -(2.0 * kz * (out[2] - zc) / c2) / sm;
    }
    return 0;
}

// Quartic roots by Ferrari reduction with a bisected resolvent cubic (root432.cpp:53-284).
struct Quartic {
    double a[5][5];
    double r[5];
    double aa = 0, b = 0, c = 0, d = 0, ii = 0, im = 0, k = 0, l = 0, m = 0, q = 0, rr = 0, s = 0, sw = 0;
    double f(double x) const { return x * x * x + a[3][2] * x * x + a[3][1] * x + a[3][0]; }
    void root2() {
        const double w = a[2][1] * a[2][1] - 4 * a[2][0];
        const double q1 = -a[2][1] / 2.0;
        if (w < 0) {
            im = sqrt(-w) / 2.0;
            r[1] = q1;
            r[2] = q1;
        } else if (w == 0) {
            r[1] = q1;
            r[2] = q1;
            im = 0.0;
        } else if (w > 0) {
            const double q2 = sqrt(w) / 2.0;
            im = 0.0;
            r[1] = q1 + q2;
            r[2] = q1 - q2;
        }
    }
    void root3() {
        double xc;
        if (a[3][0] == 0) {
            xc = 0;
        } else {
            double am = fabs(a[3][0]);
            for (int i = 1; i <= 3; ++i) {
                const double tt = fabs(a[3][i]);
                if (am < tt) am = tt;
            }
            double lo, hi;
            if (a[3][0] > 0) {
                lo = -am - 1;
                hi = 0;
            } else {
                lo = 0;
                hi = am + 1;
            }
            aa = lo;
            b = hi;
            double xa = lo, xb = hi;
            const double y1 = f(lo), y2 = f(hi);
            const double er = 0.000001;
            if (y1 == 0) {
                xc = lo;
            } else if (y2 == 0) {
                xc = hi;
            } else {
                for (;;) {
                    xc = (xa + xb) / 2.0;
                    const double te = f(xc);
                    if (te == 0) break;
                    if (xb - xa < er) break;
                    if (f(xa) * te > 0)
                        xa = xc;
                    else
                        xb = xc;
                }
            }
        }
        r[3] = xc;
        if (sw == -1) return;
        a[2][1] = a[3][2] + xc;
        a[2][0] = a[3][1] + a[3][2] * xc + xc * xc;
        root2();
    }
    void solve4() {
        const int n = 4;
        for (int i = 0; i < n; ++i) a[n][i] = a[n][i] / a[n][n];
        aa = a[4][3];
        b = a[4][2];
        c = a[4][1];
        d = a[4][0];
        q = b - (3.0 * aa * aa / 8.0);
        rr = c - (aa * b / 2) + (aa * aa * aa / 8.0);
        s = d - (aa * c / 4) + (aa * aa * b / 16.0) - (3 * aa * aa * aa * aa / 256.0);
        a[3][2] = q / 2.0;
        a[3][1] = (q * q - 4 * s) / 16.0;
        a[3][0] = -(rr * rr / 64.0);
        if ((rr != 0) || (a[3][1] >= 0)) {
            sw = -1;
            root3();
        } else {
            a[2][1] = a[3][2];
            a[2][0] = a[3][1];
            root2();
            r[3] = r[1];
        }
        k = sqrt(r[3]);
        if (k == 0) {
            rr = sqrt(q * q - 4 * s);
        } else {
            q = q + (4 * r[3]);
            rr = rr / (2 * k);
        }
        l = (q - rr) / 2.0;
        m = (q + rr) / 2.0;
        a[2][1] = 2 * k;
        a[2][0] = l;
        root2();
        r[3] = r[1] - (a[4][3] / 4);
        r[4] = r[2] - (a[4][3] / 4.0);
        ii = im;
        a[2][1] = -2 * k;
        a[2][0] = m;
        root2();
        r[2] = r[2] - (a[4][3] / 4.0);
        r[1] = r[1] - (a[4][3] / 4.0);
    }
};

// insertion sort of arr[0..n-1] as written in mathproc.cpp:333-348 (including its
// placement of a new minimum at index 1)
void pik_sort(int n, double arr[5]) {
    for (int j = 1; j < n; ++j) {
        const double a = arr[j];
        int i;
        for (i = j - 1; i >= 0; --i) {
            if (arr[i] <= a) break;
            arr[i + 1] = arr[i];
        }
        if (i < 0) i = 0;
        arr[i + 1] = a;
    }
}

int torus_closed(const Element *e, const double P[3], const double D[3], double out[3], double n[3], double *plen) {
    const double Rs = e->cross_r, Ra = e->annular_r;
    const double Xo = P[0], Yo = P[1], Zo = P[2];
    const double Ep = D[0], Et = D[1], Rh = D[2];
    Quartic qs;
    for (int i = 0; i < 5; ++i) {
        qs.r[i] = 0.0;
        for (int j = 0; j < 5; ++j) qs.a[i][j] = 0.0;
    }
    qs.a[4][4] = pow(Ep, 4) + 2.0 * Ep * Ep * (Et * Et + Rh * Rh) + pow(Et, 4) + 2.0 * Et * Et * Rh * Rh + pow(Rh, 4);
    qs.a[4][3] = 4.0 * (Ep * Ep + Et * Et + Rh * Rh) * (Ep * Xo + Et * Yo + Rh * Zo - Rh * Rs);
    qs.a[4][2] = Xo * Xo * (6.0 * Ep * Ep + 2.0 * Et * Et + 2.0 * Rh * Rh) + 8.0 * Ep * Xo * (Et * Yo + Rh * Zo - Rh * Rs) +
                 2.0 * Yo * Yo * (Ep * Ep + 3.0 * Et * Et + Rh * Rh) + 8.0 * Et * Rh * Yo * (Zo - Rs) +
                 (Ep * Ep + Et * Et + 3.0 * Rh * Rh) * (2.0 * Zo * Zo - 4.0 * Rs * Zo) -
                 2.0 * Ra * Ra * (Ep * Ep + Et * Et - Rh * Rh) + 4.0 * Rh * Rh * Rs * Rs;
    qs.a[4][1] = 4.0 * (Xo * Xo * (Ep * Xo + Et * Yo + Rh * Zo - Rh * Rs) + Yo * Yo * (Ep * Xo + Et * Yo + Rh * Zo - Rh * Rs) +
                        Zo * Zo * (Ep * Xo + Et * Yo + Rh * Zo - 3.0 * Rh * Rs) - 2.0 * Ep * Rs * Xo * Zo - Ep * Ra * Ra * Xo -
                        2.0 * Et * Rs * Yo * Zo - Et * Ra * Ra * Yo + Rh * Ra * Ra * (Zo - Rs) + 2.0 * Rh * Rs * Rs * Zo);
    qs.a[4][0] = pow(Xo, 4) + 2.0 * Xo * Xo * (Yo * Yo + Zo * Zo - 2.0 * Rs * Zo - Ra * Ra) + pow(Yo, 4) +
                 2.0 * Yo * Yo * (Zo * Zo - 2.0 * Rs * Zo - Ra * Ra) + pow(Zo, 4) - 4.0 * Rs * Zo * Zo * Zo +
                 2.0 * Ra * Ra * Zo * Zo + 4.0 * Rs * Rs * Zo * Zo - 4.0 * Ra * Ra * Rs * Zo + pow(Ra, 4);
    qs.solve4();
    double rv[5] = {qs.r[0], qs.r[1], qs.r[2], qs.r[3], qs.r[4]};
    const double im1 = qs.im, im2 = qs.ii;
    double pl = 0.0;
    if (im1 == 0.0 && im2 == 0.0) {
        pik_sort(4, rv);
        if (rv[4] <= 0.0) {
            *plen = rv[4];
            return 1;
        }
        pl = rv[4];
        if (rv[3] > 0.0) {
            pl = rv[3];
            if (rv[2] > 0.0) {
                pl = rv[2];
                if (rv[1] > 0.0) pl = rv[1];
            }
        }
    } else if (im1 == 0.0 && im2 != 0.0) {
        pl = (rv[1] <= rv[2]) ? rv[1] : rv[2];
    } else if (im1 != 0.0 && im2 == 0.0) {
        pl = (rv[3] <= rv[4]) ? rv[3] : rv[4];
    } else {
        pl = 0.0;
    }
    *plen = pl;
    if (pl == 0.0) return 1;
    const double X = Xo + pl * Ep, Y = Yo + pl * Et, Z = Zo + pl * Rh;
    const double fx = -2.0 * X * (Ra - sqrt(X * X + Y * Y)) / sqrt(X * X + Y * Y);
    const double fy = -2.0 * Y * (Ra - sqrt(X * X + Y * Y)) / sqrt(X * X + Y * Y);
    const double fz = 2.0 * (Z - Rs);
    out[0] = X;
    out[1] = Y;
    out[2] = Z;
    n[0] = -fx;
    n[1] = -fy;
    n[2] = -fz;
    return 0;
}

// Cubic-spline start plane (newzstartforcubicsplinesurf.cpp:57-142)
int spline_zstart(double cr, const double P[3], const double D[3], char ap, double *z0) {
    if (ap == 'a' || ap == 'A') {
        const double A = D[0] * D[0] + D[1] * D[1];
        const double B = 2.0 * (P[0] * D[0] + P[1] * D[1]);
        const double C = P[0] * P[0] + P[1] * P[1] - cr * cr;
        if (B * B > 4.0 * A * C) {
            const double t1 = (-B + sqrt(B * B - 4.0 * A * C)) / (2.0 * A);
            const double t2 = (-B - sqrt(B * B - 4.0 * A * C)) / (2.0 * A);
            if (t2 > 0) {
                *z0 = P[2] + t2 * D[2];
                return 0;
            }
            if (t2 == 0 || (t2 < 0 && t1 > 0)) {
                *z0 = P[2] + t1 * D[2];
                return 0;
            }
            return 1;
        }
        return 2;
    }
    if (ap == 'l' || ap == 'L') {
        const double t1 = (cr - P[0]) / D[0];
        if (t1 >= 0.0) {
            *z0 = P[2] + t1 * D[2];
            return 0;
        }
        return 1;
    }
    return 0;
}

// Starting plane for the spline Newton iteration (intersect.cpp:597-945)
double spline_start(const Element *e, const double P[3], const double D[3], int *err) {
    const double outer = e->spl_x.back(), inner = e->spl_x.front();
    const char ap = e->shape;
    const bool annular = (ap == 'a' || ap == 'A'), line = (ap == 'l' || ap == 'L');
    const double ZA = e->spl_y.back();
    const double s00 = -P[2] / (D[2] + 0.00000000001);
    const double X10 = P[0] + D[0] * s00, Y10 = P[1] + D[1] * s00, R10 = sqrt(X10 * X10 + Y10 * Y10);
    const double s0a = (ZA - P[2]) / (D[2] + 0.00000000001);
    const double X1A = P[0] + D[0] * s0a, Y1A = P[1] + D[1] * s0a, R1A = sqrt(X1A * X1A + Y1A * Y1A);
    double z = 0.0, zc;
    auto outer_test = [&](double R, double X) { return (annular && R > outer) || (line && X > outer); };
    auto outer_ge = [&](double R, double X) { return (annular && R >= outer) || (line && X >= outer); };
    auto outer_le = [&](double R, double X) { return (annular && R <= outer) || (line && X <= outer); };
    auto inner_le = [&](double R, double X) { return (annular && R <= inner) || (line && X <= inner); };
    auto between = [&](double R, double X) {
        return (annular && R < outer && R > inner) || (line && X < outer && X > inner);
    };
    if (P[2] >= ZA && D[2] < 0.0) {
        const double PA[3] = {X1A, Y1A, ZA};
        if (outer_test(R1A, X1A)) {
            if (spline_zstart(outer * 0.999999, PA, D, ap, &zc) == 0) z = zc;
            return z;
        }
        if (outer_le(R1A, X1A)) {
            if (outer_ge(R10, X10)) {
                if (spline_zstart(outer * 0.999999, PA, D, ap, &zc) == 0) z = zc;
                return z;
            }
            return 0.0;
        }
    }
    if (P[2] <= 0.0 && D[2] > 0.0) {
        const double P0[3] = {X10, Y10, 0.0};
        if (outer_ge(R10, X10)) {
            if (spline_zstart(outer * 0.999999, P0, D, ap, &zc) == 0) z = zc;
            return z;
        }
        if (between(R10, X10)) return 0.0;
        if (inner_le(R10, X10)) {
            if (spline_zstart(inner / 0.999999, P0, D, ap, &zc) == 0) z = zc;
            return z;
        }
    }
    if (P[2] < ZA && P[2] > 0.0 && D[2] < 0.0) {
        const double R1 = sqrt(P[0] * P[0] + P[1] * P[1]);
        if (outer_ge(R1, P[0])) {
            if (spline_zstart(outer * 0.999999, P, D, ap, &zc) == 0) z = zc;
            return z;
        }
        if (between(R1, P[0])) {
            double z1, dz;
            if (!splint(e->spl_x, e->spl_y, e->spl_y2, annular ? R1 : P[0], &z1, &dz)) {
                *err = 3;
                return 0.0;
            }
            if (z1 < P[2]) {
                if (outer_ge(R10, X10)) {
                    if (spline_zstart(outer * 0.999999, P, D, ap, &zc) == 0) z = zc;
                    return z;
                }
                return 0.0;
            }
            return P[2];
        }
        if (inner_le(R1, P[0])) {
            if (spline_zstart(inner / 0.999999, P, D, ap, &zc) == 0) z = zc;
            return z;
        }
    }
    if (P[2] < ZA && P[2] > 0.0 && D[2] > 0.0) {
        const double R1 = sqrt(P[0] * P[0] + P[1] * P[1]);
        if (outer_ge(R1, P[0])) {
            if (spline_zstart(outer * 0.999999, P, D, ap, &zc) == 0) z = zc;
            return z;
        }
        if (between(R1, P[0])) {
            double z1, dz;
            if (!splint(e->spl_x, e->spl_y, e->spl_y2, annular ? R1 : P[0], &z1, &dz)) {
                *err = 3;
                return 0.0;
            }
            if (z1 < P[2]) {
                if (outer_ge(R1A, X1A)) {
                    if (spline_zstart(outer * 0.999999, P, D, ap, &zc) == 0) z = zc;
                }
                return z;
            }
            if (between(R10, X10) || (annular ? R10 < outer : X10 < outer)) {
                if ((annular && R10 < outer) || (line && X10 < outer)) return 0.0;
            }
            if (outer_ge(R10, X10)) {
                const double PD[3] = {X10, Y10, 0.0};
                if (spline_zstart(outer * 0.999999, PD, D, ap, &zc) == 0) z = zc;
                return z;
            }
        }
        if (inner_le(R1, P[0])) {
            if (spline_zstart(outer * 0.999999, P, D, ap, &zc) == 0) z = zc;
            return z;
        }
    }
    return z;
}

// Intersect (intersect.cpp:140-1011): closed forms, or start plane + Newton.
int intersect(const Element *e, const double P[3], const double D[3], double out[3], double n[3], double *plen) {
    for (int i = 0; i < 3; ++i) out[i] = P[i];
    const char s = e->surface;
    if (e->surface_type == 2) return quadric_closed(e, P, D, out, n, plen);
    if ((e->surface_type == 1 || e->surface_type == 7) && (s == 's' || s == 'S')) return quadric_closed(e, P, D, out, n, plen);
    if (e->surface_type == 1 && (s == 'o' || s == 'O')) return quadric_closed(e, P, D, out, n, plen);
    if (s == 'p' || s == 'P') return quadric_closed(e, P, D, out, n, plen);
    if (e->surface_type == 10) return torus_closed(e, P, D, out, n, plen);

    int err = 0;
    double s0a = 0.0;
    if (e->z_aperture - P[2] != 0.0) s0a = (e->z_aperture - P[2]) / (D[2] + 0.00000000001);
    const double xa = P[0] + D[0] * s0a, ya = P[1] + D[1] * s0a;
    const bool za_inside = aperture_contains(e, xa, ya, true) == 1;

    double zstart = 0.0;
    const int st = e->surface_type;
    if (st != 3 && st != 4 && st != 9) {
        const double fxy = surface_z_at(P, e);
        if (P[2] <= 0.0 && D[2] > 0.0)
            zstart = 0.0;
        else if (P[2] <= fxy && D[2] > 0.0)
            zstart = 0.0;
        else if (P[2] <= fxy && D[2] < 0.0 && P[2] > e->z_aperture && za_inside)
            zstart = 0.0;
        else if (P[2] <= fxy && D[2] < 0.0)
            zstart = e->z_aperture;
        else if (P[2] > fxy && D[2] < 0.0)
            zstart = 0.0;
        else if (P[2] > fxy && D[2] > 0.0)
            zstart = e->z_aperture;
    }
    if (st == 9) {
        zstart = spline_start(e, P, D, &err);
        if (err) return err;
    }
    double s0 = 0.0;
    if (zstart - P[2] != 0.0) s0 = (zstart - P[2]) / (D[2] + 0.00000000001);
    const double x1 = P[0] + D[0] * s0, y1 = P[1] + D[1] * s0;
    double lo = -1e10, hi = 1e10;
    if (st == 9) {
        const double sa = (e->spl_x.front() - x1) / (D[0] + 0.00000000001);
        const double sb = (e->spl_x.back() - x1) / (D[0] + 0.00000000001);
        lo = fmin(sa, sb);
        hi = fmax(sa, sb);
    }
    double sj = 0.0, sj1 = 0.0;
    for (int it = 0; it < 20; ++it) {
        sj = sj1;
        out[0] = x1 + D[0] * sj;
        out[1] = y1 + D[1] * sj;
        out[2] = zstart + D[2] * sj;
        double F;
        if (surface_eval(out, e, &F, n) != 0) {
            *plen = s0 + sj;
            return 2;
        }
        const double dfd = dot3(n, D);
        if (fabs(F) <= 0.000001 * fabs(dfd)) {
            *plen = s0 + sj;
            return 0;
        }
        sj1 = sj - F / dfd;
        if (st == 9) {
            if ((F < 0 && D[2] > 0) || (F > 0 && D[2] < 0))
                lo = fmax(sj, lo);
            else if ((F < 0 && D[2] < 0) || (F > 0 && D[2] > 0))
                hi = fmin(sj, hi);
            if (sj1 < lo || sj1 > hi) sj1 = 0.5 * (lo + hi);
            if (hi <= lo) break;
        }
    }
    *plen = s0 + sj;
    return 1;
}

// DetermineElementIntersectionNew (determineelementintersectionnew.cpp:58-633)
// returns intercept flag; sets backside and flips the normal when hit from behind
bool element_hit(const Element *e, const double P[3], const double D[3], double out[3], double n[3], double *plen,
                 int *back) {
    *back = 0;
    const int err = intersect(e, P, D, out, n, plen);
    if (err > 0 || *plen < 0) {
        *plen = 0.0;
        return false;
    }
    const int in = aperture_contains(e, out[0], out[1], false);
    if (in != 1) return false;
    *back = (dot3(D, n) < 0) ? 0 : 1;
    if (*back) {
        n[0] = -n[0];
        n[1] = -n[1];
        n[2] = -n[2];
    }
    return true;
}

// ------------------------------------------------------------------------------------
// Random draws and error samplers (errors.cpp:60-226, surfacenormalerrors.cpp:58-167)
// ------------------------------------------------------------------------------------
struct RayRng {
    Minstd *seq = nullptr;  // reference stream (shared by all rays)
    uint32_t seed = 0;
    uint64_t sid = 0;  // per-ray stream id
    uint32_t k = 0;    // per-ray draw counter
    double u() { return seq ? seq->uniform() : philox_draw(seed, sid, k++); }
};

double table_intensity(const Sun &sun, double theta) {
    size_t i = 0;
    while (i < sun.ang.size() - 1 && sun.ang[i] < theta) i++;
    if (i == 0) return sun.inten[0];
    return sun.inten[i - 1] + (sun.inten[i] - sun.inten[i - 1]) * (theta - sun.ang[i - 1]) / (sun.ang[i] - sun.ang[i - 1]);
}

// Inverse CDF of p(theta) ~ theta * I(theta) on [0, MaxAngle] (mrad): trapezoid CDF on
// 4096 cells, then theta(u) tabulated at 8193 equally spaced probabilities; a sample
// interpolates linearly between two table entries.  (Per-ray stream only; the
// reference stream reproduces the reference's 2-D rejection sampling instead.)
constexpr int kCdfCells = 4096;
constexpr int kInvCells = 8192;
void build_sun_cdf(Sun &sun) {
    sun.cdf_theta.clear();
    sun.cdf.clear();
    if (sun.ang.size() < 3 || !(sun.max_angle > 0)) return;
    std::vector<double> th(kCdfCells + 1, 0.0), cdf(kCdfCells + 1, 0.0);
    const double dt = sun.max_angle / kCdfCells;
    double prev = 0.0;
    for (int j = 0; j <= kCdfCells; ++j) {
        th[j] = dt * j;
        const double pdf = th[j] * table_intensity(sun, th[j]);
        if (j > 0) cdf[j] = cdf[j - 1] + 0.5 * (prev + pdf) * dt;
        prev = pdf;
    }
    const double tot = cdf[kCdfCells];
    for (int j = 0; j <= kCdfCells; ++j) cdf[j] = tot > 0 ? cdf[j] / tot : 0.0;
    sun.cdf.assign(kInvCells + 1, 0.0);  // theta at u = j / kInvCells
    for (int j = 0; j <= kInvCells; ++j) {
        const double u = double(j) / kInvCells;
        int lo = 0, hi = kCdfCells;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (cdf[mid] <= u)
                lo = mid;
            else
                hi = mid;
        }
        const double f = (cdf[hi] > cdf[lo]) ? (u - cdf[lo]) / (cdf[hi] - cdf[lo]) : 0.0;
        sun.cdf[j] = th[lo] + f * (th[hi] - th[lo]);
    }
}
double sample_sun_table(const Sun &sun, double u) {
    if (sun.cdf.empty()) return 0.0;
    const double x = u * kInvCells;
    const int j = std::min(int(x), kInvCells - 1);
    const double f = x - j;
    return sun.cdf[j] + f * (sun.cdf[j + 1] - sun.cdf[j]);
}

// rotate (sin t cos p, sin t sin p, cos t) from the frame whose z axis is 'axis'
void perturb_about(const double axis[3], double theta, double phi, double out[3]) {
    double eul[3] = {0, 0, 0};
    if (axis[2] == 0.0) {
        if (axis[0] == 0.0) {
            eul[0] = 0.0;
            eul[1] = kPi / 2.0;
        } else {
            eul[0] = kPi / 2.0;
            eul[1] = atan2(axis[1], sqrt(axis[0] * axis[0] + axis[2] * axis[2]));
        }
    } else {
        eul[0] = atan2(axis[0], axis[2]);
        eul[1] = atan2(axis[1], sqrt(axis[0] * axis[0] + axis[2] * axis[2]));
    }
    double R[3][3], Rt[3][3];
    euler_matrices(eul, R, Rt);
    const double loc[3] = {sin(theta) * cos(phi), sin(theta) * sin(phi), cos(theta)};
    mat_vec(Rt, loc, out);
}

// Source 1 = sunshape, 2 = specularity.  Returns the perturbed direction.
void apply_errors(RayRng &rng, const double cin[3], int source, const Sun &sun, const Element *e, const Optics *op,
                  double cout[3], const double nrm[3]) {
    char dist = 'g';
    double delop = 0.0;
    if (source == 1) {
        dist = sun.shape;
        delop = sun.sigma / 1000.0;
    } else {
        dist = op->dist;
        delop = op->spec / 1000.0;
    }
    unsigned maxcall = 0;
    for (;;) {
        double theta = 0.0, theta2 = 0.0;
        if (rng.seq) {
            switch (dist) {
                case 'g':
                case 'G': {
                    const double tx = 0.0 + rng.seq->normal() * delop;
                    const double ty = 0.0 + rng.seq->normal() * delop;
                    theta2 = tx * tx + ty * ty;
                    break;
                }
                case 'p':
                case 'P': {
                    double tx, ty;
                    do {
                        tx = 2.0 * delop * rng.u() - delop;
                        ty = 2.0 * delop * rng.u() - delop;
                        theta2 = tx * tx + ty * ty;
                    } while (theta2 > delop * delop);
                    break;
                }
                case 'd':
                case 'D': {
                    for (;;) {
                        const double tx = 2.0 * sun.max_angle * rng.u() - sun.max_angle;
                        const double ty = 2.0 * sun.max_angle * rng.u() - sun.max_angle;
                        theta2 = tx * tx + ty * ty;
                        const double th = sqrt(theta2);
                        const double stest = table_intensity(sun, th);
                        if (rng.u() > stest / sun.max_intensity) continue;
                        if (theta2 > sun.max_angle * sun.max_angle) continue;
                        break;
                    }
                    theta2 = theta2 / 1000000.0;
                    break;
                }
                case 'f':
                case 'F':
                    theta2 = pow(asin(sqrt(rng.u())), 2);
                    break;
                default:
                    break;
            }
            theta = sqrt(theta2);
        } else {
            const double ut = rng.u();
            switch (dist) {
                case 'g':
                case 'G':
                    theta = delop * sqrt(-2.0 * log(1.0 - ut));
                    break;
                case 'p':
                case 'P':
                    theta = delop * sqrt(ut);
                    break;
                case 'd':
                case 'D':
                    theta = sample_sun_table(sun, ut) / 1000.0;
                    break;
                case 'f':
                case 'F':
                    theta = asin(sqrt(ut));
                    break;
                default:
                    theta = 0.0;
            }
        }
        const double phi = rng.u() * 2.0 * 3.1415926535897932385;
        perturb_about(cin, theta, phi, cout);
        if (source == 2 && e->interaction == 2 && dot3(cout, nrm) < 0 && maxcall++ < 50000) continue;
        break;
    }
}

void slope_errors(RayRng &rng, const double nin[3], const Optics *op, double nout[3]) {
    const char dist = op->dist;
    const double delop = op->slope / 1000.0;
    double theta = 0.0;
    if (rng.seq) {
        double theta2 = 0.0;
        if (dist == 'g' || dist == 'G') {
            const double tx = 0.0 + rng.seq->normal() * delop;
            const double ty = 0.0 + rng.seq->normal() * delop;
            theta2 = tx * tx + ty * ty;
        } else if (dist == 'p' || dist == 'P') {
            double tx, ty;
            do {
                tx = 2.0 * delop * rng.u() - delop;
                ty = 2.0 * delop * rng.u() - delop;
                theta2 = tx * tx + ty * ty;
            } while (theta2 > delop * delop);
        }
        theta = sqrt(theta2);
    } else {
        const double ut = rng.u();
        if (dist == 'g' || dist == 'G')
            theta = delop * sqrt(-2.0 * log(1.0 - ut));
        else if (dist == 'p' || dist == 'P')
            theta = delop * sqrt(ut);
    }
    const double phi = rng.u() * 2.0 * 3.1415926535897932385;
    perturb_about(nin, theta, phi, nout);
}

// Interaction types 1 (refraction with unpolarised Fresnel split) and 2 (reflection)
// (interaction.cpp:58-199).  Returns false if the refraction Newton failed (the
// reference then leaves the outgoing direction unchanged).
bool interact(RayRng &rng, const double cin[3], const double n[3], int type, const Optics *op, double cout[3]) {
    if (type == 1) {
        const double r1 = op->rindex[0], r2 = op->rindex[2];
        const double mu = r1 / r2;
        const double d2 = dot3(n, n);
        const double B = (mu * mu - 1.0) / d2;
        double A = mu * dot3(cin, n) / d2;
        if (B > A * A) {
            const double a = dot3(cin, n) / dot3(n, n);
            for (int i = 0; i < 3; ++i) cout[i] = cin[i] - 2.0 * a * n[i];
            return true;
        }
        const double un[3] = {-n[0] / sqrt(dot3(n, n)), -n[1] / sqrt(dot3(n, n)), -n[2] / sqrt(dot3(n, n))};
        const double ia = acos(dot3(cin, un));
        const double st = r1 * sin(ia) / r2;
        const double ct = sqrt(1 - st * st);
        const double rs_n = r1 * cos(ia) - r2 * ct, rs_d = r1 * cos(ia) + r2 * ct;
        const double rs = (rs_n / rs_d) * (rs_n / rs_d);
        const double rp_n = r1 * ct - r2 * cos(ia), rp_d = r1 * ct + r2 * cos(ia);
        const double rp = (rp_n / rp_d) * (rp_n / rp_d);
        const double rave = (rp + rs) / 2.0;
        if (rave < rng.u()) {
            double g = -B / (2.0 * A), g1 = 0.0;
            bool ok = false;
            for (int i = 1; i < 10; ++i) {
                g1 = (g * g - B) / (2.0 * (g + A));
                if (fabs(g - g1) < 0.000005) {
                    ok = true;
                    break;
                }
                g = g1;
            }
            if (!ok) return false;
            for (int i = 0; i < 3; ++i) cout[i] = mu * cin[i] + g1 * n[i];
        } else {
            const double a = dot3(cin, n) / dot3(n, n);
            for (int i = 0; i < 3; ++i) cout[i] = cin[i] - 2.0 * a * n[i];
        }
        return true;
    }
    const double a = dot3(cin, n) / dot3(n, n);
    for (int i = 0; i < 3; ++i) cout[i] = cin[i] - 2.0 * a * n[i];
    return true;
}

// ------------------------------------------------------------------------------------
// Setup: surface parameters, aperture plane, geometry init, sun box
// ------------------------------------------------------------------------------------
bool translate_surface(Context *cx, Element *e, const double p[8]) {  // input.cpp:288-366
    switch (e->surface) {
        case 's':
        case 'S':
            e->vcx = p[0];
            e->vcy = (e->shape == 'l' || e->shape == 'L') ? 0.0 : e->vcx;
            e->kappa = 1.0;
            e->surface_type = (e->vcy == 0.0) ? 7 : 1;
            return true;
        case 'p':
        case 'P':
            e->vcx = p[0];
            e->vcy = p[1];
            e->kappa = 0.0;
            e->surface_type = (e->vcy == 0.0) ? 7 : 1;
            return true;
        case 'o':
        case 'O':
            e->vcx = p[0];
            e->vcy = p[0];
            e->kappa = p[1];
            e->surface_type = (e->vcy == 0.0) ? 7 : 1;
            return true;
        case 'g':
        case 'G':
            e->vcx = p[0];
            e->vcy = p[1];
            e->kappa = p[2];
            for (int i = 0; i < 5; ++i) e->alpha[i] = p[3 + i];
            e->surface_type = (e->vcy == 0.0) ? 7 : 1;
            return true;
        case 'f':
        case 'F':
            e->alpha[0] = 0;
            e->alpha[1] = 0;
            e->alpha[2] = 1;
            e->alpha[3] = 0;
            e->alpha[4] = 0;
            e->surface_type = 3;
            return true;
        case 'c':
        case 'C':
            e->cone_half_angle = p[0];
            e->surface_type = 1;
            return true;
        case 't':
        case 'T':
            if ((e->shape != 'l' && e->shape != 'L') || e->p[0] != 0.0 || e->p[1] != 0.0) {
                cx->log("Bad aperture or parameters of element not consistent with cylindrical surface\n");
                return false;
            }
            e->curv_rev = p[0];
            e->vcx = e->curv_rev;
            e->surface_type = 2;
            return true;
        case 'd':
        case 'D':
            if ((e->shape != 'a' && e->shape != 'A') || e->p[0] != 0.0 || e->p[1] != 0.0) {
                cx->log("Bad aperture or parameters of element not consistent with toroidal surface\n");
                return false;
            }
            e->annular_r = p[0];
            e->cross_r = p[1];
            e->surface_type = 10;
            return true;
        default:
            cx->log("invalid surface index: %c\n", e->surface);
            return false;
    }
}

void aperture_plane(Element *e) {  // apertureplane.cpp:57-491
    auto sq = [](double v) { return v * v; };
    double maxr = 0.0;
    if (e->shape == 'i' || e->shape == 'I' || e->shape == 'q' || e->shape == 'Q') {
        maxr = sqrt(sq(e->p[0]) + sq(e->p[1]));
        maxr = fmax(maxr, sqrt(sq(e->p[2]) + sq(e->p[3])));
        maxr = fmax(maxr, sqrt(sq(e->p[4]) + sq(e->p[5])));
        if (e->shape == 'q' || e->shape == 'Q') maxr = fmax(maxr, sqrt(sq(e->p[6]) + sq(e->p[7])));
    }
    const char sh = (char)tolower(e->shape);
    // radius^2 used by each aperture family
    auto rad2 = [&](int &kind) -> double {
        kind = 0;
        switch (sh) {
            case 'c':
            case 'h':
            case 't':
                kind = 1;
                return sq(e->p[0] / 2.0);
            case 'r':
                kind = 2;
                return sq(e->p[0] / 2.0) + sq(e->p[1] / 2.0);
            case 'a':
            case 'l':
                kind = 3;
                return (fabs(e->p[1]) >= fabs(e->p[0])) ? sq(e->p[1]) : sq(e->p[0]);
            case 'i':
            case 'q':
                kind = 4;
                return sq(maxr);
        }
        return 0.0;
    };
    int kind;
    switch (tolower(e->surface)) {
        case 'g': {
            const double r2 = rad2(kind);
            if (!kind) break;
            double sum = 0.0;
            if (kind == 1) {
                double rho2i = 1.0;
                for (int i = 0; i < 5; ++i) {
                    rho2i = rho2i * r2;
                    sum += e->alpha[i] * rho2i;
                }
            } else if (kind == 2 || kind == 3) {
                for (int i = 0; i < 5; ++i) sum += e->alpha[i] * pow(r2, (int)(i + 1));
            }
            if (kind == 1)  // apertureplane.cpp:130 spells the product without sqr()
                e->z_aperture = e->vcx * r2 / (1 + sqrt(1 - e->kappa * e->vcx * e->vcx * r2)) + sum;
            else
                e->z_aperture = e->vcx * r2 / (1 + sqrt(1 - e->kappa * sq(e->vcx) * r2)) + sum;
            break;
        }
        case 's': {
            const double f = 1.0 / (2.0 * e->vcx);
            const double r2 = rad2(kind);
            if (!kind) break;
            e->z_aperture = 2.0 * f - sqrt(sq(2.0 * f) - r2);
            break;
        }
        case 'p':
        case 'm': {
            double f;
            if (tolower(e->surface) == 'p') {
                f = 1.0 / (2.0 * e->vcx);
            } else {
                if (e->fit_order < 2) return;
                f = (1.0 / (4.0 * bco(e, 2, 0)) + 1.0 / (4.0 * bco(e, 2, 2))) / 2.0;
            }
            const double r2 = rad2(kind);
            if (!kind) break;
            e->z_aperture = r2 / (4.0 * f);
            break;
        }
        case 'f':
            e->z_aperture = 0.0;
            break;
        case 'o': {
            const double r2 = rad2(kind);
            if (!kind) break;
            e->z_aperture = (1 - sqrt(1 - e->kappa * sq(e->vcx) * r2)) / (e->kappa * e->vcx);
            break;
        }
        case 'c': {
            const double t = tan(e->cone_half_angle * kDegToRad);
            if (sh == 'c' || sh == 'h' || sh == 't')
                e->z_aperture = e->p[0] / (2.0 * t);
            else if (sh == 'r')
                e->z_aperture = sqrt(sq(e->p[0] / 2.0) + sq(e->p[1] / 2.0)) / (2.0 * t);
            else if (sh == 'a')
                e->z_aperture = e->p[1] / t;
            else if (sh == 'i' || sh == 'q')
                e->z_aperture = sqrt(sq(maxr)) / (2.0 * t);
            break;
        }
        case 't':
            e->z_aperture = 2.0 / e->curv_rev;
            break;
        case 'd':
            e->z_aperture = 2.0 * e->cross_r;
            break;
        case 'r': {
            const double r2 = rad2(kind);
            if (!kind) break;
            const double r = (kind == 1) ? e->p[0] / 2.0 : sqrt(r2);
            e->z_aperture = eval_poly(r, 0, e->poly, e->fit_order);
            break;
        }
        case 'i':
            e->z_aperture = e->spl_y.back();
            break;
        case 'v': {
            double lastz = 0.0;
            for (int i = 0; i < e->vshot_rows; ++i) {
                const double zm = eval_mono(e, e->vshot[5 * i], e->vshot[5 * i + 1]);
                if (zm > lastz) lastz = zm;
            }
            e->z_aperture = lastz;
            break;
        }
        case 'e': {  // apertureplane.cpp:455-468 scans the nodes' second coordinate
            double lastz = 0.0;
            for (size_t i = 0; i + 2 < e->fe_nodes.size(); i += 3)
                if (e->fe_nodes[i + 1] > lastz) lastz = e->fe_nodes[i + 1];
            e->z_aperture = lastz;
            break;
        }
        default:
            break;
    }
}

bool check_inputs(Context *cx) {  // input.cpp:87-150
    for (size_t i = 0; i < cx->stages.size(); ++i)
        for (size_t j = 0; j < cx->stages[i]->elements.size(); ++j) {
            const Element *e = cx->stages[i]->elements[j];
            const bool pp = e->surface == 'p' || e->surface == 'P';
            const bool ss = e->surface == 's' || e->surface == 'S';
            const bool line = e->shape == 'l' || e->shape == 'L';
            if (pp && line && e->vcy != 0.0) {
                cx->log("Parabolic surface combined with single axis curvature section aperture must have Cy = 0.  Element %d Stage %d.",
                        int(j + 1), int(i + 1));
                return false;
            }
            if (ss) {
                if (e->vcx == 0.0) {
                    cx->log("Spherical surface must have a curvature greater than 0.0.  Consider using a flat surface instead. Element %d, Stage %d.",
                            int(j + 1), int(i + 1));
                    return false;
                }
                if (e->vcy != 0.0 && e->vcy != e->vcx) {
                    cx->log("Spherical surface must have Cy=0 or Cy=Cx.  Currently, Cy=%lg for Element %d, Stage %d", e->vcy,
                            int(j + 1), int(i + 1));
                    return false;
                }
            }
            if ((e->surface == 'o' || e->surface == 'O') && (e->kappa == 1.0 || e->kappa == 0.0)) {
                cx->log("Kappa = 0.0 or 1.0 defines either a parabola or a sphere.  Use the specific surface definition for either of those cases. Element %d, Stage %d.",
                        int(j + 1), int(i + 1));
                return false;
            }
        }
    return true;
}

bool init_geometries(Context *cx) {  // input.cpp:153-286
    for (size_t i = 0; i < cx->stages.size(); ++i) {
        Stage *st = cx->stages[i];
        if (!aim_euler(st->origin, st->aim, st->zrot, st->euler)) {
            cx->log("Stage %d geometry as defined not possible.\n", int(i));
            return false;
        }
        euler_matrices(st->euler, st->r_to_loc, st->r_to_ref);
        for (size_t j = 0; j < st->elements.size(); ++j) {
            Element *e = st->elements[j];
            if (!aim_euler(e->origin, e->aim, e->zrot, e->euler)) {
                cx->log("Stage %d element %d geometry as defined not possible.\n", int(i), int(j));
                return false;
            }
            euler_matrices(e->euler, e->r_to_loc, e->r_to_ref);
            auto sq = [](double v) { return v * v; };
            const double *p = e->p;
            switch (e->shape) {
                case 'c':
                case 'C':
                    e->aperture_area = kPi * sq(p[0] / 2);
                    break;
                case 'h':
                case 'H':
                    e->aperture_area = 5.0 * sq(p[0] / 2.0) * cos(30.0 * kDegToRad) * sin(30.0 * kDegToRad);
                    break;
                case 'r':
                case 'R':
                    e->aperture_area = p[0] * p[1];
                    break;
                case 't':
                case 'T':
                    e->aperture_area = 0.25 * sq(p[0] * cos(30.0 * kDegToRad)) * sqrt(3.0);
                    break;
                case 'a':
                case 'A':
                    e->aperture_area = p[2] * kDegToRad * (p[1] - p[0]);
                    break;
                case 'l':
                case 'L':
                    e->aperture_area = (p[1] - p[0]) * p[2];
                    break;
                case 'i':
                case 'I': {
                    const double v11 = p[0] - p[2], v12 = p[1] - p[3], v21 = p[4] - p[2], v22 = p[5] - p[3];
                    const double v1m = sqrt(v11 * v11 + v12 * v12), v2m = sqrt(v21 * v21 + v22 * v22);
                    e->aperture_area = 0.5 * v1m * v2m * sin(acos((v11 * v21 + v12 * v22) / (v1m * v2m)));
                    break;
                }
                case 'q':
                case 'Q': {
                    const double v11 = p[0] - p[2], v12 = p[1] - p[3], v21 = p[4] - p[2], v22 = p[5] - p[3];
                    const double v31 = p[4] - p[6], v32 = p[5] - p[7], v41 = p[0] - p[6], v42 = p[1] - p[7];
                    const double v1m = sqrt(v11 * v11 + v12 * v12), v2m = sqrt(v21 * v21 + v22 * v22);
                    const double v3m = sqrt(v31 * v31 + v32 * v32), v4m = sqrt(v41 * v41 + v42 * v42);
                    const double t1 = acos((v11 * v21 + v12 * v22) / (v1m * v2m));
                    const double t2 = acos((v31 * v41 + v32 * v42) / (v3m * v4m));
                    e->aperture_area = 0.5 * (v1m * v2m * sin(t1) + v3m * v4m * sin(t2));
                    break;
                }
                default:
                    cx->log("invalid shape '%c' for aperture, element %d\n", e->shape, int(j));
                    return false;
            }
            if (!st->virt) {
                OpticSet *set = nullptr;
                for (auto *o : cx->optics)
                    if (strcasecmp(o->name.c_str(), e->optic_name.c_str()) == 0) set = o;
                if (!set) {
                    cx->log("Stage %d element %d invalid optical property set name: '%s'\n", int(i), int(j),
                            e->optic_name.c_str());
                    return false;
                }
                e->optics = set;
                set->front.rindex[2] = set->back.rindex[0];
                set->front.rindex[3] = set->back.rindex[1];
                set->back.rindex[2] = set->front.rindex[0];
                set->back.rindex[3] = set->front.rindex[1];
            } else {
                e->optics = nullptr;
            }
            aperture_plane(e);
        }
    }
    return check_inputs(cx);
}

// SunToPrimaryStage (suntoprimarystage.cpp:59-293): sun frame, sun box, projected centres
bool sun_to_primary(Context *cx, Stage *st, double pos_sun_stage[3], std::vector<double> &proj) {
    Sun &sun = cx->sun;
    double dx = 0.0 - sun.origin[0], dy = 0.0 - sun.origin[1], dz = 0.0 - sun.origin[2];
    const double dt = sqrt(dx * dx + dy * dy + dz * dz);
    if (dt == 0.0) {
        cx->log("error calculating sun position in primary stage, dtot = 0.0\n");
        return false;
    }
    const double cg[3] = {dx / dt, dy / dt, dz / dt};
    double cs[3];
    to_local(st->origin, cg, st->origin, st->r_to_loc, pos_sun_stage, cs);
    sun.euler[0] = atan2(cs[0], cs[2]);
    sun.euler[1] = asin(cs[1]);
    sun.euler[2] = 0.0;
    double R[3][3];
    euler_matrices(sun.euler, R, sun.r_to_ref);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) sun.r_to_loc[i][j] = R[i][j];
    sun.xmax = -1.0e20;
    sun.xmin = 1.0e20;
    sun.ymax = -1.0e20;
    sun.ymin = 1.0e20;
    const double zero[3] = {0, 0, 0}, cdum[3] = {0, 0, 1};
    proj.assign(3 * st->elements.size(), 0.0);
    size_t n = 0;
    for (size_t i = 0; i < st->elements.size(); ++i) {
        const Element *e = st->elements[i];
        if (!e->enabled) continue;
        double pl[3], cl[3];
        to_local(e->origin, cdum, zero, R, pl, cl);
        proj[3 * i] = pl[0];
        proj[3 * i + 1] = pl[1];
        proj[3 * i + 2] = pl[2];
        double ext = 0.0;
        const double *p = e->p;
        switch (e->shape) {
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
                m = fmax(m, sqrt(p[2] * p[2] + p[3] * p[3]));
                m = fmax(m, sqrt(p[4] * p[4] + p[5] * p[5]));
                if (e->shape == 'q' || e->shape == 'Q') m = fmax(m, sqrt(p[6] * p[6] + p[7] * p[7]));
                ext = m;
                break;
            }
            default:
                ext = 0.0;
        }
        const double x0 = pl[0] - ext, x1 = pl[0] + ext, y0 = pl[1] - ext, y1 = pl[1] + ext;
        if (x0 < sun.xmin) sun.xmin = x0;
        if (x1 > sun.xmax) sun.xmax = x1;
        if (y0 < sun.ymin) sun.ymin = y0;
        if (y1 > sun.ymax) sun.ymax = y1;
        n++;
    }
    if (n == 0) cx->log("error calculating sun position in primary stage because no elements were enabled");
    return n > 0;
}

// ------------------------------------------------------------------------------------
// The trace (raytrace.cpp:137-1113), restated per ray and per stage.
// ------------------------------------------------------------------------------------
struct InRay {
    double pos[3], cos[3];
    unsigned num;
    uint64_t sid;
    uint32_t k;
};

enum Fate { kMissFirst, kAbsorbed, kExited };

struct TraceState {
    Context *cx;
    Minstd *seq;
    uint32_t seed;
    bool sunshape, errors;
    double prev_out[3];
};

double optic_test_value(const Optics *op, int type, const double cin[3], const double n[3]) {
    const bool use_table = (type == 1) ? op->use_trans_table : op->use_refl_table;
    if (!use_table) return (type == 1) ? op->trans : op->refl;
    const std::vector<double> &ang = (type == 1) ? op->trans_ang : op->refl_ang;
    const std::vector<double> &val = (type == 1) ? op->trans_val : op->refl_val;
    const double nn = sqrt(dot3(n, n));
    const double un[3] = {-n[0] / nn, -n[1] / nn, -n[2] / nn};
    const double ia = acos(dot3(cin, un)) * 1000.;
    const size_t np = ang.size();
    if (ia >= ang[np - 1]) return val[np - 1];
    size_t m = 0;
    while (ang[m] < ia) m++;
    if (m == 0) return val[0];
    return (val[m] + val[m - 1]) / 2.0;
}

// Trace one ray through stage index si; appends records; returns its fate and, for
// kExited, the outgoing global ray.
Fate trace_in_stage(TraceState &ts, Stage *st, int si, double pg[3], double cg[3], unsigned raynum, RayRng &rng,
                    std::vector<Record> &recs) {
    Context *cx = ts.cx;
    double ps[3], cs[3];
    to_local(pg, cg, st->origin, st->r_to_loc, ps, cs);
    int hits = 0;
    for (;;) {
        double best = 1e99;
        int best_j = -1, best_back = 0;
        double bpos_e[3], bcos_e[3], bn[3], bpos_s[3], bcos_s[3];
        for (size_t j = 0; j < st->elements.size(); ++j) {
            const Element *e = st->elements[j];
            if (!e->enabled) continue;
            double pe[3], ce[3];
            to_local(ps, cs, e->origin, e->r_to_loc, pe, ce);
            pe[0] = pe[0] + 1.0e-5 * ce[0];
            pe[1] = pe[1] + 1.0e-5 * ce[1];
            pe[2] = pe[2] + 1.0e-5 * ce[2];
            double out[3], n[3], pl;
            int back;
            if (!element_hit(e, pe, ce, out, n, &pl, &back)) continue;
            if (pl < best) {
                const char sf = e->surface;
                if (out[2] <= e->z_aperture || sf == 'm' || sf == 'M' || sf == 'r' || sf == 'R') {
                    best = pl;
                    best_j = int(j);
                    best_back = back;
                    for (int q = 0; q < 3; ++q) {
                        bpos_e[q] = out[q];
                        bcos_e[q] = ce[q];
                        bn[q] = n[q];
                    }
                    to_ref(out, ce, e->origin, e->r_to_ref, bpos_s, bcos_s);
                }
            }
        }
        if (best_j < 0) return hits == 0 ? kMissFirst : kExited;

        const Element *e = st->elements[best_j];
        Record r;
        for (int q = 0; q < 3; ++q) {
            r.pos[q] = bpos_s[q];
            r.cos[q] = bcos_s[q];
            r.loc[q] = bpos_e[q];
        }
        r.element = best_j + 1;
        r.stage = si + 1;
        r.raynum = raynum;
        recs.push_back(r);
        hits++;

        double pout[3], cout[3];
        if (st->virt) {
            for (int q = 0; q < 3; ++q) {
                pout[q] = bpos_e[q];
                cout[q] = bcos_e[q];
            }
        } else {
            const Optics *op = best_back ? &e->optics->back : &e->optics->front;
            if (e->interaction != 1 && e->interaction != 2) {
                cx->log("Bad optical interaction type = %d (stage %d)", si, e->interaction);
                throw 1;
            }
            const double tv = optic_test_value(op, e->interaction, bcos_e, bn);
            if (tv <= rng.u()) {
                recs.back().element = -recs.back().element;
                return kAbsorbed;
            }
            if (ts.sunshape && si == 0 && hits == 1) {
                double c2[3];
                apply_errors(rng, bcos_e, 1, cx->sun, e, op, c2, bn);
                for (int q = 0; q < 3; ++q) bcos_e[q] = c2[q];
            }
            if (ts.errors) {
                double n2[3];
                slope_errors(rng, bn, op, n2);
                for (int q = 0; q < 3; ++q) bn[q] = n2[q];
            }
            for (int q = 0; q < 3; ++q) pout[q] = bpos_e[q];
            // A failed refraction Newton (interaction.cpp:167-169) leaves the outgoing
            // direction untouched: with the reference stream that is the run-wide
            // CosRayOutElement of whichever ray set it last (raytrace.cpp:171); with the
            // per-ray stream the ray keeps its incoming direction, as on the GPU.
            double co[3];
            for (int q = 0; q < 3; ++q) co[q] = ts.seq ? ts.prev_out[q] : bcos_e[q];
            interact(rng, bcos_e, bn, e->interaction, op, co);
            for (int q = 0; q < 3; ++q) cout[q] = co[q];
            if (ts.errors) {
                double axis[3];
                const bool diffuse = (op->dist == 'F' || op->dist == 'f');
                for (int q = 0; q < 3; ++q) axis[q] = diffuse ? bn[q] : cout[q];
                double c3[3];
                apply_errors(rng, axis, 2, cx->sun, e, op, c3, bn);
                for (int q = 0; q < 3; ++q) cout[q] = c3[q];
            }
        }
        for (int q = 0; q < 3; ++q) ts.prev_out[q] = cout[q];
        to_ref(pout, cout, e->origin, e->r_to_ref, ps, cs);
        to_ref(ps, cs, st->origin, st->r_to_ref, pg, cg);
        if (!st->multihit) return kExited;
    }
}

// Reference record order after TRayData::Merge of every stage (types.cpp:311-355):
// full 8192-record blocks first, partial blocks appended in turn.
void merge_records(Context *cx) {
    const size_t B = 8192;
    struct Blk {
        std::vector<const Record *> r;
    };
    std::vector<Blk> all;
    for (auto &sr : cx->stage_records) {
        std::vector<Blk> src;
        for (size_t i = 0; i < sr.size(); i += B) {
            Blk b;
            for (size_t j = i; j < std::min(sr.size(), i + B); ++j) b.r.push_back(&sr[j]);
            src.push_back(b);
        }
        std::vector<Blk> full, partial;
        for (auto &b : all) (b.r.size() == B ? full : partial).push_back(b);
        for (auto &b : src) (b.r.size() == B ? full : partial).push_back(b);
        all = full;
        for (auto &b : partial)
            for (auto *r : b.r) {
                if (all.empty() || all.back().r.size() == B) all.push_back(Blk());
                all.back().r.push_back(r);
            }
    }
    cx->all.clear();
    for (auto &b : all)
        for (auto *r : b.r) cx->all.push_back(*r);
}

int run_trace(Context *cx, unsigned seed) {
    cx->all.clear();
    g_fe_failed = false;
    cx->stage_records.assign(cx->stages.size(), {});
    if (!init_geometries(cx)) return -1;
    const bool explicit_rays = !cx->explicit_pos.empty();
    const st_uint_t N = explicit_rays ? ~0ul : (st_uint_t)cx->raycount;
    const st_uint_t maxr = (st_uint_t)cx->raymax;
    if (!explicit_rays && cx->raycount < 1) {
        cx->log("invalid number of rays: %d", cx->raycount);
        return -1;
    }
    if (cx->stages.empty()) {
        cx->log("no stages defined.");
        return -1;
    }
    Stage *s0 = cx->stages[0];
    double pos_sun_stage[3];
    std::vector<double> proj;
    if (!sun_to_primary(cx, s0, pos_sun_stage, proj)) return -1;
    build_sun_cdf(cx->sun);

    Minstd seq;
    seq.seed(seed);
    TraceState ts{cx, cx->rng_mode == 0 ? &seq : nullptr, seed, cx->err_sun, cx->err_opt, {0.0, 0.0, 0.0}};
    cx->sun_ray_count = 0;

    std::vector<InRay> carry;
    try {
        // ---- first stage: sun rays (or explicit rays) ----
        unsigned raynum = 1;
        bool carried_nonlast = false;
        const size_t nexp = cx->explicit_pos.size() / 3;
        uint64_t sid = 0;
        for (;;) {
            if (explicit_rays && sid >= nexp) break;
            RayRng rng;
            rng.seq = ts.seq;
            rng.seed = seed;
            rng.sid = sid;
            rng.k = 0;
            double pg[3], cg[3];
            if (explicit_rays) {
                for (int q = 0; q < 3; ++q) {
                    pg[q] = cx->explicit_pos[3 * sid + q];
                    cg[q] = cx->explicit_cos[3 * sid + q];
                }
            } else if (cx->sun.point_source) {  // generateray.cpp:101-133
                for (int q = 0; q < 3; ++q) pg[q] = cx->sun.origin[q];
                for (int q = 0; q < 3; ++q) {
                    const int sg = (rng.u() <= 0.5) ? -1 : 1;
                    cg[q] = sg * rng.u();
                }
                const double m = sqrt(cg[0] * cg[0] + cg[1] * cg[1] + cg[2] * cg[2]);
                for (int q = 0; q < 3; ++q) cg[q] = cg[q] / m;
            } else {  // generateray.cpp:142-159
                const Sun &sun = cx->sun;
                const double xs = sun.xmin + (sun.xmax - sun.xmin) * rng.u();
                const double ys = sun.ymin + (sun.ymax - sun.ymin) * rng.u();
                const double psun[3] = {xs, ys, -10000.0}, csun[3] = {0.0, 0.0, 1.0};
                double pst[3], cst[3];
                to_ref(psun, csun, pos_sun_stage, sun.r_to_ref, pst, cst);
                to_ref(pst, cst, s0->origin, s0->r_to_ref, pg, cg);
            }
            sid++;
            cx->sun_ray_count++;
            if (!explicit_rays && cx->sun_ray_count > maxr) {
                cx->log("generated sun rays reached maximum count: %d", cx->raymax);
                return -1;
            }
            const Fate f = trace_in_stage(ts, s0, 0, pg, cg, raynum, rng, cx->stage_records[0]);
            if (f == kMissFirst) continue;
            const bool last = (raynum == N);
            if (f == kExited) {
                InRay ir;
                for (int q = 0; q < 3; ++q) {
                    ir.pos[q] = pg[q];
                    ir.cos[q] = cg[q];
                }
                ir.num = raynum;
                ir.sid = rng.sid;
                ir.k = rng.k;
                carry.push_back(ir);
                if (!last) carried_nonlast = true;
            }
            if (last) break;
            raynum++;
        }
        if (explicit_rays) carried_nonlast = !carry.empty() && (carry.size() > 1 || carry.back().num != raynum - 1);
        // raytrace.cpp:786-797: the final ray's store does not mark the stage as having rays
        if (!carried_nonlast) carry.clear();

        // ---- later stages ----
        for (size_t si = 1; si < cx->stages.size(); ++si) {
            if (carry.empty()) break;
            Stage *st = cx->stages[si];
            std::vector<InRay> next;
            const unsigned last_num = carry.back().num;
            for (const InRay &in : carry) {
                RayRng rng;
                rng.seq = ts.seq;
                rng.seed = seed;
                rng.sid = in.sid;
                rng.k = in.k;
                double pg[3] = {in.pos[0], in.pos[1], in.pos[2]}, cg[3] = {in.cos[0], in.cos[1], in.cos[2]};
                const size_t before = cx->stage_records[si].size();
                const Fate f = trace_in_stage(ts, st, int(si), pg, cg, in.num, rng, cx->stage_records[si]);
                (void)before;
                if (f == kMissFirst) {
                    if (st->tracethrough) {
                        InRay o = in;
                        o.k = rng.k;
                        next.push_back(o);
                        if (in.num == last_num) continue;  // raytrace.cpp:810-811: no miss record
                    }
                    double ps[3], cs[3];
                    to_local(in.pos, in.cos, st->origin, st->r_to_loc, ps, cs);
                    Record r;
                    for (int q = 0; q < 3; ++q) {
                        r.pos[q] = ps[q];
                        r.cos[q] = cs[q];
                        r.loc[q] = 0.0;
                    }
                    r.element = 0;
                    r.stage = int(si) + 1;
                    r.raynum = in.num;
                    cx->stage_records[si].push_back(r);
                } else if (f == kExited) {
                    InRay o;
                    for (int q = 0; q < 3; ++q) {
                        o.pos[q] = pg[q];
                        o.cos[q] = cg[q];
                    }
                    o.num = in.num;
                    o.sid = in.sid;
                    o.k = rng.k;
                    next.push_back(o);
                }
            }
            carry.swap(next);
        }
    } catch (int) {
        return -1;
    }
    if (g_fe_failed) {
        g_fe_failed = false;
        cx->log("Interpolation failed to find nearby nodes to ray hit in FEA surface.");
        return -1;
    }
    merge_records(cx);
    return int(cx->all.size());
}

}  // namespace

// ======================================================================================
// C API (same surface as coretrace/stapi.h:68-176)
// ======================================================================================
#define CTX(p, r)                                   \
    Context *cx = reinterpret_cast<Context *>(p); \
    if (!cx) return r;
#define STG(i)                                                      \
    if ((i) >= cx->stages.size()) return -1;                        \
    Stage *st = cx->stages[i];
#define ELM(i)                                                      \
    if ((i) >= st->elements.size()) return -1;                      \
    Element *e = st->elements[i];

// message hook of the product's .stinput reader, when the tests compile it into the oracle
extern "C" void st_input_report(void *p, const char *msg) {
    Context *cx = reinterpret_cast<Context *>(p);
    if (cx) cx->log("%s", msg ? msg : "");
}

extern "C" {

void *st_create_context() { return new Context; }
int st_free_context(void *p) {
    CTX(p, -1);
    delete cx;
    return 1;
}
int st_num_messages(void *p) {
    CTX(p, -1);
    return int(cx->messages.size());
}
const char *st_message(void *p, st_uint_t i) {
    CTX(p, nullptr);
    return i < cx->messages.size() ? cx->messages[i].c_str() : nullptr;
}
void st_clear_messages(void *p) {
    Context *cx = reinterpret_cast<Context *>(p);
    if (cx) cx->messages.clear();
}
int st_num_optics(void *p) {
    CTX(p, -1);
    return int(cx->optics.size());
}
int st_add_optic(void *p, const char *name) {
    CTX(p, -1);
    cx->optics.push_back(new OpticSet);
    cx->optics.back()->name = name;
    return int(cx->optics.size()) - 1;
}
int st_delete_optic(void *p, st_uint_t i) {
    CTX(p, -1);
    if (i >= cx->optics.size()) return -1;
    delete cx->optics[i];
    cx->optics.erase(cx->optics.begin() + i);
    return 1;
}
int st_clear_optics(void *p) {
    CTX(p, -1);
    for (auto *o : cx->optics) delete o;
    cx->optics.clear();
    return 1;
}
int st_optic(void *p, st_uint_t idx, int fb, char dist, int optnum, int apgr, int order, double rreal, double rimag,
             double ref, double tra, double gratingab12[3], double rmsslope, double rmsspec, int userefltable,
             int refl_npoints, double *refl_angles, double *refls, int usetranstable, int trans_npoints,
             double *trans_angles, double *transs) {
    CTX(p, -1);
    if (idx >= cx->optics.size()) return -1;
    Optics *o = (fb == 2) ? &cx->optics[idx]->back : &cx->optics[idx]->front;
    o->dist = dist;
    o->optnum = optnum;
    o->apgr = apgr;
    o->order = order;
    o->rindex[0] = rreal;
    o->rindex[1] = rimag;
    o->refl = ref;
    o->trans = tra;
    for (int i = 0; i < 4; ++i) o->ab12[i] = gratingab12[i];
    o->slope = rmsslope;
    o->spec = rmsspec;
    if (userefltable && refl_npoints > 0 && refl_angles && refls) {
        o->use_refl_table = true;
        o->refl_ang.assign(refl_angles, refl_angles + refl_npoints);
        o->refl_val.assign(refls, refls + refl_npoints);
    }
    if (usetranstable && trans_npoints > 0 && trans_angles && transs) {
        o->use_trans_table = true;
        o->trans_ang.assign(trans_angles, trans_angles + trans_npoints);
        o->trans_val.assign(transs, transs + trans_npoints);
    }
    return 1;
}
int st_num_stages(void *p) {
    CTX(p, -1);
    return int(cx->stages.size());
}
int st_add_stage(void *p) {
    CTX(p, -1);
    cx->stages.push_back(new Stage);
    return int(cx->stages.size()) - 1;
}
int st_add_stages(void *p, st_uint_t n) {
    CTX(p, -1);
    for (st_uint_t i = 0; i < n; ++i) cx->stages.push_back(new Stage);
    return int(n);
}
int st_delete_stage(void *p, st_uint_t i) {
    CTX(p, -1);
    if (i >= cx->stages.size()) return -1;
    delete cx->stages[i];
    cx->stages.erase(cx->stages.begin() + i);
    return 1;
}
int st_clear_stages(void *p) {
    CTX(p, -1);
    for (auto *s : cx->stages) delete s;
    cx->stages.clear();
    return 1;
}
int st_stage_xyz(void *p, st_uint_t i, double x, double y, double z) {
    CTX(p, -1);
    STG(i);
    st->origin[0] = x;
    st->origin[1] = y;
    st->origin[2] = z;
    return 1;
}
int st_stage_aim(void *p, st_uint_t i, double x, double y, double z) {
    CTX(p, -1);
    STG(i);
    st->aim[0] = x;
    st->aim[1] = y;
    st->aim[2] = z;
    return 1;
}
int st_stage_zrot(void *p, st_uint_t i, double z) {
    CTX(p, -1);
    STG(i);
    st->zrot = z;
    return 1;
}
int st_stage_flags(void *p, st_uint_t i, int virt, int multihit, int tracethrough) {
    CTX(p, -1);
    STG(i);
    st->virt = virt != 0;
    st->multihit = multihit != 0;
    st->tracethrough = tracethrough != 0;
    return 1;
}
int st_num_elements(void *p, st_uint_t s) {
    CTX(p, -1);
    STG(s);
    return int(st->elements.size());
}
int st_add_element(void *p, st_uint_t s) {
    CTX(p, -1);
    STG(s);
    st->elements.push_back(new Element);
    return int(st->elements.size()) - 1;
}
int st_add_elements(void *p, st_uint_t s, st_uint_t n) {
    CTX(p, -1);
    if (n < 1) return -1;
    STG(s);
    for (st_uint_t i = 0; i < n; ++i) st->elements.push_back(new Element);
    return int(n);
}
int st_delete_element(void *p, st_uint_t s, st_uint_t i) {
    CTX(p, -1);
    STG(s);
    if (i >= st->elements.size()) return -1;
    delete st->elements[i];
    st->elements.erase(st->elements.begin() + i);
    return 1;
}
int st_clear_elements(void *p, st_uint_t s) {
    CTX(p, -1);
    STG(s);
    for (auto *e : st->elements) delete e;
    st->elements.clear();
    return 1;
}
int st_element_enabled(void *p, st_uint_t s, st_uint_t i, int en) {
    CTX(p, -1);
    STG(s);
    ELM(i);
    e->enabled = en != 0;
    return 1;
}
int st_element_xyz(void *p, st_uint_t s, st_uint_t i, double x, double y, double z) {
    CTX(p, -1);
    STG(s);
    ELM(i);
    e->origin[0] = x;
    e->origin[1] = y;
    e->origin[2] = z;
    return 1;
}
int st_element_aim(void *p, st_uint_t s, st_uint_t i, double x, double y, double z) {
    CTX(p, -1);
    STG(s);
    ELM(i);
    e->aim[0] = x;
    e->aim[1] = y;
    e->aim[2] = z;
    return 1;
}
int st_element_zrot(void *p, st_uint_t s, st_uint_t i, double z) {
    CTX(p, -1);
    STG(s);
    ELM(i);
    e->zrot = z;
    return 1;
}
int st_element_aperture(void *p, st_uint_t s, st_uint_t i, char ap) {
    CTX(p, -1);
    STG(s);
    ELM(i);
    e->shape = ap;
    return 1;
}
int st_element_aperture_params(void *p, st_uint_t s, st_uint_t i, double prm[8]) {
    CTX(p, -1);
    STG(s);
    ELM(i);
    for (int k = 0; k < 8; ++k) e->p[k] = prm[k];
    return 1;
}
int st_element_surface(void *p, st_uint_t s, st_uint_t i, char sf) {
    CTX(p, -1);
    STG(s);
    ELM(i);
    e->surface = sf;
    return 1;
}
int st_element_surface_params(void *p, st_uint_t s, st_uint_t i, double prm[8]) {
    CTX(p, -1);
    STG(s);
    ELM(i);
    return translate_surface(cx, e, prm) ? 1 : -1;
}
int st_element_interaction(void *p, st_uint_t s, st_uint_t i, int t) {
    CTX(p, -1);
    STG(s);
    ELM(i);
    e->interaction = t;
    return 1;
}
int st_element_optic(void *p, st_uint_t s, st_uint_t i, const char *name) {
    CTX(p, -1);
    STG(s);
    ELM(i);
    e->optic_name = name;
    return 1;
}

// surface files (input.cpp:368-573); the finite-element ".fed" surface is not restated
int st_element_surface_file(void *p, st_uint_t s, st_uint_t i, const char *file) {
    CTX(p, -1);
    STG(s);
    ELM(i);
    const char *dot = strrchr(file, '.');
    if (!dot) {
        cx->log("Could not determine surface file type: '%s'\n", file);
        return -1;
    }
    std::string ext(dot + 1);
    for (auto &c : ext) c = (char)tolower(c);
    FILE *fp = fopen(file, "r");
    if (!fp) {
        cx->log("Could not open surface file for read: %s\n", file);
        return -1;
    }
    char line[1024];
    auto rd = [&]() -> bool { return fgets(line, sizeof line, fp) != nullptr; };
    bool ok = true;
    if (ext == "mon") {
        rd();
        const int order = atoi(line);
        e->bcoef.assign((order + 1) * (order + 1), 0.0);
        e->fit_order = order;
        for (int k = 0; k <= order; ++k)
            for (int m = 0; m <= k; ++m) {
                rd();
                e->bcoef[k * (order + 1) + m] = atof(line);
            }
        e->surface = 'm';
        e->surface_type = 6;
    } else if (ext == "sht") {
        rd();
        rd();
        double vr, vf, vt;
        sscanf(line, "%lg %lg %lg", &vr, &vf, &vt);
        int idum, order = 0, np = 0;
        rd();
        sscanf(line, "%d %d %d", &idum, &order, &np);
        rd();
        e->fit_order = order;
        e->bcoef.assign((order + 1) * (order + 1), 0.0);
        for (int k = 0; k <= order; ++k)
            for (int m = 0; m <= k; ++m) {
                rd();
                e->bcoef[k * (order + 1) + m] = atof(line);
            }
        e->vshot.assign(5 * np, 0.0);
        e->vshot_rows = np;
        for (int k = 0; k < np; ++k) {
            rd();
            double *v = &e->vshot[5 * k];
            sscanf(line, "%lg %lg %lg %lg %lg", v, v + 1, v + 2, v + 3, v + 4);
        }
        e->surface = 'v';
        e->surface_type = 5;
    } else if (ext == "ply") {
        rd();
        const int order = atoi(line);
        e->poly.assign(order + 1, 0.0);
        for (int k = 0; k <= order; ++k) {
            rd();
            e->poly[k] = atof(line);
        }
        e->fit_order = order;
        e->surface = 'r';
        e->surface_type = 8;
    } else if (ext == "csi") {
        rd();
        const int np = atoi(line);
        e->spl_x.assign(np, 0.0);
        e->spl_y.assign(np, 0.0);
        for (int k = 0; k < np; ++k) {
            rd();
            sscanf(line, "%lg %lg", &e->spl_x[k], &e->spl_y[k]);
        }
        double x, y;
        rd();
        sscanf(line, "%lg %lg", &x, &y);
        spline_setup(e->spl_x, e->spl_y, x, y, e->spl_y2);
        if ((e->shape != 'a' && e->shape != 'A' && e->shape != 'l' && e->shape != 'L') || e->p[0] < e->spl_x[0] ||
            e->p[1] > e->spl_x.back()) {
            cx->log("Error: Element uses cubic spline interpolation:"
                    "\tMake sure aperture is type 'a' or 'l' and that "
                    "1st and 2nd parameters are not < and not > the "
                    "1st and last X values in file respectively.\n");
            ok = false;
        } else {
            e->surface = 'i';
            e->surface_type = 9;
        }
    } else if (ext == "fed") {  // input.cpp:510-561
        rd();  // name line
        rd();
        const int np = atoi(line);
        e->fe_nodes.assign(3 * size_t(np > 0 ? np : 0), 0.0);
        for (int k = 0; k < np; ++k) {
            rd();
            sscanf(line, "%lg %lg %lg", &e->fe_nodes[3 * k], &e->fe_nodes[3 * k + 1], &e->fe_nodes[3 * k + 2]);
        }
        if (np > 0) fe_build(e);
        e->surface = 'e';
        e->surface_type = 4;
    } else {
        cx->log("Surface file type extension unknown: '%s'\n", ext.c_str());
        ok = false;
    }
    fclose(fp);
    return ok ? 1 : -1;
}

int st_sun(void *p, int ps, char shape, double sigma) {
    CTX(p, -1);
    cx->sun.point_source = ps != 0;
    cx->sun.shape = shape;
    cx->sun.sigma = sigma;
    return 1;
}
int st_sun_xyz(void *p, double x, double y, double z) {
    CTX(p, -1);
    cx->sun.origin[0] = x;
    cx->sun.origin[1] = y;
    cx->sun.origin[2] = z;
    return 1;
}
// solar position from latitude, day of year and solar hour (stapi.cpp:500-527): the
// declination and hour angle give elevation and azimuth; returns the unit vector toward
// the sun with x west, y zenith, z north.  Same arithmetic order as the reference.
int st_sun_position(void *, double lat, double day, double hour, double *x, double *y, double *z) {
    const double decl = 180 / kPi * asin(0.39795 * cos(0.98563 * kPi / 180 * (day - 173)));
    const double ha = 15 * (hour - 12);
    const double el = 180 / kPi * asin(sin(decl * kPi / 180) * sin(lat * kPi / 180) +
                                       cos(decl * kPi / 180) * cos(ha * kPi / 180) * cos(lat * kPi / 180));
    double az = 180 / kPi * acos((sin(kPi / 180 * decl) * cos(kPi / 180 * lat) -
                                  cos(kPi / 180 * decl) * sin(kPi / 180 * lat) * cos(kPi / 180 * ha)) /
                                     cos(kPi / 180 * el) +
                                 0.0000000001);
    if (sin(ha * kPi / 180) > 0.0) az = 360 - az;
    if (x) *x = -sin(az * kPi / 180) * cos(el * kPi / 180);
    if (y) *y = sin(el * kPi / 180);
    if (z) *z = cos(az * kPi / 180) * cos(el * kPi / 180);
    return 1;
}
int st_sun_userdata(void *p, st_uint_t n, double angle[], double intensity[]) {
    CTX(p, -1);
    if (n <= 2) return -1;
    Sun &s = cx->sun;
    s.max_angle = 0;
    s.max_intensity = 0;
    s.ang.assign(2 * n - 1, 0.0);
    s.inten.assign(2 * n - 1, 0.0);
    for (st_uint_t i = 0; i < n; ++i) {
        s.ang[n + i - 1] = angle[i];
        s.inten[n + i - 1] = intensity[i];
        if (angle[i] > s.max_angle) s.max_angle = angle[i];
        if (intensity[i] > s.max_intensity) s.max_intensity = intensity[i];
    }
    for (st_uint_t i = 0; i < n - 1; ++i) {
        s.ang[i] = -angle[n - i - 1];
        s.inten[i] = intensity[n - i - 1];
    }
    return int(n);
}
int st_num_intersections(void *p) {
    CTX(p, -1);
    return int(cx->all.size());
}
int st_locations(void *p, double *x, double *y, double *z) {
    CTX(p, -1);
    for (size_t i = 0; i < cx->all.size(); ++i) {
        x[i] = cx->all[i].pos[0];
        y[i] = cx->all[i].pos[1];
        z[i] = cx->all[i].pos[2];
    }
    return 1;
}
int st_cosines(void *p, double *x, double *y, double *z) {
    CTX(p, -1);
    for (size_t i = 0; i < cx->all.size(); ++i) {
        x[i] = cx->all[i].cos[0];
        y[i] = cx->all[i].cos[1];
        z[i] = cx->all[i].cos[2];
    }
    return 1;
}
int st_elementmap(void *p, int *m) {
    CTX(p, -1);
    for (size_t i = 0; i < cx->all.size(); ++i) m[i] = cx->all[i].element;
    return 1;
}
int st_stagemap(void *p, int *m) {
    CTX(p, -1);
    for (size_t i = 0; i < cx->all.size(); ++i) m[i] = cx->all[i].stage;
    return 1;
}
int st_raynumbers(void *p, int *m) {
    CTX(p, -1);
    for (size_t i = 0; i < cx->all.size(); ++i) m[i] = int(cx->all[i].raynum);
    return 1;
}
int st_sun_stats(void *p, double *xmin, double *xmax, double *ymin, double *ymax, int *nsun) {
    CTX(p, -1);
    if (xmin) *xmin = cx->sun.xmin;
    if (xmax) *xmax = cx->sun.xmax;
    if (ymin) *ymin = cx->sun.ymin;
    if (ymax) *ymax = cx->sun.ymax;
    if (nsun) *nsun = int(cx->sun_ray_count);
    return 1;
}
int st_sim_params(void *p, int raycount, int maxcount, int dyn) {
    CTX(p, -1);
    cx->raycount = raycount;
    cx->raymax = maxcount;
    cx->dyn_group = dyn != 0;
    return 1;
}
int st_sim_errors(void *p, int sun, int opt) {
    CTX(p, -1);
    cx->err_sun = sun != 0;
    cx->err_opt = opt != 0;
    return 1;
}
int st_sim_run(void *p, unsigned seed, int (*)(st_uint_t, st_uint_t, st_uint_t, st_uint_t, st_uint_t, void *), void *) {
    CTX(p, -1);
    return run_trace(cx, seed);
}

// ---- oracle-only extras ----
int st_oracle_set_rng(void *p, int mode) {
    CTX(p, -1);
    cx->rng_mode = mode;
    return 1;
}
int st_oracle_explicit_rays(void *p, st_uint_t n, const double *pos, const double *cos) {
    CTX(p, -1);
    cx->explicit_pos.assign(pos, pos + 3 * n);
    cx->explicit_cos.assign(cos, cos + 3 * n);
    return int(n);
}
// kind 0: planar bins over element-local x in [x0,x1), y in [y0,y1);
// kind 1: cylinder bins, angle atan2(x, z - r) + pi over [0, 2 pi) x axial y in [y0, y1)
//          with r = x1 (the cylinder radius).  absorbed_only selects element == -target.
// GUI statistics binning (app/src/project.cpp:1367-1403): bin g is the smallest g >= -1
// with vmin + (g+1) b >= v, counted only when 0 <= g < n; a full cylinder unwraps x to
// the arc length R asin(x/R) on the front half, +-(pi R/2 + R acos(|x|/R)) behind it.
static int oracle_gui_bin(double v, double vmin, double b, int n) {
    if (!(v > vmin - b) || !(v <= vmin + (n + 1) * b)) return -1;
    int g = -1;
    while (g + 1 <= n && vmin + (g + 1) * b < v) g++;
    return (g >= 0 && g < n) ? g : -1;
}
static double oracle_gui_arc(double x, double z, double R) {
    if (z <= R) return R * asin(x / R);
    return (x < 0) ? -(kPi * R / 2.0 + R * acos(fabs(x) / R)) : kPi * R / 2.0 + R * acos(x / R);
}

// Kind 4, the trough example's nearest-node binning
// (app/deploy/api/examples/parabolic-trough-tracking-timeseries/st_processing_functions.py):
// create_polar_mesh_cyl (174-204) builds cell-centre nodes with numpy.arange -- for even n
// arange(d/2, S/2, d), for odd n arange(0, S/2, d), mirrored and sorted -- and
// compute_fluxmap (236-250) takes numpy.argmin(|nodes - v|), the first of equals.  The node
// list is built as numpy fills an arange (start, start + step, then start + k (v1 - start))
// and scanned whole.
static std::vector<double> oracle_mesh_nodes(int n, double span) {
    const double d = span / n;
    const double start = (n % 2 == 0) ? 0.0 + d / 2 : 0.0;
    const long len = (long)ceil((span / 2.0 - start) / d);
    std::vector<double> pos(size_t(len > 0 ? len : 0));
    for (long k = 0; k < len; ++k) pos[k] = k == 0 ? start : k == 1 ? start + d : start + double(k) * ((start + d) - start);
    std::vector<double> nodes;
    for (long k = len - 1; k >= (n % 2 == 0 ? 0 : 1); --k) nodes.push_back(-pos[k]);
    for (long k = 0; k < len; ++k) nodes.push_back(pos[k]);
    return nodes;
}
static int oracle_argmin_abs(const std::vector<double> &nodes, double v) {
    int best = -1;
    double bd = 0;
    for (size_t i = 0; i < nodes.size(); ++i) {
        const double dd = fabs(nodes[i] - v);
        if (dd != dd) return int(i);  // numpy.argmin returns the first NaN
        if (best < 0 || dd < bd) {
            best = int(i);
            bd = dd;
        }
    }
    return best;
}

// Bin (ix, iy) of an element-local point for a map kind; 1 when it lands in the map, 0 not.
int st_oracle_bin_point(int kind, int nx, int ny, double x0, double x1, double y0, double y1, double x, double y,
                        double z, int *ix_out, int *iy_out) {
    long ix = -1, iy = -1;
    if (kind == 4) {
        if (x != x || y != y || z != z) return 0;
        const double r = x1;
        ix = oracle_argmin_abs(oracle_mesh_nodes(nx, kPi * (2.0 * r)), r * atan2(x, z - r));
        iy = oracle_argmin_abs(oracle_mesh_nodes(ny, y1 - y0), y - 0.5 * (y0 + y1));
    } else if (kind >= 2) {
        ix = kind == 2 ? oracle_gui_bin(x, x0, (x1 - x0) / nx, nx)
                       : oracle_gui_bin(oracle_gui_arc(x, z, x1), -kPi * x1, 2.0 * kPi * x1 / nx, nx);
        iy = oracle_gui_bin(y, y0, (y1 - y0) / ny, ny);
    } else {
        double u, u0, u1;
        if (kind == 0) {
            u = x;
            u0 = x0;
            u1 = x1;
        } else {
            u = atan2(x, z - x1) + kPi;
            u0 = 0.0;
            u1 = 2.0 * kPi;
        }
        const double fx = floor((u - u0) / (u1 - u0) * nx), fy = floor((y - y0) / (y1 - y0) * ny);
        if (!(fx >= 0 && fx < nx && fy >= 0 && fy < ny)) return 0;
        ix = long(fx);
        iy = long(fy);
    }
    if (ix < 0 || ix >= nx || iy < 0 || iy >= ny) return 0;
    *ix_out = int(ix);
    *iy_out = int(iy);
    return 1;
}

int st_oracle_flux(void *p, int stage, int element, int kind, int nx, int ny, double x0, double x1, double y0,
                   double y1, int absorbed_only, unsigned long long *bins) {
    CTX(p, -1);
    for (const Record &r : cx->all) {
        if (r.stage != stage) continue;
        if (absorbed_only ? r.element != -element : (r.element != element && r.element != -element)) continue;
        if (kind == 4) {
            int ix, iy;
            if (st_oracle_bin_point(kind, nx, ny, x0, x1, y0, y1, r.loc[0], r.loc[1], r.loc[2], &ix, &iy))
                bins[size_t(iy) * nx + ix]++;
            continue;
        }
        if (kind >= 2) {
            const int ix = kind == 2 ? oracle_gui_bin(r.loc[0], x0, (x1 - x0) / nx, nx)
                                     : oracle_gui_bin(oracle_gui_arc(r.loc[0], r.loc[2], x1), -kPi * x1,
                                                      2.0 * kPi * x1 / nx, nx);
            const int iy = oracle_gui_bin(r.loc[1], y0, (y1 - y0) / ny, ny);
            if (ix >= 0 && iy >= 0) bins[size_t(iy) * nx + ix]++;
            continue;
        }
        double u, v, u0, u1;
        if (kind == 0) {
            u = r.loc[0];
            u0 = x0;
            u1 = x1;
        } else {
            u = atan2(r.loc[0], r.loc[2] - x1) + kPi;
            u0 = 0.0;
            u1 = 2.0 * kPi;
        }
        v = r.loc[1];
        const long ix = (long)floor((u - u0) / (u1 - u0) * nx);
        const long iy = (long)floor((v - y0) / (y1 - y0) * ny);
        if (ix < 0 || ix >= nx || iy < 0 || iy >= ny) continue;
        bins[iy * nx + ix]++;
    }
    return 1;
}
unsigned long st_oracle_sun_rays(void *p) {
    CTX(p, 0);
    return cx->sun_ray_count;
}

}  // extern "C"
