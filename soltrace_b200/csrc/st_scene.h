// Flattened scene tables as they sit in device memory, shared by the host
// set-up code (st_host.cpp) and the CUDA trace (st_trace.cu).
//
// Layout: one contiguous array of ElemRec for all stages (stage s owns
// [first_elem, first_elem + n_elem)), one array of OpticRec (front/back faces of
// every optical property set), plain double arrays for surface-file data and
// property tables, and the acceleration structures (sun-plane grid for the
// first stage's sun rays, one BVH per large stage).  Everything is read-only
// during a trace and small (about 400 B per element), so it stays L2-resident.
#pragma once
#include <cstdint>
#include <vector_types.h>

#ifdef __CUDACC__
#define ST_HD __host__ __device__
#else
#define ST_HD
#endif

namespace stb {

constexpr int kMaxStages = 16;
constexpr int kMaxFluxMaps = 8;
constexpr int kSunCdfCells = 4096;
constexpr int kSunInvCells = 8192;

// surface model codes after coretrace/input.cpp:288-366 translation
enum SurfType : int {
    kSurfConic = 1,      // conic of revolution / cone (g, s, p, o, c)
    kSurfCylinder = 2,   // 't'
    kSurfFlat = 3,       // 'f'
    kSurfFE = 4,         // 'e' finite-element data
    kSurfVshot = 5,      // 'v'
    kSurfZernike = 6,    // 'm'
    kSurfSingleAxis = 7, // conic with one curvature (Cy = 0)
    kSurfPoly = 8,       // 'r'
    kSurfSpline = 9,     // 'i'
    kSurfTorus = 10,     // 'd'
};

// Surfaces the element test intersects in closed form (flat, cylinder and the conics it
// solves directly); the others (torus, Newton-iterated surfaces) take its out-of-line path.
ST_HD inline bool closed_form_surface(int stype, int surf) {
    if (stype == kSurfFlat || stype == kSurfCylinder) return true;
    if (stype == kSurfTorus) return false;
    const int s = surf | 0x20;
    return (s == 'p') || (s == 's' && (stype == kSurfConic || stype == kSurfSingleAxis)) ||
           (s == 'o' && stype == kSurfConic);
}

struct ElemRec {
    double R[9];      // stage -> element rotation, row-major (RRefToLoc)
    double o[3];      // element origin in stage coordinates
    double ap[8];     // aperture parameters A..H
    double zap;       // ZAperture
    double kappa, vcx, vcy, curv_rev, cone_deg, ra, rs;
    double area;      // aperture area
    double bound_r;   // radius about the origin holding every accepted hit (<0: unbounded)
    int shape;        // aperture code (lower-case char)
    int surf;         // surface code as given (char, case preserved)
    int stype;        // SurfType
    int interaction;  // 1 refract, 2 reflect
    int opt_front, opt_back;  // OpticRec index, -1 on virtual stages
    int enabled;
    int data_off, data_n, fit_order;  // surface data in SceneDev::surf_data
    int spl_n;        // spline points (x, y, y2 consecutive blocks)
    int pad_;
};

struct OpticRec {
    double refl, trans, slope, spec;  // slope/spec in mrad
    double n_in, n_out;               // RefractiveIndex[0], [2] after cross-wiring
    int dist;                         // 'g', 'p', 'f', ...
    int refl_tab_off, refl_tab_n;     // (angle, value) pairs in SceneDev::tables
    int trans_tab_off, trans_tab_n;
    int pad_;
};

struct StageRec {
    double R[9];   // global -> stage rotation
    double o[3];
    int first_elem, n_elem;
    int virt, multihit, tracethrough;
    int bvh_off;   // first node in SceneDev::bvh, -1 when brute force is used
    int bvh_items_off;
    // ground grid over the stage's x-y plane (stages spread in x, y within a thin z band,
    // such as heliostat fields): cell (ix, iy) lists every enabled element whose padded
    // bounding disc overlaps it; grid_on = 0 when not built
    int grid_on;
    int gnx, gny, gcell_off;  // cells, first cell in SceneDev::stage_cells
    int flat_only;            // every element of the stage is flat (surface type 3)
    int closed_only;          // every element's surface is intersected in closed form
    float gx0, gy0, gcell, ginv, gzlo, gzhi;
};

// BVH node over element bounding spheres in stage coordinates.  Leaf when
// count > 0: items [first, first + count) of SceneDev::bvh_items; inner nodes
// have children first (left) and first + 1.
struct BvhNode {
    float lo[3], hi[3];
    int first, count;
};

struct FluxMapDev {
    int stage, elem;      // 0-based stage, 0-based element index within the stage
    int kind, nx, ny, absorbed_only;
    int n_src;            // > 0: one map per first-stage element the ray first hit (n_src maps)
    int pad_;
    double x0, x1, y0, y1;
    unsigned long long *bins;
};

struct SunDev {
    double xmin, xmax, ymin, ymax;  // sun box in the sun frame
    double Rsun[9];                 // sun -> first-stage rotation (RLocToRef of the sun frame)
    double pos_sun_stage[3];
    double origin[3];               // sun position (point source)
    int shape;                      // 'g', 'p', 'd', 'f', ...
    int point_source;
    double sigma;                   // mrad
    const double *inv_cdf;          // theta (mrad) at u = j / kSunInvCells, j = 0..kSunInvCells
    // sun-plane culling grid for the first stage (cells over the sun box)
    int grid_on, gnx, gny;
    double gx0, gy0, ginv;          // origin and 1/cell size
    const int *cell_start;          // (start, end) per cell: cell c at [2c, 2c+1], read as int2
    const float4 *cell_disc;        // per cell entry, ascending element order: projected
                                    // centre x, y, radius, element index (int bits)
    const float4 *cell_par;         // per cell entry: rows (a, b), (c, d) of the footprint's
                                    // dual basis; (x, y) about the centre is kept when
                                    // |a x + b y| <= 1 and |c x + d y| <= 1 (all zero: disc only)
    double gcell;                   // cell size (1 / ginv)
    // first stages of flat rectangles only (exact_flat), per cell entry: the footprint centre
    // relative to the cell's lower corner, the padded disc radius squared and the element
    // (xa); the exact footprint's dual basis rows, unpadded (xb); the depth slopes along the
    // sun's z and the depth at the centre (xc; z +inf: the element accepts no hit, NaN: no
    // exact footprint, the float test defers to double)
    int exact_flat;
    const float4 *cell_xa;          // centre x, y (cell-relative), r^2, element (int bits)
    const float4 *cell_xb;          // i00, i01, i10, i11
    const float4 *cell_xc;          // dz/dx, dz/dy, z at the centre, unused
};

struct SceneDev {
    const ElemRec *elems;
    const float4 *elem_sphere;  // per element: origin in stage coordinates and padded bounding radius
    const OpticRec *optics;
    const double *surf_data;
    const double *tables;
    const BvhNode *bvh;
    const int *bvh_items;
    const int2 *stage_cells;     // ground-grid cells of every stage: [start, end) of the entries
    const float4 *grid_sphere;   // ground-grid entries: element bounding sphere (stage coordinates)
    const int *grid_elem;        // ground-grid entries: element index within the stage
    // outgoing-beam lists of flat first-stage elements: rays leaving element j with a
    // direction d such that d . axis >= w (beam_axis[j] = axis, w; w > 1: no list) can only
    // meet the elements beam_elem[beam_range[j].x .. beam_range[j].y) of the stage
    const float4 *beam_axis;
    const int2 *beam_range;
    const int *beam_elem;
    StageRec stages[kMaxStages];
    int n_stages;
    SunDev sun;
    int sunshape_on, errors_on;
    uint32_t seed;
    int precision;  // 0 FP64, 1 mixed
    int explicit_rays;
    const double *ex_pos, *ex_cos;
    int n_flux;
    FluxMapDev flux[kMaxFluxMaps];
};

// One intersection record as the reference stores it (coretrace/types.h:239-246),
// plus the within-(ray, stage) hit index used to restore the reference's order.
struct RecordDev {
    double pos[3], cos[3];
    int element, stage;
    uint32_t raynum, seq;
};

}  // namespace stb
