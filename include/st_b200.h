/*
 * B200 extensions to the SolTrace C API (coretrace_api.so).
 *
 * These entry points have no counterpart in the reference's stapi.h; they
 * expose controls and results of the CUDA trace that a caller of st_sim_run
 * may want without changing the reference-compatible calls in stapi.h.
 * All return 1 (or a non-negative count/index) on success and -1 on a bad
 * context or argument, with the reason in st_message().
 */
#ifndef SOLTRACE_B200_EXT_H
#define SOLTRACE_B200_EXT_H

#include "stapi.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Arithmetic of the per-ray work.
 *   ST_B200_FP64  (default): every ray computation in double precision, rounded as the
 *                  reference's x86-64 build rounds it (no fused multiply-add).
 *   ST_B200_MIXED: aperture tests, property tables, Fresnel coefficients, error sampling
 *                  and flux binning in float; the first-stage probe of flat rectangles
 *                  decides hits in float and defers to double within float rounding (the
 *                  hits are the FP64 probe's); transforms, closed-form roots, the torus
 *                  quartic, Newton refinement, reflection and refraction directions and
 *                  all counters in double / 64-bit integers (positions of explicit rays
 *                  agree with FP64 within 1e-5 m on km paths). */
#define ST_B200_FP64 0
#define ST_B200_MIXED 1
int st_b200_set_precision(st_context_t pcxt, int mode);

/* 1 (default): build the per-intersection records that st_locations & co. read
 * back, in the reference's order (put in that order on the device; the context keeps
 * them in page-locked host memory until its next run).  A run with records holds at
 * most 2^31 of them, and its stages times its ray numbers stay below 2^31.  0: keep
 * only counters and flux maps (the records are then never materialised in device or
 * host memory). */
int st_b200_set_records(st_context_t pcxt, int on);

/* CUDA device ordinal used by st_sim_run (default 0). */
int st_b200_set_device(st_context_t pcxt, int device);

/* Deterministic input: trace these n rays (global position/direction, 3 doubles
 * each) into the first stage instead of sampling sun rays; every supplied ray is
 * traced once and rays that hit the first stage are numbered in input order.
 * n = 0 returns to sun-ray sampling. */
int st_b200_explicit_rays(st_context_t pcxt, st_uint_t n, const double *pos, const double *cos);

/* Flux maps binned on the device at every intersection with (stage, element)
 * (1-based, as in the records), in element-local coordinates (x, y, z).
 *   kind 0: x in [x0,x1) by y in [y0,y1), bins [lower, upper) (pysoltrace's flat map,
 *           pysoltrace.py:1926-1929);
 *   kind 1: cylinder of radius x1: angle atan2(x, z - x1) + pi over [0, 2 pi) by y in
 *           [y0,y1) (pysoltrace's cylinder map, pysoltrace.py:1937-1942; x0 unused);
 *   kind 2: flat, the GUI's rule (app/src/project.cpp:1392-1403): bins (lower, upper]
 *           over [x0,x1] by [y0,y1];
 *   kind 3: full cylinder of radius x1, the GUI's unwrapped arc length over
 *           [-pi x1, pi x1] (project.cpp:1370-1378) by y, bins (lower, upper];
 *   kind 4: tube of radius x1, the nearest node of the polar mesh of the trough example
 *           (app/deploy/api/examples/parabolic-trough-tracking-timeseries/
 *           st_processing_functions.py:174-250): arc r atan2(x, z - x1) against nx cell
 *           centres over the circumference 2 pi x1, y - (y0 + y1)/2 against ny centres over
 *           y1 - y0; every intersection lands in a bin (x0 unused).
 * absorbed_only selects absorbed intersections.  Returns the map index. */
int st_b200_add_flux_map(st_context_t pcxt, int stage, int element, int kind, int nx, int ny, double x0, double x1,
                         double y0, double y1, int absorbed_only);
/* The same map kept once per first-stage element: an intersection is binned into the map of
 * the first-stage element its ray hit first (per heliostat, the flux image it puts on the
 * receiver).  Its counts are n1 maps of nx*ny, [e][iy][ix], n1 the first stage's element count. */
int st_b200_add_source_flux_map(st_context_t pcxt, int stage, int element, int kind, int nx, int ny, double x0,
                                double x1, double y0, double y1, int absorbed_only);
int st_b200_clear_flux_maps(st_context_t pcxt);
/* nx*ny counts (per-source maps: n1*nx*ny), row-major [iy][ix], of the last run. */
int st_b200_flux_counts(st_context_t pcxt, int map, unsigned long long *counts);

typedef struct st_b200_stats {
    unsigned long long sun_rays;          /* generated sun rays (64-bit SunRayCount) */
    unsigned long long ray_hits;          /* rays numbered by a first-stage hit */
    unsigned long long stage_entries[16]; /* rays entering stage i (i < 16) */
    unsigned long long ray_stage_units;   /* sun_rays + sum over stages >= 2 of stage_entries */
    unsigned long long records;           /* intersection records produced */
    double kernel_ms;                     /* device time of the trace kernels */
    double probe_ms, trace_ms;            /* split of kernel_ms */
    double setup_ms, readback_ms;         /* host-side scene upload / result download */
    int batches;                          /* sun-ray batches launched */
    int gpu_launches;                     /* kernels launched by the run */
    unsigned long long h2d_bytes;         /* host -> device bytes copied by the run */
    unsigned long long d2h_bytes;         /* device -> host bytes copied by the run */
    int probe_variant, trace_variant;     /* autotuned kernel variants used */
    unsigned long long intersections;     /* records of the run by the reference's rules,
                                             counted on the device when records are off */
} st_b200_stats;
int st_b200_run_stats(st_context_t pcxt, st_b200_stats *out);

/* Flux statistics of map `map` after a run, as the SolTrace GUI reports them for an element
 * (app/src/project.cpp:1139-1288), for direct normal irradiance `dni` (W/m2):
 * power per ray = dni x sun-box area / SunRayCount; flux of a bin = its count x power per
 * ray / bin area (W/m2); peak and minimum over the bins (the first in x-major order on
 * ties), mean, population standard deviation, uniformity = sigma / mean, and the Monte-
 * Carlo uncertainties 100/sqrt(rays in the peak bin) and 100/sqrt(run intersections), in %.
 * Bin areas: (x1-x0)/nx x (y1-y0)/ny, with 2 pi x1 / nx across a cylinder. */
typedef struct st_b200_flux_stats_t {
    double peak_flux, min_flux, ave_flux, sigma_flux, uniformity;
    double peak_flux_uncertainty, ave_flux_uncertainty;
    double power_per_ray, bin_area;
    unsigned long long rays_binned, rays_in_peak_bin, rays_in_min_bin;
} st_b200_flux_stats_t;
int st_b200_flux_stats(st_context_t pcxt, int map, double dni, st_b200_flux_stats_t *out);

/* Per-element ray accounting of the last run for a stage (1-based): first_hits[e]
 * counts rays whose first intersection in that stage was element e+1; absorbed[e]
 * counts intersections with element e+1 that were absorbed; delivered[e] counts
 * rays whose first stage-1 element was e+1 and that were absorbed in the last
 * stage (the per-heliostat intercept numerator; only filled for stage 1). */
int st_b200_element_counts(st_context_t pcxt, int stage, unsigned long long *first_hits,
                           unsigned long long *absorbed, unsigned long long *delivered);

/* File front end of the SolTrace CLI (coretrace/strace/main.cpp:78-483) as library calls.
 * st_b200_load_stinput reads a .stinput system file (sun, optical property pairs, stages
 * and elements; surface files named in it are read relative to the working directory)
 * into the context, replacing its optics and stages; 1 on success, -1 with the line and
 * the reason in st_message() otherwise.  st_b200_write_rays writes the last run's
 * intersection records in the CLI's .rays text format (sun box, SunRayCount, count, then
 * one line per record in readback order); 1 on success, -1 otherwise. */
int st_b200_load_stinput(st_context_t pcxt, const char *path);
int st_b200_write_rays(st_context_t pcxt, const char *path);

/* Stage-data save and replay: the C form of the reference's st_sim_run_data
 * (coretrace/stapi.cpp:680-728, raytrace.cpp:544-578 and 1044-1078), for loops that
 * re-trace only the stages after the first (a receiver design over a fixed heliostat field).
 *
 * st_b200_set_save_stage_data(ctx, 1): st_sim_run then keeps (records must be on)
 *   s0: every first-stage intersection record in ray order, 8 doubles each: position and
 *       direction (stage frame, as in st_locations/st_cosines), element (negative when
 *       absorbed), ray number;
 *   s1: the second stage's input, 7 doubles each: global position, direction, ray number,
 *       as the reference saves it: its array of the rays that entered the second stage, in
 *       ray order, whose first positions were overwritten in place by the rays that left it.
 * st_b200_stage_data_sizes / st_b200_stage_data read them back (caller-allocated arrays of
 * 8 n0 and 7 n1 doubles).
 * st_b200_sim_run_replay runs the scene from such data: s0 becomes the first stage's records,
 * the s1 rays enter the second stage, SunRayCount is the ray number of the last s0 row, and
 * the stages after the first are traced as by st_sim_run (the replayed rays draw from their
 * own random streams).  Returns the record count, or -1 with a message. */
int st_b200_set_save_stage_data(st_context_t pcxt, int on);
int st_b200_stage_data_sizes(st_context_t pcxt, st_uint_t *n0, st_uint_t *n1);
int st_b200_stage_data(st_context_t pcxt, double *s0, double *s1);
int st_b200_sim_run_replay(st_context_t pcxt, unsigned int seed, st_uint_t n0, const double *s0, st_uint_t n1,
                           const double *s1,
                           int (*callback)(st_uint_t ntracedtotal, st_uint_t ntraced, st_uint_t ntotrace,
                                           st_uint_t curstage, st_uint_t nstages, void *data),
                           void *cbdata);

/* Cap on the sun rays a run may generate beyond the int of st_sim_params' maxcount
 * (stapi.h:154), for runs of more than about 2^31 sun rays (large hit counts, runs over
 * several GPUs); 0 (default) uses maxcount.  SunRayCount is then read from
 * st_b200_run_stats, whose count is 64-bit (st_sun_stats reports an int). */
int st_b200_set_max_sun_rays(st_context_t pcxt, unsigned long long n);

/* One run over several GPUs, one process (or thread) per GPU, each with its own context
 * holding the same scene, flux maps and settings.  No counterpart in the reference, whose
 * front ends run independent contexts with seeds seed + i*123 and concatenate them
 * (app/src/trace.cpp:709-735); here the ranks together make the one run st_sim_run makes
 * on one GPU.  With nranks > 1, st_sim_run(seed) on rank r traces a contiguous slice of every
 * sun-ray batch (every ray keeping its own random stream), numbers its hits after those of
 * the ranks before it, and stops at the same hit as a single-GPU run; the counters, flux maps,
 * per-element counts and SunRayCount it then reports are the whole run's, equal to a single-GPU
 * run's, and its records (st_locations & co.) are the rays this rank traced, numbered as in
 * the whole run.  Every rank must call st_sim_run with the same seed at the same time.
 *   allgather(send[count] -> recv[count * nranks], rank-major) and allreduce(buf[count], op:
 *   0 sum, 1 max) are the caller's collectives over the ranks (torch.distributed, MPI, NCCL);
 *   they return 1 on success, 0 on failure, which fails the run.
 * Explicit rays, replay and stage-data saving are single-GPU only.  nranks = 1 turns it off. */
typedef int (*st_b200_allgather_t)(const unsigned long long *send, unsigned long long *recv, int count, void *user);
typedef int (*st_b200_allreduce_t)(unsigned long long *buf, unsigned long long count, int op, void *user);
int st_b200_set_ranks(st_context_t pcxt, int rank, int nranks, st_b200_allgather_t allgather,
                      st_b200_allreduce_t allreduce, void *user);

/* Batched multi-sun run: K sun positions traced over the context's scene in one launch
 * sequence.  It stands in for K calls of st_sun_xyz + st_sim_run (coretrace/stapi.cpp:
 * 680-734, one Trace per call) that a front end makes for an annual or daily simulation,
 * whose sun vectors come from st_sun_position (stapi.cpp:500-527).
 *   sun_xyz       3 K doubles: the sun position of each run, as st_sun_xyz takes it;
 *   hits          K first-stage hit counts (each as st_sim_params' raycount; maxcount and
 *                 include_dynamic_group come from st_sim_params and apply to every position);
 *   track_target  NULL, or 3 doubles: every first-stage element then tracks the sun,
 *                 re-aimed per position so that its normal bisects the sun direction and
 *                 the direction from its origin to the target (aim point origin + 100 n,
 *                 zrot kept), as a heliostat field aimed at a receiver.
 * Position k draws from the random streams of seed + k: its counters, flux maps and
 * SunRayCount are those of st_sim_run(seed + k) on the context with sun k (and the first
 * stage aimed for sun k).  Precision and flux maps (st_b200_add_flux_map, kept per position)
 * come from the context; records are not built.  The host reads the positions' progress
 * once per wave (a few times per call), not once per position.  Positions go to the device
 * in chunks of 64 through two page-locked staging areas that the context keeps (each sized
 * for its largest chunk: a chunk is staged while the previous one runs) until
 * st_free_context.  Returns 1, or -1 with the reason in st_message(). */
int st_b200_sim_run_batch(st_context_t pcxt, unsigned int seed, int n_positions, const double *sun_xyz,
                          const st_uint_t *hits, const double *track_target);
/* Results of the last batched run.  position >= 0: that position's SunRayCount, hits, stage
 * entries, ray-stage units and intersections; position -1: their sums with the call's device
 * time, set-up time, launches and copies. */
int st_b200_batch_stats(st_context_t pcxt, int position, st_b200_stats *out);
/* nx*ny counts of flux map `map` for one position, row-major [iy][ix]. */
int st_b200_batch_flux_counts(st_context_t pcxt, int map, int position, unsigned long long *counts);
/* absorbed intersections per element of stage `stage` (1-based) for one position. */
int st_b200_batch_absorbed(st_context_t pcxt, int position, int stage, unsigned long long *absorbed);
/* the position's sun box in the sun frame (the power per ray is dni x box area / SunRayCount). */
int st_b200_batch_sun_box(st_context_t pcxt, int position, double *xmin, double *xmax, double *ymin, double *ymax);

/* Flux-surrogate network primitives (BF16 multilayer perceptron on the tensor cores, FP32
 * accumulation).  No counterpart in the reference, which traces every ray; the plain trace
 * makes the network's training data (st_b200_add_source_flux_map) and judges it.  All pointers
 * are device memory of the current device, `stream` a cudaStream_t (NULL: legacy stream);
 * calls are asynchronous.  Return 1, or -1 on a bad argument or launch failure.
 *
 * st_b200_mlp_gemm: C[m x n] = epilogue(A[m x k] B[n x k]^T), A(i, j) at A[i lam + j lak] and
 *   B(i, j) at B[i lbn + j lbk] (bf16), C with leading dimension ldc; epilogue
 *     0: C bf16 = max(acc + bias, 0)        1: C float = acc + bias
 *     2: C bf16 = acc where aux bf16 > 0 (aux shaped as C), else 0
 *     3: C float = acc                      4: C float += acc (atomic; splits > 1 allowed)
 * st_b200_mlp_mse: dy bf16 = 2 (y - t) / (rows cols) and *loss += sum (y - t)^2 (double).
 * st_b200_mlp_colsum: db[c] = sum over rows of dz bf16 [rows x cols].
 * st_b200_mlp_adam: one Adam step of n float weights (w, moments m and v) from gradient g,
 *   writing the bf16 copy w_bf16 when given; step counts from 1.
 * st_b200_mlp_to_bf16: y bf16 = x float.
 * st_b200_mlp_error: 1 when a GEMM's wait for its tensor-core products ran out since the
 *   last call (the flag is then cleared), 0 otherwise. */
int st_b200_mlp_gemm(int m, int n, int k, const void *A, long long lam, long long lak, const void *B, long long lbn,
                     long long lbk, void *C, long long ldc, int epilogue, const float *bias, const void *aux, int splits,
                     void *stream);
int st_b200_mlp_mse(int rows, int cols, const float *y, const float *target, long long ldt, void *dy, double *loss,
                    void *stream);
int st_b200_mlp_colsum(int rows, int cols, const void *dz, float *db, void *stream);
int st_b200_mlp_adam(long long n, float *w, const float *g, float *m, float *v, void *w_bf16, float lr, float beta1,
                     float beta2, float eps, int step, void *stream);
int st_b200_mlp_to_bf16(long long n, const float *x, void *y, void *stream);
int st_b200_mlp_error(void);

/* Fused inference: the whole network in one persistent kernel (one CTA per SM), activations
 * kept in shared memory between layers, weights streamed from a packed copy.  Shapes: 2 to 8
 * layers, dims[0] (inputs) 1 to 16, every hidden width 256, the output width dims[n_layers] a
 * multiple of 256 up to 4096.
 *
 * st_b200_mlp_packed_bytes: size of the packed weights for those dims, -1 if unsupported.
 * st_b200_mlp_pack: lays the bf16 weights w[l] (dims[l+1] x dims[l], row-major) out in
 *   `packed` in the order and shared-memory layout the fused kernel streams them.
 * st_b200_mlp_forward_fused: y = the network applied to the m rows of x (bf16, leading
 *   dimension ldx), bias[l] float; each output value becomes v = y scale (clamped to >= 0
 *   when clamp is set) and
 *     mode 0: out[r dims[n_layers] + j] = v                       (every row's output)
 *     mode 1: out[(r / group_rows) dims[n_layers] + j] += v       (sum over groups of rows,
 *             e.g. every heliostat of a field: the field's receiver map; out pre-zeroed) */
long long st_b200_mlp_packed_bytes(int n_layers, const int *dims);
int st_b200_mlp_pack(int n_layers, const int *dims, const void *const *w, void *packed, void *stream);
int st_b200_mlp_forward_fused(int n_layers, const int *dims, const void *packed, const float *const *bias, int m,
                              const void *x, long long ldx, float *out, int mode, int group_rows, float scale,
                              int clamp, void *stream);

/* First-stage probe without device allocation.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: code running inside a framework that owns
 * the device's memory pool, or a real-time loop in which an allocation (which may
 * synchronise the whole device) is not allowed.  For the context's scene it traces sun
 * rays [s0, s0 + n) (with the per-ray streams of `seed`, exactly as st_sim_run does)
 * to the first stage and writes, in sun-ray order, the sun index and the 0-based
 * element of every ray that hits into the caller's device arrays hit_sid and
 * hit_elem (room for n entries each); *n_hits receives the count.  The k-th listed
 * hit is the ray st_sim_run numbers k.  Arithmetic is FP64.
 *
 * The call runs on the context's device (st_b200_set_device, default 0): hit_sid,
 * hit_elem and `stream` must belong to that device; the caller's current device is
 * restored before returning.  A context given explicit rays (st_b200_explicit_rays) is
 * rejected with -1: the probe lists generated sun rays only.
 *
 * Scene tables and scratch live in a 48 MiB static device array that every GPU
 * loading this library keeps until the process exits; n <= 4194304 and scenes whose
 * tables do not fit are rejected with -1 and a message.  The first call on a device
 * looks up the array's address.  Every call copies its tables from host memory and
 * waits for its work to finish, so the entry point must not be called while `stream`
 * is being captured into a CUDA graph.  Calls share the array: calls that overlap on
 * the GPU race.  `stream` is a cudaStream_t (NULL: the legacy default stream). */
int st_b200_probe_noalloc(st_context_t pcxt, unsigned int seed, unsigned long long s0, unsigned int n,
                          unsigned long long *hit_sid, unsigned int *hit_elem, unsigned int *n_hits, void *stream);

#ifdef __cplusplus
}
#endif
#endif
