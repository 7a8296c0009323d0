/*
 * SolTrace core C API, served by the B200 trace (coretrace_api.so).
 *
 * Every declaration below is the one a SolTrace front end binds today; each
 * replaces the function of the same name declared in coretrace/stapi.h of the
 * reference (lines cited per group) with the same argument meaning, return
 * codes and ownership:
 *   - setters return 1 on success and -1 on a bad context, stage or element index;
 *   - st_add_* return the new index (or the count added);
 *   - readback functions fill caller-allocated arrays of st_num_intersections()
 *     entries and return 1;
 *   - st_sim_run returns the number of intersection records, or -1 with the
 *     reason available through st_num_messages()/st_message().
 * Types are the reference's: st_uint_t is `unsigned long`, st_context_t is an
 * opaque pointer.  B200-specific controls live in st_b200.h.
 */
#ifndef SOLTRACE_B200_STAPI_H
#define SOLTRACE_B200_STAPI_H

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned long st_uint_t;
typedef void *st_context_t;

/* contexts (reference coretrace/stapi.h:76-77) */
st_context_t st_create_context(void);
int st_free_context(st_context_t pcxt);

/* messages (stapi.h:80-82) */
int st_num_messages(st_context_t pcxt);
const char *st_message(st_context_t pcxt, st_uint_t idx);
void st_clear_messages(st_context_t pcxt);

/* optical property sets (stapi.h:92-105) */
int st_num_optics(st_context_t pcxt);
int st_add_optic(st_context_t pcxt, const char *name);
int st_delete_optic(st_context_t pcxt, st_uint_t idx);
int st_clear_optics(st_context_t pcxt);
int st_optic(st_context_t pcxt, st_uint_t idx, int fb, /* 1 = front, 2 = back */
             char dist, int optnum, int apgr, int order, double rreal, double rimag, double ref, double tra,
             double gratingab12[3], double rmsslope, double rmsspec, int userefltable, int refl_npoints,
             double *refl_angles, double *refls, int usetranstable, int trans_npoints, double *trans_angles,
             double *transs);

/* stages (stapi.h:108-116) */
int st_num_stages(st_context_t pcxt);
int st_add_stage(st_context_t pcxt);
int st_add_stages(st_context_t pcxt, st_uint_t num);
int st_delete_stage(st_context_t pcxt, st_uint_t idx);
int st_clear_stages(st_context_t pcxt);
int st_stage_xyz(st_context_t pcxt, st_uint_t idx, double x, double y, double z);
int st_stage_aim(st_context_t pcxt, st_uint_t idx, double ax, double ay, double az);
int st_stage_zrot(st_context_t pcxt, st_uint_t idx, double zrot);
int st_stage_flags(st_context_t pcxt, st_uint_t idx, int virt, int multihit, int tracethrough);

/* elements (stapi.h:119-136) */
int st_num_elements(st_context_t pcxt, st_uint_t stage);
int st_add_element(st_context_t pcxt, st_uint_t stage);
int st_add_elements(st_context_t pcxt, st_uint_t stage, st_uint_t num);
int st_delete_element(st_context_t pcxt, st_uint_t stage, st_uint_t idx);
int st_clear_elements(st_context_t pcxt, st_uint_t stage);
int st_element_enabled(st_context_t pcxt, st_uint_t stage, st_uint_t idx, int enabled);
int st_element_xyz(st_context_t pcxt, st_uint_t stage, st_uint_t idx, double x, double y, double z);
int st_element_aim(st_context_t pcxt, st_uint_t stage, st_uint_t idx, double ax, double ay, double az);
int st_element_zrot(st_context_t pcxt, st_uint_t stage, st_uint_t idx, double zrot);
int st_element_aperture(st_context_t pcxt, st_uint_t stage, st_uint_t idx, char ap);
int st_element_aperture_params(st_context_t pcxt, st_uint_t stage, st_uint_t idx, double params[8]);
int st_element_surface(st_context_t pcxt, st_uint_t stage, st_uint_t idx, char surf);
int st_element_surface_params(st_context_t pcxt, st_uint_t stage, st_uint_t idx, double params[8]);
int st_element_surface_file(st_context_t pcxt, st_uint_t stage, st_uint_t idx, const char *file);
int st_element_interaction(st_context_t pcxt, st_uint_t stage, st_uint_t idx, int type); /* 1 refract, 2 reflect */
int st_element_optic(st_context_t pcxt, st_uint_t stage, st_uint_t idx, const char *name);

/* sun (stapi.h:139-142) */
int st_sun(st_context_t pcxt, int point_source, char shape, double sigma_halfwidth);
int st_sun_xyz(st_context_t pcxt, double x, double y, double z);
int st_sun_position(st_context_t pcxt, double lat, double day, double hour, double *x, double *y, double *z);
int st_sun_userdata(st_context_t pcxt, st_uint_t npoints, double angle[], double intensity[]);

/* intersection readback (stapi.h:145-151) */
int st_num_intersections(st_context_t pcxt);
int st_locations(st_context_t pcxt, double *loc_x, double *loc_y, double *loc_z);
int st_cosines(st_context_t pcxt, double *cos_x, double *cos_y, double *cos_z);
int st_elementmap(st_context_t pcxt, int *element_map);
int st_stagemap(st_context_t pcxt, int *stage_map);
int st_raynumbers(st_context_t pcxt, int *ray_numbers);
int st_sun_stats(st_context_t pcxt, double *xmin, double *xmax, double *ymin, double *ymax, int *nsunrays);

/* simulation (stapi.h:154-157) */
int st_sim_params(st_context_t pcxt, int raycount, int maxcount, int include_dynamic_group);
int st_sim_errors(st_context_t pcxt, int include_sun_shape, int include_optics);
int st_sim_run(st_context_t pcxt, unsigned int seed,
               int (*callback)(st_uint_t ntracedtotal, st_uint_t ntraced, st_uint_t ntotrace, st_uint_t curstage,
                               st_uint_t nstages, void *data),
               void *data);

/* transform utilities (stapi.h:166-171) */
void st_calc_euler_angles(double origin[3], double aimpoint[3], double zrot, double euler[3]);
void st_transform_to_local(double posref[3], double cosref[3], double origin[3], double rreftoloc[3][3],
                           double posloc[3], double cosloc[3]);
void st_transform_to_reference(double posloc[3], double cosloc[3], double origin[3], double rloctoref[3][3],
                               double posref[3], double cosref[3]);
void st_matrix_vector_mult(double m[3][3], double v[3], double mxv[3]);
void st_calc_transform_matrices(double euler[3], double rreftoloc[3][3], double rloctoref[3][3]);
void st_matrix_transpose(double input[3][3], double output[3][3]);

#ifdef __cplusplus
}
#endif
#endif
