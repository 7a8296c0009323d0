// Test harness (not product code): C entry points around the reference's C++-only
// st_sim_run_data (coretrace/stapi.cpp:680-728), so that the tests can save stage data
// with the reference and replay it, through ctypes.  Built with the reference's own
// objects by `make -C oracle ref` into oracle/_ref/coretrace_ref_sd.so.
#include <cstddef>
#include <vector>

#include "stapi.h"

// defined in the reference's stapi.cpp with C++ linkage; its header leaves the declaration
// commented out, so it is declared here with the definition's signature
int st_sim_run_data(st_context_t pcxt, unsigned int seed, std::vector<std::vector<double> > *data_s1,
                    std::vector<std::vector<double> > *data_s2, bool save_stage_data,
                    int (*callback)(st_uint_t, st_uint_t, st_uint_t, st_uint_t, st_uint_t, void *), void *data);

static std::vector<std::vector<double>> g_s0, g_s1;

extern "C" int ref_sd_run_save(st_context_t cx, unsigned int seed) {
    g_s0.clear();
    g_s1.clear();
    return st_sim_run_data(cx, seed, &g_s0, &g_s1, true, nullptr, nullptr);
}

extern "C" int ref_sd_sizes(unsigned long *n0, unsigned long *n1) {
    *n0 = g_s0.size();
    *n1 = g_s1.size();
    return 1;
}

extern "C" int ref_sd_get(double *s0, double *s1) {
    for (size_t i = 0; i < g_s0.size(); ++i)
        for (size_t j = 0; j < 8; ++j) s0[8 * i + j] = j < g_s0[i].size() ? g_s0[i][j] : 0.0;
    for (size_t i = 0; i < g_s1.size(); ++i)
        for (size_t j = 0; j < 7; ++j) s1[7 * i + j] = j < g_s1[i].size() ? g_s1[i][j] : 0.0;
    return 1;
}

extern "C" int ref_sd_run_replay(st_context_t cx, unsigned int seed, unsigned long n0, const double *s0,
                                 unsigned long n1, const double *s1) {
    std::vector<std::vector<double>> v0(n0, std::vector<double>(8)), v1(n1, std::vector<double>(7));
    for (unsigned long i = 0; i < n0; ++i)
        for (int j = 0; j < 8; ++j) v0[i][j] = s0[8 * i + j];
    for (unsigned long i = 0; i < n1; ++i)
        for (int j = 0; j < 7; ++j) v1[i][j] = s1[7 * i + j];
    return st_sim_run_data(cx, seed, &v0, &v1, false, nullptr, nullptr);
}
