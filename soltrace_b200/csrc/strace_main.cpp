// strace_b200: the SolTrace command-line tracer on the B200 library.
//
//   strace_b200 <system.stinput> <rays> <max rays> <seed> <sunshape 0/1> <errors 0/1>
//               [<point focus 0/1>] [--mixed] [--device N] [--no-rays]
//
// The positional arguments are those of the reference CLI (coretrace/strace/main.cpp:
// 501-560): rays = first-stage hits to trace, max rays = cap on generated sun rays, point
// focus = the "as power tower" flag of st_sim_params.  The system is read with
// st_b200_load_stinput, traced with st_sim_run, and the records are written next to the
// input as <system.stinput>.rays (st_b200_write_rays).  --mixed selects the mixed
// FP32/FP64 trace, --device the CUDA device, --no-rays skips the records (counters only).
// Exit status 0 on success, 1 on a failed read, trace or write (messages on stderr).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "stapi.h"
#include "st_b200.h"

static void print_messages(st_context_t cx) {
    for (int j = 0; j < st_num_messages(cx); ++j) fprintf(stderr, "error: %s\n", st_message(cx, j));
}

int main(int argc, char **argv) {
    if (argc < 7) {
        fprintf(stderr,
                "usage: strace_b200 <system.stinput> <rays> <max rays> <seed> <sunshape 0/1> <errors 0/1> "
                "[<point focus 0/1>] [--mixed] [--device N] [--no-rays]\n");
        return 1;
    }
    const char *file = argv[1];
    const int nrays = atoi(argv[2]), maxrays = atoi(argv[3]), seed = atoi(argv[4]);
    const int sunshape = atoi(argv[5]), errors = atoi(argv[6]);
    int point_focus = 0, mixed = 0, device = 0, write = 1;
    for (int i = 7; i < argc; ++i) {
        if (!strcmp(argv[i], "--mixed"))
            mixed = 1;
        else if (!strcmp(argv[i], "--no-rays"))
            write = 0;
        else if (!strcmp(argv[i], "--device") && i + 1 < argc)
            device = atoi(argv[++i]);
        else if (i == 7)
            point_focus = atoi(argv[i]);
    }
    st_context_t cx = st_create_context();
    int rc = 1;
    if (st_b200_load_stinput(cx, file) < 0) {
        print_messages(cx);
    } else {
        st_sim_params(cx, nrays, maxrays, point_focus);
        st_sim_errors(cx, sunshape, errors);
        st_b200_set_precision(cx, mixed ? ST_B200_MIXED : ST_B200_FP64);
        st_b200_set_records(cx, write);
        st_b200_set_device(cx, device);
        const int code = st_sim_run(cx, (unsigned int)seed, nullptr, nullptr);
        if (code < 0) {
            print_messages(cx);
        } else {
            st_b200_stats s;
            st_b200_run_stats(cx, &s);
            printf("trace finished: %llu sun rays, %llu hits, %llu records, %.3f ms on the device\n", s.sun_rays,
                   s.ray_hits, s.intersections, s.kernel_ms);
            rc = 0;
            if (write) {
                const std::string out = std::string(file) + ".rays";
                if (st_b200_write_rays(cx, out.c_str()) < 0) {
                    print_messages(cx);
                    rc = 1;
                } else {
                    printf("records written to %s\n", out.c_str());
                }
            }
        }
    }
    st_free_context(cx);
    return rc;
}
