// scmf: command-line drop-in for the reference's `scmf` executable
// (main.cpp:7-19, test.cpp:9-135, init.cpp:3-52).
//
// Reads configuration.dat and polymer.dat from the working directory, accepts
// the reference flags -GPU_N= -gpu<i>= -Check_T= (default 1000) -Start_time=
// (0) -Steps_N= (100) -read_file= (0), and writes density_<step>.dat every
// Check_T steps, coord.dat at the end, and the "step %d end to end dis %g" /
// "time =%g" lines.  Added flags: -seed= (default time(NULL), as
// init_config.cu:864), -field_rule=every, -Aver_T=<n> (time-averaged density
// over every n-th sweep, density_aver_<step>.dat beside each density file,
// io.cpp:57-94), -checkpoint=1 (binary checkpoint.bin at the end) and
// -read_file=2 (exact resume from checkpoint.bin, its step replacing
// -Start_time).  One GPU only: -GPU_N > 1 is an error (the multi-GPU density
// reduction of mesh.cu:10-81 is not built).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "scmf.h"

static int arg_int(int argc, char** argv, const char* name, int dflt, bool* present = nullptr) {
    const size_t n = strlen(name);
    for (int i = 1; i < argc; ++i) {
        const char* a = argv[i];
        while (*a == '-') ++a;
        if (strncmp(a, name, n) == 0 && a[n] == '=') {
            if (present) *present = true;
            return atoi(a + n + 1);
        }
    }
    if (present) *present = false;
    return dflt;
}

static const char* arg_str(int argc, char** argv, const char* name) {
    const size_t n = strlen(name);
    for (int i = 1; i < argc; ++i) {
        const char* a = argv[i];
        while (*a == '-') ++a;
        if (strncmp(a, name, n) == 0 && a[n] == '=') return a + n + 1;
    }
    return nullptr;
}

#define TRY(expr)                                                                  \
    do {                                                                           \
        scmf_status rc_ = (expr);                                                  \
        if (rc_ != SCMF_OK) {                                                      \
            fprintf(stderr, "scmf: %s failed: %s\n", #expr, scmf_last_error());   \
            return 1;                                                              \
        }                                                                          \
    } while (0)

// Mean squared end-to-end distance over all chains (test.cpp:47-68 averages
// |r_0 - r_31|^2 over every chain), from the device reduction.
static scmf_status end_to_end(const scmf_system* sys, int n_arch, double* out) {
    std::vector<scmf_observables> o((size_t)n_arch);
    scmf_status rc = scmf_analyze(sys, o.data(), n_arch);
    if (rc) return rc;
    double s = 0, n = 0;
    for (const auto& v : o) {
        if (v.n_chains == 0) continue;
        s += v.re2[3] * v.n_chains;
        n += v.n_chains;
    }
    *out = n > 0 ? s / n : 0.0;
    return SCMF_OK;
}

int main(int argc, char** argv) {
    int gpu_n = arg_int(argc, argv, "GPU_N", 0);
    if (gpu_n == 0) gpu_n = 1;
    if (gpu_n != 1) {
        fprintf(stderr, "scmf: this engine runs one system on one GPU (-GPU_N=%d)\n", gpu_n);
        return 2;
    }
    const int gpu0 = arg_int(argc, argv, "gpu0", 0);
    int tcheck = arg_int(argc, argv, "Check_T", 0);
    if (tcheck == 0) tcheck = 1000;
    const int start = arg_int(argc, argv, "Start_time", 0);
    int nsteps = arg_int(argc, argv, "Steps_N", 0);
    if (nsteps == 0) nsteps = 100;
    const int read_file = arg_int(argc, argv, "read_file", 0);
    const int aver_t = arg_int(argc, argv, "Aver_T", 0);
    const int want_checkpoint = arg_int(argc, argv, "checkpoint", 0);
    bool seed_given = false;
    const int seed_arg = arg_int(argc, argv, "seed", 0, &seed_given);
    const uint64_t seed = seed_given ? (uint64_t)(uint32_t)seed_arg : (uint64_t)time(NULL);
    const char* rule = arg_str(argc, argv, "field_rule");
    if (cudaSetDevice(gpu0) != cudaSuccess) {
        fprintf(stderr, "scmf: cannot use GPU %d\n", gpu0);
        return 1;
    }

    scmf_spec* spec = nullptr;
    TRY(scmf_spec_load_files("configuration.dat", "polymer.dat", seed, &spec));
    if (rule && strcmp(rule, "every") == 0) {
        scmf_params p;
        TRY(scmf_spec_get_params(spec, &p));
        p.field_rule = SCMF_FIELD_EVERY;
        TRY(scmf_spec_set_params(spec, &p));
    }
    scmf_spec_info info;
    TRY(scmf_spec_get_info(spec, &info));
    scmf_system* sys = nullptr;
    TRY(scmf_system_create(spec, nullptr, &sys));
    TRY(scmf_init_coords(sys));
    std::vector<float> xyz((size_t)info.n_beads * 3);
    if (read_file == 1) {
        FILE* f = fopen("coord.dat", "r");
        if (!f) {
            printf("coord.dat did not exit ^_^, program smartly change config to generate a random coord.\n");
        } else {
            fclose(f);
            TRY(scmf_read_coords_file("coord.dat", 0, xyz.data(), xyz.size()));
            TRY(scmf_set_coords(sys, xyz.data(), xyz.size()));
        }
    }
    int step = start;
    if (read_file == 2) {
        FILE* f = fopen("checkpoint.bin", "rb");
        if (!f) {
            fprintf(stderr, "scmf: -read_file=2 needs checkpoint.bin\n");
            return 1;
        }
        fclose(f);
        TRY(scmf_checkpoint_read(sys, "checkpoint.bin"));
        scmf_stats st;
        TRY(scmf_get_sweep_stats(sys, &st));
        step = (int)st.step;
    } else {
        TRY(scmf_set_step(sys, (uint64_t)start));
    }
    bool have_samples = false;  // the accumulator holds at least one sweep
    const int aver_from = step;
    if (aver_t > 0) {
        scmf_checkpoint_header h;
        // a resumed run keeps the checkpoint's accumulator when it averages at the same cadence
        const bool keep = read_file == 2 && scmf_checkpoint_info("checkpoint.bin", &h) == SCMF_OK &&
                          h.avg_every == (uint32_t)aver_t;
        if (!keep) TRY(scmf_average_start(sys, (uint32_t)aver_t));
        have_samples = keep && h.avg_samples > 0;
    }
    const int last = step + nsteps;
    while (step < last) {
        int next = ((step / tcheck) + 1) * tcheck;
        if (next > last) next = last;
        TRY(scmf_step(sys, next - step));
        step = next;
        if (step % tcheck == 0) {
            double ree = 0;
            TRY(end_to_end(sys, info.n_arch, &ree));
            printf("step %d end to end dis %g\n", step, ree);
            TRY(scmf_write_density(sys, nullptr, step));
            if (aver_t > 0 && (have_samples || step / aver_t > aver_from / aver_t))
                TRY(scmf_write_average_density(sys, nullptr, step));
        }
    }
    TRY(scmf_write_coords(sys, "coord.dat"));
    if (want_checkpoint) TRY(scmf_checkpoint_write(sys, "checkpoint.bin"));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    void* st = nullptr;
    scmf_system_stream(sys, &st);
    cudaEventRecord(e0, (cudaStream_t)st);
    TRY(scmf_smc_move(sys, 1));
    TRY(scmf_reset_density_fields(sys));
    TRY(scmf_update_omega_fields_scmf0(sys));
    cudaEventRecord(e1, (cudaStream_t)st);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    printf("time =%g\n", ms);
    scmf_system_destroy(sys);
    scmf_spec_destroy(spec);
    return 0;
}
