// C entry points into the reference's own device functions, compiled for the
// host (test infrastructure only; built by `make -C oracle ref_harness` from
// the reference checkout into _ref/, never shipped).  They let the tests check
// the oracle's restatement function by function:
//   rh_fold   coord_to_index_unified_high   device_function.cu:313-360
//   rh_omega  omega_field_update            device_function.cu:373-412
//   rh_trial  trial_move_smc_arr + add_bond_forces_arr + calc_delta_energy_arr
//             (+ calc_delta_bonded_energy_arr)  device_function.cu:509-717
//   rh_sweeps mc_polymer_move_arr, the whole sweep  device_function.cu:718-799
// Each call builds the reference's Phase_info_gpu / Poly_arch for the case at
// hand (one linear chain architecture), with the derived quantities the
// reference's initialisation gives them (init_config.cu:565, 664, 807-808).
#include <stdint.h>

#include <cstring>
#include <random>
#include <vector>

#include "struct.h"

dim3 blockIdx, threadIdx, gridDim, blockDim;

// cuRAND stand-ins.  For single trials (rh_trial) the harness sets the next
// Gaussian triple and uniforms are 1/2.  For whole sweeps (rh_sweeps) they
// draw from a seeded host generator instead: uniforms in (0, 1] as cuRAND's,
// independent standard normals.  In that mode the bead-selection draw of each
// trial (the one curand_uniform_double call per trial of mc_polymer_move_arr,
// device_function.cu:749) also notes the bead it selects, so the harness can
// tell afterwards whether that trial moved it (accepted moves are counted
// without touching the reference's code).
static float4 g_normal = {0.0f, 0.0f, 0.0f, 0.0f};
static bool g_random = false;
static std::mt19937_64 g_rng;
static const float* g_pos = nullptr;
static int g_len = 0;
static long g_pending = -1;  // global bead index of the last selected bead, -1: none
static float g_before[3];
static long long g_accepts = 0;

static double uniform_open0() {  // (0, 1]
    return 1.0 - std::uniform_real_distribution<double>(0.0, 1.0)(g_rng);
}
static void settle_trial() {
    if (g_pending < 0) return;
    const float* q = g_pos + 3 * g_pending;
    if (q[0] != g_before[0] || q[1] != g_before[1] || q[2] != g_before[2]) ++g_accepts;
    g_pending = -1;
}
void curand_init(unsigned long long, unsigned long long, unsigned long long, curandStatePhilox4_32_10_t*) {}
float curand_uniform(curandStatePhilox4_32_10_t*) { return g_random ? (float)uniform_open0() : 0.5f; }
double curand_uniform_double(curandStatePhilox4_32_10_t*) {
    if (!g_random) return 0.5;
    settle_trial();
    const double u = uniform_open0();
    int b = (int)(u * g_len);  // the reference's selection rule (device_function.cu:749-751)
    if (b == g_len) b = g_len - 1;
    g_pending = (long)blockIdx.x * g_len + b;
    std::memcpy(g_before, g_pos + 3 * g_pending, sizeof g_before);
    return u;
}
float4 curand_normal4(curandStatePhilox4_32_10_t*) {
    if (!g_random) return g_normal;
    std::normal_distribution<double> n(0.0, 1.0);
    return float4{(float)n(g_rng), (float)n(g_rng), (float)n(g_rng), (float)n(g_rng)};
}
double4 curand_normal4_double(curandStatePhilox4_32_10_t*) {
    return double4{g_normal.x, g_normal.y, g_normal.z, g_normal.w};
}

// the reference functions (external linkage in device_function.cu)
unsigned int coord_to_index_unified_high(const double rx, const double ry, const double rz, const unsigned int rtype,
                                         Phase_info_gpu* phase_info_gpu);
void omega_field_update(int* density, double* omega_field, Phase_info_gpu* phase_info_gpu);
void trial_move_smc_arr(curandStatePhilox4_32_10_t* state, float* pos, int poly_id, int mono_id, int poly_type,
                        int poly_index, Phase_info_gpu* phase_info_gpu, Poly_arch* poly_arch, float* dx, float* dy,
                        float* dz, double* smc_deltaE);
double calc_delta_energy_arr(int poly_id, int mono_id, int poly_type, float* pos, Phase_info_gpu* phase_info_gpu,
                             Poly_arch* poly_arch, double* omega_field_unified, double xold, double yold, double zold,
                             double dx, double dy, double dz, const unsigned int iwtype);
void mc_polymer_move_arr(Phase_info_gpu* phase_info_gpu, Poly_arch* poly_arch, float* pos,
                         curandStatePhilox4_32_10_t* state, double* omega_field_unified);

namespace {
struct Grid {
    Phase_info_gpu p{};
    std::vector<double> A, R, scaling, xn;
    std::vector<unsigned int> poly_basis, mono_basis;
    Grid(double lx, double ly, double lz, int nx, int ny, int nz, int n_types) {
        p.Lx = lx; p.Ly = ly; p.Lz = lz;
        p.nx = nx; p.ny = ny; p.nz = nz;
        p.dx = lx / nx; p.dy = ly / ny; p.dz = lz / nz;   // init_config.cu:565
        p.n_cells = (long)nx * ny * nz;
        p.n_mono_types = n_types;
        A.assign(n_types, 0.0);
        R.assign(n_types, 0.0);
        p.A = A.data();
        p.R = R.data();
    }
};
}  // namespace

extern "C" {

// Cell index (type * n_cells + x + y nx + z nx ny) of each point, the FP32
// coordinates widened to double as the reference's callers do.
void rh_fold(double lx, double ly, double lz, int nx, int ny, int nz, int type, int64_t n, const float* xyz,
             uint32_t* out) {
    Grid g(lx, ly, lz, nx, ny, nz, type + 1);
    for (int64_t i = 0; i < n; ++i)
        out[i] = coord_to_index_unified_high((double)xyz[3 * i], (double)xyz[3 * i + 1], (double)xyz[3 * i + 2],
                                             (unsigned)type, &g.p);
}

// omega (FP64, [type][cell]) of integer counts with the SCMF0 field, every
// type scaled by `scaling` (n_cells / n_beads, init_config.cu:785) and
// 1/N_ref (inverse_refbeads), xn[t + n*s] as Phase_info_gpu::xn.
void rh_omega(int n_types, int64_t n_cells, const int* counts, const double* xn, int nref, double scaling,
              double* omega) {
    Grid g(1, 1, 1, 1, 1, 1, n_types);
    g.p.n_cells = n_cells;
    g.scaling.assign(n_types, scaling);
    g.p.field_scaling_type = g.scaling.data();
    g.p.inverse_refbeads = 1.0 / nref;
    g.p.reference_Nbeads = nref;
    g.xn.assign(xn, xn + n_types * n_types);
    g.p.xn = g.xn.data();
    blockDim = dim3{1, 1, 1};
    gridDim = dim3{(unsigned)n_cells, 1, (unsigned)n_types};
    std::vector<int> dens(counts, counts + n_types * n_cells);
    for (unsigned t = 0; t < (unsigned)n_types; ++t)
        for (int64_t c = 0; c < n_cells; ++c) {
            blockIdx = dim3{(unsigned)c, 0, t};
            threadIdx = dim3{0, 0, 0};
            omega_field_update(dens.data(), omega, &g.p);
        }
}

// One smart-MC trial of bead b of a linear chain of L beads (positions AoS
// float[3L], monomer types[L]) with the Gaussian triple r: the reference's
// displacement d (float, trial_move_smc_arr), its smart-MC term, and
// calc_delta_energy_arr (omega difference + bonded change, FP64) on omega
// (double [n_types * n_cells]).  e_out = {smc_deltaE, calc_delta_energy_arr}.
void rh_trial(int L, const int* types, const float* pos, int b, double harmonic_normb, double smc_a, const float* r,
              double lx, double ly, double lz, int nx, int ny, int nz, int n_types, const double* omega,
              float* d_out, double* e_out) {
    Grid g(lx, ly, lz, nx, ny, nz, n_types);
    for (int t = 0; t < n_types; ++t) {
        g.A[t] = smc_a;
        g.R[t] = sqrt(smc_a * 2);   // init_config.cu:807-808
    }
    g.p.harmonic_normb = harmonic_normb;
    g.p.polymer_type_number = 1;
    g.poly_basis = {0u, 1u};
    g.mono_basis = {0u};
    g.p.polymer_basis_gpu = g.poly_basis.data();
    g.p.monomer_poly_basis_gpu = g.mono_basis.data();
    g.p.num_all_beads_per_gpu = (unsigned)L;
    std::vector<int> mono(types, types + L), neigh_num(L);
    std::vector<std::vector<int>> lists(L);
    for (int i = 0; i < L; ++i) {
        if (i > 0) lists[i].push_back(i - 1);
        if (i + 1 < L) lists[i].push_back(i + 1);
        neigh_num[i] = (int)lists[i].size();
    }
    std::vector<int*> list_ptr(L);
    for (int i = 0; i < L; ++i) list_ptr[i] = lists[i].data();
    Poly_arch arch{};
    arch.poly_length = L;
    arch.Monotype = mono.data();
    arch.neigh_num = neigh_num.data();
    arch.conection_list = list_ptr.data();
    std::vector<float> p(pos, pos + 3 * L);
    std::vector<double> w(omega, omega + (size_t)n_types * g.p.n_cells);
    curandStatePhilox4_32_10_t st{};
    g_normal = float4{r[0], r[1], r[2], 0.0f};
    float dx = 0, dy = 0, dz = 0;
    double smc = 0;
    trial_move_smc_arr(&st, p.data(), 0, b, 0, 0, &g.p, &arch, &dx, &dy, &dz, &smc);
    const double e = calc_delta_energy_arr(0, b, 0, p.data(), &g.p, &arch, w.data(), p[3 * b], p[3 * b + 1],
                                           p[3 * b + 2], dx, dy, dz, (unsigned)types[b]);
    d_out[0] = dx;
    d_out[1] = dy;
    d_out[2] = dz;
    e_out[0] = smc;
    e_out[1] = e;
}

// K sweeps of the reference's own sweep kernel, mc_polymer_move_arr
// (device_function.cu:718-799: per chain, L trials of beads picked at random
// with replacement), over n_chains linear chains of L beads (monomer types[L])
// whose positions (AoS float[3 n_chains L]) are updated in place, in a static
// field omega (double [n_types * n_cells]; no field update between sweeps), with
// the cuRAND stand-ins drawing from a host generator seeded with `seed`.  The
// chains run one after another (a chain's kernel thread at a time; chains do
// not interact within a sweep in a static field).  Returns the accepted moves.
long long rh_sweeps(int n_chains, int L, const int* types, float* pos, int K, double harmonic_normb, double smc_a,
                    double lx, double ly, double lz, int nx, int ny, int nz, int n_types, const double* omega,
                    uint64_t seed) {
    Grid g(lx, ly, lz, nx, ny, nz, n_types);
    for (int t = 0; t < n_types; ++t) {
        g.A[t] = smc_a;
        g.R[t] = sqrt(smc_a * 2);   // init_config.cu:807-808
    }
    g.p.harmonic_normb = harmonic_normb;
    g.p.polymer_type_number = 1;
    g.poly_basis = {0u, (unsigned)n_chains};
    g.mono_basis = {0u};
    g.p.polymer_basis_gpu = g.poly_basis.data();
    g.p.monomer_poly_basis_gpu = g.mono_basis.data();
    g.p.num_all_beads_per_gpu = (unsigned)(n_chains * L);
    std::vector<int> mono(types, types + L), neigh_num(L);
    std::vector<std::vector<int>> lists(L);
    for (int i = 0; i < L; ++i) {
        if (i > 0) lists[i].push_back(i - 1);
        if (i + 1 < L) lists[i].push_back(i + 1);
        neigh_num[i] = (int)lists[i].size();
    }
    std::vector<int*> list_ptr(L);
    for (int i = 0; i < L; ++i) list_ptr[i] = lists[i].data();
    Poly_arch arch{};
    arch.poly_length = L;
    arch.Monotype = mono.data();
    arch.neigh_num = neigh_num.data();
    arch.conection_list = list_ptr.data();
    std::vector<double> w(omega, omega + (size_t)n_types * g.p.n_cells);
    std::vector<curandStatePhilox4_32_10_t> states((size_t)n_chains);
    g_rng.seed(seed);
    g_random = true;
    g_pos = pos;
    g_len = L;
    g_pending = -1;
    g_accepts = 0;
    blockDim = dim3{1, 1, 1};
    gridDim = dim3{(unsigned)n_chains, 1, 1};
    threadIdx = dim3{0, 0, 0};
    for (int k = 0; k < K; ++k)
        for (int c = 0; c < n_chains; ++c) {
            blockIdx = dim3{(unsigned)c, 0, 0};
            mc_polymer_move_arr(&g.p, &arch, pos, states.data(), w.data());
            settle_trial();
        }
    g_random = false;
    g_pos = nullptr;
    return g_accepts;
}

}  // extern "C"
