/*
 * CPU oracle for the SCMF polymer Monte Carlo hot path (move -> grid -> field).
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker: a single-threaded C
 * restatement of the reference algorithm (plus an OpenMP twin that must give
 * bit-identical positions and counts).  Only the tests, the smoke check and the
 * CPU-baseline leg of the benchmark may load it; the product library never
 * links or calls it.
 *
 * Parity pins (see tests/test_oracle_*.py): Philox4x32-10 known-answer
 * vectors (Salmon et al., SC'11), the reference's density-file format and
 * integer invariants, its per-type mean omega, and the byte-exact VTK
 * converter output.  Trajectories of the reference itself are not
 * reproducible (time(NULL) seed, cuRAND stream), so beyond those pins the
 * oracle restates the algorithm and is the contract.
 *
 * Algorithm sources in the reference (ren5885a/New_arch):
 *   move   device_function.cu:444-454 (accept), 509-588 (dE), 589-717 (SMC trial), 718-799 (kernel)
 *   cell   device_function.cu:313-360 (periodic fold)
 *   grid   device_function.cu:479-508
 *   field  device_function.cu:373-412 (SCMF0)
 *   init   device_function.cu:140-207 (random-walk chains)
 *   consts init_config.cu:480-484 (harmonic_normb), 785 (field scaling), 807-808 (A, R)
 *   steps  test.cpp:37-43 (field skipped when step % 10 == 0)
 */
#ifndef SCMF_ORACLE_H
#define SCMF_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_system orc_system;

typedef struct orc_stats {
    uint64_t step;            /* completed sweeps */
    uint64_t last_accepts;    /* accepted moves in the last sweep */
    uint64_t total_accepts;
    uint64_t total_moves;
    double e_bond;            /* sum over bonds k |r_i - r_j|^2 after the last sweep */
    double e_field;           /* sum_T sum_c omega_T(c) n_T(c) after the last field step */
} orc_stats;

orc_system* orc_create(int n_types, int nx, int ny, int nz, double lx, double ly, double lz,
                       const double* xn, int nref, double harmonic_normb, double smc_a,
                       uint64_t seed, int hamiltonian, int field_rule);
int  orc_add_arch(orc_system* s, int length, int n_chains, const int* mono_type,
                  int n_bonds, const int* bonds, double init_sigma);
int  orc_finalize(orc_system* s);
void orc_destroy(orc_system* s);

void orc_set_threads(int n);
int  orc_get_threads(void);

int64_t orc_n_beads(const orc_system* s);
int64_t orc_n_cells(const orc_system* s);
int     orc_n_chains(const orc_system* s);

void orc_init_coords(orc_system* s);
void orc_set_coords(orc_system* s, const float* xyz_aos);
void orc_get_coords(const orc_system* s, float* xyz_aos);
void orc_set_step(orc_system* s, uint64_t step);

void orc_smc_move(orc_system* s, int n_sweeps);   /* move only, like smc_move() */
void orc_reset_density(orc_system* s);            /* grid, like reset_density_fields() */
void orc_update_omega(orc_system* s);             /* field, like update_omega_fields_scmf0() */
void orc_step(orc_system* s, int n_sweeps);       /* one full MC step per sweep, field rule applied */

void orc_get_counts(const orc_system* s, uint32_t* out);
void orc_get_omega(const orc_system* s, float* out);
void orc_set_omega(orc_system* s, const float* in);
void orc_get_stats(const orc_system* s, orc_stats* out);

/* time-averaged density: orc_step adds the counts of every sweep s with
 * s % every == 0 (every = 0 stops); orc_average_get returns the sample count */
void     orc_average_start(orc_system* s, uint32_t every);
void     orc_average_sample(orc_system* s);
uint64_t orc_average_get(const orc_system* s, uint64_t* sums);

/* chain observables (means in double): out[15] = re2 xyz, rg2 xyz, bond2 xyz,
 * msd xyz, msd_com xyz; displacements are NaN before orc_analysis_reference */
/* Plants a known mistake (tests of the tests only): no_smc = 1 accepts moves
 * by plain Metropolis on the bond energy, dropping the smart-MC correction. */
void orc_set_fault(orc_system* s, int no_smc);

void orc_analysis_reference(orc_system* s);
int  orc_analyze(const orc_system* s, int arch, double* out);

/* math building blocks (exported for known-answer tests) */
void  orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
float orc_logf(float x);
long orc_log_lower_violations(float c1, float c0, float* min_margin);
float orc_normal(uint32_t w);   /* one standard normal from one word (inverse CDF) */
void  orc_normals3(const uint32_t w[4], float* n0, float* n1, float* n2);
float orc_u01(uint32_t w);
uint32_t orc_accept_word(const uint32_t w[4]);
int   orc_fold(float x, float inv_d, int n);
double orc_dE_literal(int deg, const float* q, const float* p, const float* d, double k, double A);
float  orc_dE_closed(int deg, const float* q, const float* p, const float* d, float k2, float A);
/* energy change of one trial of bead b of a chain of architecture `arch`
 * (chain-local positions X, Y, Z) with the normals n0..n2; p_out[3] gets the
 * proposed position */
/* chain shard: per-architecture random-stream bases and the whole system's bead count */
void   orc_set_shard(orc_system* s, const int* rng_base, int64_t n_beads_total);
/* omega (and field energy) of the given counts instead of the system's own */
void   orc_field_from(orc_system* s, const uint32_t* counts);
float  orc_trial_energy(const orc_system* s, int arch, int b, const float* X, const float* Y, const float* Z, float n0,
                        float n1, float n2, float* p_out);

#ifdef __cplusplus
}
#endif
#endif
