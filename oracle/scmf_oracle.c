/*
 * CPU oracle for the SCMF polymer Monte Carlo hot path.  TEST INFRASTRUCTURE
 * ONLY: it is the checker the CUDA engine is compared against and never the
 * thing measured or shipped.  See scmf_oracle.h for the reference file:line
 * map.
 *
 * Build with -ffp-contract=off so that no multiply-add is contracted: every
 * fused multiply-add below is an explicit fmaf() call, and the CUDA side uses
 * the same explicit fused operations with --fmad=false.  Division and sqrtf
 * are IEEE correctly rounded on both sides.  Chain and bead indices key the
 * generator, so the storage order of chains does not matter either.
 *
 * Algorithm (one sweep at step s):
 *   for every chain, for colour c = 0 .. n_colours-1, for every bead b of
 *   colour c: a smart-MC (force-biased, Rossky-Doll-Friedman) trial against the
 *   frozen omega field.  The Philox4x32-10 block with counter (chain, b, s, 0)
 *   gives the Gaussian displacement of bead b (words 0..2, one normal each by
 *   a tabulated inverse normal CDF) and its Metropolis uniform (word 3).
 *   Bonded beads never share a colour, so the result does not depend on the
 *   order in which beads of one colour are visited, nor on chain order.
 * The reference instead draws `length` random beads with replacement per chain
 * (device_function.cu:747-751); the odd/even colouring is this engine's update
 * order and is applied identically here and on the GPU.
 */
#include "scmf_oracle.h"
#include "../new_arch_b200/csrc/scmf_normal_table.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAX_TYPES 8
#define ORC_MAX_ARCH 64
#define ORC_MAX_DEG 8
#define ORC_INIT_STEP 0xFFFFFFFFu

/* ------------------------------------------------------------------ math */

static inline uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).  Multipliers and Weyl
 * constants are the published ones. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Uniform in (0, 1] from bits 9..31: 2 - 1.m with the 23 bits as mantissa. */
float orc_u01(uint32_t w) { return 2.0f - u2f(0x3F800000u | (w >> 9)); }

/* Test helper for the kernels' early Metropolis reject: over all 2^23 values
 * orc_u01 yields, counts those whose orc_logf lies below the bound
 * fma((float)bits(u), c1, c0) (a conversion and one fma, as the kernels'
 * log_lower computes it) and returns the smallest margin log - bound in
 * *min_margin. */
long orc_log_lower_violations(float c1, float c0, float* min_margin) {
    long bad = 0;
    float mm = 1e30f;
    for (uint32_t j = 0; j < (1u << 23); ++j) {
        const float u = orc_u01(j << 9);
        const float lo = fmaf((float)f2u(u), c1, c0);
        const float l = orc_logf(u);
        if (!(l >= lo)) ++bad;
        if (l - lo < mm) mm = l - lo;
    }
    *min_margin = mm;
    return bad;
}

/* Natural log for normal positive floats: x = 2^e m, m in [sqrt(1/2), sqrt(2)),
 * log m = log1p(t) = t + t^2 Q(t), t = m - 1 (exact), Q of degree 8 fitted by
 * weighted least squares on Chebyshev nodes (new_arch_b200/csrc/gen_log_poly.py);
 * e ln2 added with a two-part ln2 (12-bit head so that e*head is exact). */
float orc_logf(float x) {
    uint32_t ix = f2u(x);
    int e = (int)(ix >> 23) - 127;
    uint32_t mb = (ix & 0x007FFFFFu) | 0x3F800000u;
    if (mb > 0x3FB504F3u) { mb -= 0x00800000u; e += 1; }
    float t = u2f(mb) - 1.0f;
    float q = -0x1.321a4cp-4f;
    q = fmaf(q, t, 0x1.068b2ap-3f);
    q = fmaf(q, t, -0x1.0f9b0cp-3f);
    q = fmaf(q, t, 0x1.22bf86p-3f);
    q = fmaf(q, t, -0x1.5424e0p-3f);
    q = fmaf(q, t, 0x1.999fc2p-3f);
    q = fmaf(q, t, -0x1.000422p-2f);
    q = fmaf(q, t, 0x1.555558p-2f);
    q = fmaf(q, t, -0x1.fffff8p-2f);
    float lm = fmaf(t * t, q, t);
    float fe = (float)e;
    return fmaf(fe, 0x1.62ep-1f, fmaf(fe, 0x1.0bfbe8p-15f, lm));
}

/* The inverse normal CDF table: 513 cubic segments (c0, c1, c2, c3) of the
 * half-normal quantile h(v) = -Phi^-1(v / 2), written by
 * new_arch_b200/csrc/gen_normal_table.py (data shared with the kernels;
 * tests/test_oracle.py checks it against an independent quantile). */
static const float orc_normal_tab[SCMF_NORMAL_SEGS * 4] = {SCMF_NORMAL_TABLE_DATA};

/* One standard normal from one 32-bit word: bit 31 is the sign, bits 0..30
 * give f = float(2 (w mod 2^31) + 1) (rounded to nearest) in [1, 2^32], and
 * the magnitude is h(f 2^-32) from segment (bits(f) >> 19) - 127*16 (exponent
 * and top four mantissa bits) at t = (1 + m19 2^-23) - (1 + 2^-5), m19 the
 * low 19 mantissa bits (exact), by Horner with fmaf. */
float orc_normal(uint32_t w) {
    const uint32_t b = f2u((float)((w << 1) | 1u));
    const float* c = orc_normal_tab + 4 * (size_t)((b >> 19) - (127u << 4));
    const float t = u2f((b & 0x7FFFFu) | 0x3F800000u) - 1.03125f;
    float z = fmaf(c[3], t, c[2]);
    z = fmaf(z, t, c[1]);
    z = fmaf(z, t, c[0]);
    return u2f(f2u(z) ^ (w & 0x80000000u));
}

/* The three normals of a move: words 0, 1, 2 of its Philox block.  The
 * reference draws them with curand_normal4 (device_function.cu:683-688), its
 * fourth value unused; here the fourth word is the Metropolis word. */
void orc_normals3(const uint32_t w[4], float* n0, float* n1, float* n2) {
    *n0 = orc_normal(w[0]);
    *n1 = orc_normal(w[1]);
    *n2 = orc_normal(w[2]);
}

/* The Metropolis word of a move: word 3 of the same block (orc_u01 reads its
 * bits 9..31). */
uint32_t orc_accept_word(const uint32_t w[4]) { return w[3]; }

/* Periodic fold of one coordinate to a cell index in [0, n): floor(x/dx) mod n
 * (for |x/dx| < 2^22, the range the kernels support).  Restates
 * coord_to_index_unified_high (device_function.cu:313-360): the floor of the
 * exact product x * inv_d of the two FP32 values (exact in FP64), which the
 * kernels read from one round-down fused multiply-add. */
int orc_fold(float x, float inv_d, int n) {
    double t = (double)x * (double)inv_d;
    int i = (int)floor(t);
    if ((unsigned)i >= (unsigned)n) {
        i %= n;
        if (i < 0) i += n;
    }
    return i;
}

/* ---------------------------------------------------------------- system */

typedef struct orc_arch {
    int length, n_chains, n_colors, chain_base;
    int rng_base;       /* random-stream id of the first chain: chain_base, or its id in the whole system (shard) */
    int64_t bead_base;
    float init_sigma;
    int* type;          /* [length] */
    int* deg;           /* [length] */
    int* nbr;           /* [length * ORC_MAX_DEG], ascending */
    int* color;         /* [length] */
} orc_arch;

struct orc_system {
    int n_types, nx, ny, nz;
    double lx, ly, lz;
    double xn[ORC_MAX_TYPES * ORC_MAX_TYPES];
    int nref;
    double kd, ad;
    uint64_t seed;
    int hamiltonian, field_rule;
    int n_arch;
    orc_arch arch[ORC_MAX_ARCH];
    int n_chains;
    int64_t n_beads, n_cells;
    /* derived float constants */
    float k, k2, A, R, inv_dx, inv_dy, inv_dz, scale, flx, fly, flz;
    float cdeg[ORC_MAX_DEG + 1], ac4deg[ORC_MAX_DEG + 1];   /* c = k2 deg, A c / 4 */
    float cf[ORC_MAX_TYPES * ORC_MAX_TYPES];
    /* state */
    float *x, *y, *z;
    uint32_t* counts;
    float* omega;
    uint32_t* chain_acc;
    uint64_t step;
    orc_stats st;
    int finalized;
    /* time-averaged density (io.cpp:57-94) and the displacement reference */
    uint64_t* avg;
    uint32_t avg_every;
    uint64_t avg_samples;
    float *rx, *ry, *rz;
    int fault_no_smc;  /* planted mistake for tests: plain Metropolis on the bond energy */
};

static int g_threads = 1;
void orc_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
int orc_get_threads(void) { return g_threads; }

orc_system* orc_create(int n_types, int nx, int ny, int nz, double lx, double ly, double lz,
                       const double* xn, int nref, double harmonic_normb, double smc_a,
                       uint64_t seed, int hamiltonian, int field_rule) {
    if (n_types < 1 || n_types > ORC_MAX_TYPES || nx < 1 || ny < 1 || nz < 1) return NULL;
    orc_system* s = (orc_system*)calloc(1, sizeof(orc_system));
    s->n_types = n_types; s->nx = nx; s->ny = ny; s->nz = nz;
    s->lx = lx; s->ly = ly; s->lz = lz;
    memcpy(s->xn, xn, sizeof(double) * n_types * n_types);
    s->nref = nref; s->kd = harmonic_normb; s->ad = smc_a; s->seed = seed;
    s->hamiltonian = hamiltonian; s->field_rule = field_rule;
    return s;
}

int orc_add_arch(orc_system* s, int length, int n_chains, const int* mono_type,
                 int n_bonds, const int* bonds, double init_sigma) {
    if (s->finalized || s->n_arch >= ORC_MAX_ARCH || length < 1 || n_chains < 0) return -1;
    orc_arch* a = &s->arch[s->n_arch];
    a->length = length; a->n_chains = n_chains; a->init_sigma = (float)init_sigma;
    a->type = (int*)calloc(length, sizeof(int));
    a->deg = (int*)calloc(length, sizeof(int));
    a->nbr = (int*)calloc((size_t)length * ORC_MAX_DEG, sizeof(int));
    a->color = (int*)calloc(length, sizeof(int));
    for (int i = 0; i < length; ++i) {
        if (mono_type[i] < 0 || mono_type[i] >= s->n_types) return -1;
        a->type[i] = mono_type[i];
    }
    /* adjacency lists in ascending index order, as conection_list is built by
     * scanning the connection matrix (init_config.cu:312-336) */
    char* adj = (char*)calloc((size_t)length * length, 1);
    for (int b = 0; b < n_bonds; ++b) {
        int i = bonds[2 * b], j = bonds[2 * b + 1];
        if (i < 0 || j < 0 || i >= length || j >= length || i == j) { free(adj); return -1; }
        adj[(size_t)i * length + j] = adj[(size_t)j * length + i] = 1;
    }
    for (int i = 0; i < length; ++i)
        for (int j = 0; j < length; ++j)
            if (adj[(size_t)i * length + j]) {
                if (a->deg[i] >= ORC_MAX_DEG) { free(adj); return -1; }
                a->nbr[i * ORC_MAX_DEG + a->deg[i]++] = j;
            }
    free(adj);
    /* greedy colouring in index order: smallest colour unused by lower neighbours */
    a->n_colors = 0;
    for (int i = 0; i < length; ++i) {
        int used = 0;
        for (int d = 0; d < a->deg[i]; ++d) {
            int j = a->nbr[i * ORC_MAX_DEG + d];
            if (j < i) used |= 1 << a->color[j];
        }
        int c = 0;
        while (used & (1 << c)) ++c;
        a->color[i] = c;
        if (c + 1 > a->n_colors) a->n_colors = c + 1;
    }
    s->n_arch++;
    return 0;
}

int orc_finalize(orc_system* s) {
    if (s->finalized) return 0;
    int64_t nb = 0; int nc = 0;
    for (int a = 0; a < s->n_arch; ++a) {
        s->arch[a].bead_base = nb;
        s->arch[a].chain_base = nc;
        s->arch[a].rng_base = nc;
        nb += (int64_t)s->arch[a].length * s->arch[a].n_chains;
        nc += s->arch[a].n_chains;
    }
    s->n_beads = nb; s->n_chains = nc;
    s->n_cells = (int64_t)s->nx * s->ny * s->nz;
    /* derived constants (init_config.cu:480-484, 785, 807-808), rounded to FP32 */
    s->k = (float)s->kd;
    s->k2 = (float)(2.0 * s->kd);
    s->A = (float)s->ad;
    s->R = (float)sqrt(2.0 * s->ad);
    for (int d = 0; d <= ORC_MAX_DEG; ++d) {
        s->cdeg[d] = s->k2 * (float)d;
        s->ac4deg[d] = (s->A * s->cdeg[d]) * 0.25f;
    }
    s->inv_dx = (float)((double)s->nx / s->lx);
    s->inv_dy = (float)((double)s->ny / s->ly);
    s->inv_dz = (float)((double)s->nz / s->lz);
    s->flx = (float)s->lx; s->fly = (float)s->ly; s->flz = (float)s->lz;
    s->scale = nb > 0 ? (float)((double)s->n_cells / (double)nb) : 0.0f;
    double inv_n = 1.0 / (double)s->nref;
    int n = s->n_types;
    for (int t = 0; t < n; ++t)
        for (int u = 0; u < n; ++u) {
            double v = s->xn[t + n * u];
            if (t == u) s->cf[t + n * u] = (float)(v * inv_n);
            else if (s->hamiltonian == 0) s->cf[t + n * u] = (float)(-0.5 * v * inv_n);
            else s->cf[t + n * u] = (float)(v * inv_n);
        }
    s->x = (float*)calloc(nb > 0 ? nb : 1, sizeof(float));
    s->y = (float*)calloc(nb > 0 ? nb : 1, sizeof(float));
    s->z = (float*)calloc(nb > 0 ? nb : 1, sizeof(float));
    s->counts = (uint32_t*)calloc(s->n_cells * n, sizeof(uint32_t));
    s->omega = (float*)calloc(s->n_cells * n, sizeof(float));
    s->chain_acc = (uint32_t*)calloc(nc > 0 ? nc : 1, sizeof(uint32_t));
    s->finalized = 1;
    return 0;
}

void orc_destroy(orc_system* s) {
    if (!s) return;
    for (int a = 0; a < s->n_arch; ++a) {
        free(s->arch[a].type); free(s->arch[a].deg); free(s->arch[a].nbr); free(s->arch[a].color);
    }
    free(s->x); free(s->y); free(s->z); free(s->counts); free(s->omega);
    free(s->chain_acc);
    free(s->avg); free(s->rx); free(s->ry); free(s->rz);
    free(s);
}

int64_t orc_n_beads(const orc_system* s) { return s->n_beads; }
int64_t orc_n_cells(const orc_system* s) { return s->n_cells; }
int orc_n_chains(const orc_system* s) { return s->n_chains; }
void orc_set_step(orc_system* s, uint64_t step) { s->step = step; s->st.step = step; }

void orc_set_coords(orc_system* s, const float* p) {
    for (int64_t i = 0; i < s->n_beads; ++i) { s->x[i] = p[3 * i]; s->y[i] = p[3 * i + 1]; s->z[i] = p[3 * i + 2]; }
}
void orc_get_coords(const orc_system* s, float* p) {
    for (int64_t i = 0; i < s->n_beads; ++i) { p[3 * i] = s->x[i]; p[3 * i + 1] = s->y[i]; p[3 * i + 2] = s->z[i]; }
}
void orc_get_counts(const orc_system* s, uint32_t* out) { memcpy(out, s->counts, sizeof(uint32_t) * s->n_cells * s->n_types); }
void orc_get_omega(const orc_system* s, float* out) { memcpy(out, s->omega, sizeof(float) * s->n_cells * s->n_types); }
void orc_set_omega(orc_system* s, const float* in) { memcpy(s->omega, in, sizeof(float) * s->n_cells * s->n_types); }


static inline void key_of(const orc_system* s, uint32_t key[2]) {
    key[0] = (uint32_t)s->seed; key[1] = (uint32_t)(s->seed >> 32);
}

/* Random-walk chains (device_function.cu:140-207): first bead uniform in the
 * box, then every bead i in index order places each not-yet-placed neighbour
 * at pos[i] + sigma * N(0,1)^3. */
static void init_chain(orc_system* s, const orc_arch* a, int ci, const uint32_t key[2], char* placed) {
    uint32_t gc = (uint32_t)(a->rng_base + ci);
    int64_t b0 = a->bead_base + (int64_t)ci * a->length;
    float* X = s->x + b0; float* Y = s->y + b0; float* Z = s->z + b0;
    uint32_t ctr[4] = {gc, 0u, ORC_INIT_STEP, 0u}, w[4];
    for (int i = 0; i < a->length; ++i) { X[i] = 0.0f; Y[i] = 0.0f; Z[i] = 0.0f; placed[i] = 0; }
    orc_philox4x32_10(ctr, key, w);
    X[0] = orc_u01(w[0]) * s->flx;
    Y[0] = orc_u01(w[1]) * s->fly;
    Z[0] = orc_u01(w[2]) * s->flz;
    placed[0] = 1;
    for (int i = 0; i < a->length; ++i) {
        for (int d = 0; d < a->deg[i]; ++d) {
            int j = a->nbr[i * ORC_MAX_DEG + d];
            if (placed[j]) continue;
            uint32_t c2[4] = {gc, (uint32_t)j, ORC_INIT_STEP, 1u};
            float n0, n1, n2;
            orc_philox4x32_10(c2, key, w);
            orc_normals3(w, &n0, &n1, &n2);
            X[j] = X[i] + a->init_sigma * n0;
            Y[j] = Y[i] + a->init_sigma * n1;
            Z[j] = Z[i] + a->init_sigma * n2;
            placed[j] = 1;
        }
    }
}

void orc_init_coords(orc_system* s) {
    uint32_t key[2]; key_of(s, key);
    for (int a = 0; a < s->n_arch; ++a) {
        const orc_arch* ar = &s->arch[a];
        #pragma omp parallel num_threads(g_threads)
        {
            char* placed = (char*)malloc(ar->length);
            #pragma omp for schedule(static)
            for (int c = 0; c < ar->n_chains; ++c) init_chain(s, ar, c, key, placed);
            free(placed);
        }
    }
}

static inline int64_t cell_of(const orc_system* s, float x, float y, float z) {
    int ix = orc_fold(x, s->inv_dx, s->nx);
    int iy = orc_fold(y, s->inv_dy, s->ny);
    int iz = orc_fold(z, s->inv_dz, s->nz);
    return (int64_t)ix + (int64_t)s->nx * ((int64_t)iy + (int64_t)s->ny * iz);
}

/* Bonded energy change plus smart-MC correction of a trial displacement d of
 * a bead with deg harmonic bonds, transcribed literally from the reference:
 * calc_delta_bonded_energy_arr (device_function.cu:509-561) + the smc_deltaE
 * of trial_move_smc_arr (device_function.cu:700-713), in FP64 like the
 * reference.  Used by the tests to check the closed form below. */
double orc_dE_literal(int deg, const float* q, const float* p, const float* d, double k, double A) {
    double f[3] = {0, 0, 0}, nf[3] = {0, 0, 0}, deb = 0.0;
    for (int j = 0; j < deg; ++j)
        for (int a = 0; a < 3; ++a) f[a] += ((double)q[3 * j + a] - p[a]) * 2.0 * k;
    for (int j = 0; j < deg; ++j) {
        double o2 = 0, e2 = 0;
        for (int a = 0; a < 3; ++a) {
            double o = (double)p[a] - q[3 * j + a], e = o + d[a];
            o2 += o * o;
            e2 += e * e;
            nf[a] += ((double)q[3 * j + a] - ((double)p[a] + d[a])) * 2.0 * k;
        }
        deb += k * (e2 - o2);
    }
    double smc = 0.5 * ((nf[0] + f[0]) * d[0] + (nf[1] + f[1]) * d[1] + (nf[2] + f[2]) * d[2]);
    smc += 0.25 * A * (nf[0] * nf[0] + nf[1] * nf[1] + nf[2] * nf[2] - f[0] * f[0] - f[1] * f[1] - f[2] * f[2]);
    return deb + smc;
}

/* The same quantity in closed form.  With f = 2k sum_j (q_j - p) the force at
 * p, the force at p + d is f - c d (c = 2k deg), and the bonded change plus the
 * smart-MC term reduce exactly to (A c / 4) (c |d|^2 - 2 f.d).  This is what
 * both the oracle and the kernels evaluate, in FP32 with explicit fmaf. */
static inline float dE_closed(float c, float ac4, float fx, float fy, float fz, float dx, float dy, float dz) {
    float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    float fd = fmaf(fx, dx, fmaf(fy, dy, fz * dz));
    return ac4 * fmaf(c, d2, -2.0f * fd);
}

float orc_dE_closed(int deg, const float* q, const float* p, const float* d, float k2, float A) {
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    for (int j = 0; j < deg; ++j) {
        fx = fmaf(q[3 * j] - p[0], k2, fx);
        fy = fmaf(q[3 * j + 1] - p[1], k2, fy);
        fz = fmaf(q[3 * j + 2] - p[2], k2, fz);
    }
    float c = k2 * (float)deg;
    return dE_closed(c, (A * c) * 0.25f, fx, fy, fz, d[0], d[1], d[2]);
}

/* The energy change of one smart-MC trial of bead b (device_function.cu:637-717,
 * 562-588) with the Gaussian triple (n0, n1, n2): force from the bonded
 * neighbours (ascending order), displacement d = A f + R xi, proposed position
 * (*px, *py, *pz), and omega[new cell] - omega[old cell] + the closed form
 * above. */
static inline float trial_energy(const orc_system* s, const orc_arch* a, int b, const float* X, const float* Y,
                                 const float* Z, float n0, float n1, float n2, float* px, float* py, float* pz) {
    const int* nb = a->nbr + b * ORC_MAX_DEG;
    const int deg = a->deg[b];
    const float k2 = s->k2, A = s->A, R = s->R;
    const float x = X[b], y = Y[b], z = Z[b];
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    for (int d = 0; d < deg; ++d) {
        int j = nb[d];
        fx = fmaf(X[j] - x, k2, fx);
        fy = fmaf(Y[j] - y, k2, fy);
        fz = fmaf(Z[j] - z, k2, fz);
    }
    const float dx = fmaf(A, fx, R * n0);
    const float dy = fmaf(A, fy, R * n1);
    const float dz = fmaf(A, fz, R * n2);
    *px = x + dx;
    *py = y + dy;
    *pz = z + dz;
    const float c = s->cdeg[deg], ac4 = s->ac4deg[deg];
    const int t = a->type[b];
    const float* W = s->omega + (int64_t)t * s->n_cells;
    const float w_old = W[cell_of(s, x, y, z)];
    const float w_new = W[cell_of(s, *px, *py, *pz)];
    float eb;
    if (s->fault_no_smc) {  /* the bond energy change alone, (c/2)|d|^2 - f.d, without the smart-MC correction */
        const float d2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        const float fd = fmaf(fx, dx, fmaf(fy, dy, fz * dz));
        eb = fmaf(0.5f * c, d2, -fd);
    } else {
        eb = dE_closed(c, ac4, fx, fy, fz, dx, dy, dz);
    }
    return (w_new - w_old) + eb;
}

/* One smart-MC trial of bead b (device_function.cu:637-717, 562-588, 444-454)
 * with the Gaussian triple (n0, n1, n2) and the Metropolis word aw.  Returns 1
 * if accepted (the bead then sits at the proposed position). */
static inline int move_bead(const orc_system* s, const orc_arch* a, int b, float* X, float* Y, float* Z,
                            float n0, float n1, float n2, uint32_t aw) {
    float px, py, pz;
    const float dE = trial_energy(s, a, b, X, Y, Z, n0, n1, n2, &px, &py, &pz);
    /* Metropolis: accept if dE < 0, else if log(u) < -dE.  log(u) >= -23 ln2
     * > -17 for every u the generator yields, so dE >= 17 always rejects. */
    int acc;
    if (dE < 0.0f) acc = 1;
    else if (dE < 17.0f) acc = orc_logf(orc_u01(aw)) < -dE;
    else acc = 0;
    if (acc) { X[b] = px; Y[b] = py; Z[b] = pz; }
    return acc;
}

/* trial_energy() of bead b of a chain of architecture `arch` whose positions
 * are the chain-local arrays X, Y, Z; p_out receives the proposed position.
 * For the checks against the reference's own trial functions. */
float orc_trial_energy(const orc_system* s, int arch, int b, const float* X, const float* Y, const float* Z, float n0,
                       float n1, float n2, float* p_out) {
    const orc_arch* a = &s->arch[arch];
    return trial_energy(s, a, b, X, Y, Z, n0, n1, n2, p_out, p_out + 1, p_out + 2);
}

/* One trial of bead b: its Philox block (chain, b, step, 0) gives the three
 * normals and the Metropolis word. */
static inline int move_single(const orc_system* s, const orc_arch* a, uint32_t gc, int b,
                              float* X, float* Y, float* Z, const uint32_t key[2], uint32_t step) {
    uint32_t ctr[4] = {gc, (uint32_t)b, step, 0u}, w[4];
    orc_philox4x32_10(ctr, key, w);
    float n0, n1, n2;
    orc_normals3(w, &n0, &n1, &n2);
    return move_bead(s, a, b, X, Y, Z, n0, n1, n2, orc_accept_word(w));
}

/* Bond energy of one chain, each bond once: sum k |r_i - r_j|^2. */
static double chain_bond_energy(const orc_system* s, const orc_arch* a, const float* X, const float* Y, const float* Z) {
    double e = 0.0;
    for (int i = 0; i < a->length; ++i)
        for (int d = 0; d < a->deg[i]; ++d) {
            int j = a->nbr[i * ORC_MAX_DEG + d];
            if (j <= i) continue;
            float ex = X[i] - X[j], ey = Y[i] - Y[j], ez = Z[i] - Z[j];
            e += (double)s->k * (double)(ex * ex + ey * ey + ez * ez);
        }
    return e;
}

static void sweep_moves(orc_system* s, uint32_t step) {
    uint32_t key[2]; key_of(s, key);
    for (int a = 0; a < s->n_arch; ++a) {
        const orc_arch* ar = &s->arch[a];
        #pragma omp parallel for schedule(static) num_threads(g_threads)
        for (int c = 0; c < ar->n_chains; ++c) {
            int64_t b0 = ar->bead_base + (int64_t)c * ar->length;
            float* X = s->x + b0; float* Y = s->y + b0; float* Z = s->z + b0;
            uint32_t gc = (uint32_t)(ar->rng_base + c);
            uint32_t nacc = 0;
            for (int col = 0; col < ar->n_colors; ++col)
                for (int b = 0; b < ar->length; ++b)
                    if (ar->color[b] == col) nacc += (uint32_t)move_single(s, ar, gc, b, X, Y, Z, key, step);
            s->chain_acc[ar->chain_base + c] = nacc;
        }
    }
    uint64_t acc = 0;
    for (int c = 0; c < s->n_chains; ++c) acc += s->chain_acc[c];
    s->st.last_accepts = acc;
    s->st.total_accepts += acc;
    s->st.total_moves += (uint64_t)s->n_beads;
}

void orc_smc_move(orc_system* s, int n) {
    for (int i = 0; i < n; ++i) {
        s->step += 1;
        sweep_moves(s, (uint32_t)s->step);
    }
}

/* Integer per-type cell counts (device_function.cu:471-508). */
void orc_reset_density(orc_system* s) {
    const int64_t nc = s->n_cells;
    memset(s->counts, 0, sizeof(uint32_t) * nc * s->n_types);
    for (int a = 0; a < s->n_arch; ++a) {
        const orc_arch* ar = &s->arch[a];
        #pragma omp parallel for schedule(static) num_threads(g_threads)
        for (int c = 0; c < ar->n_chains; ++c) {
            int64_t b0 = ar->bead_base + (int64_t)c * ar->length;
            for (int b = 0; b < ar->length; ++b) {
                int64_t cell = cell_of(s, s->x[b0 + b], s->y[b0 + b], s->z[b0 + b]);
                uint32_t* slot = &s->counts[(int64_t)ar->type[b] * nc + cell];
                if (g_threads > 1) __atomic_fetch_add(slot, 1u, __ATOMIC_RELAXED);
                else *slot += 1u;
            }
        }
    }
}

/* SCMF0 field (device_function.cu:373-412) in FP32, or the literal
 * omega_T = kappaN (sum phi - 1) + sum_{S!=T} chiN_TS phi_S per 1/N_ref
 * when hamiltonian == 1. */
static void field_update_from(orc_system* s, const uint32_t* counts, int write_omega) {
    const int n = s->n_types;
    const int64_t nc = s->n_cells;
    double ef = 0.0;
    #pragma omp parallel for schedule(static) reduction(+:ef) num_threads(g_threads)
    for (int64_t c = 0; c < nc; ++c) {
        float phi[ORC_MAX_TYPES];
        float tot = 0.0f;
        for (int u = 0; u < n; ++u) { phi[u] = (float)counts[u * nc + c] * s->scale; tot = tot + phi[u]; }
        for (int t = 0; t < n; ++t) {
            float w;
            if (write_omega) {
                w = (tot - 1.0f) * s->cf[t + n * t];
                for (int u = 0; u < n; ++u) {
                    if (u == t) continue;
                    if (s->hamiltonian == 0) w = w + s->cf[t + n * u] * (phi[t] - phi[u]);
                    else w = w + s->cf[t + n * u] * phi[u];
                }
                s->omega[t * nc + c] = w;
            } else {
                w = s->omega[t * nc + c];
            }
            ef += (double)w * (double)counts[t * nc + c];
        }
    }
    s->st.e_field = ef;
}

static void field_update(orc_system* s, int write_omega) { field_update_from(s, s->counts, write_omega); }

void orc_update_omega(orc_system* s) { field_update(s, 1); }

/* Chain shard of a system (the reference's per-GPU chains, init_config.cu:220-222):
 * rng_base[a] is the whole-system id of this system's first chain of
 * architecture a, and the field scaling uses the whole system's bead count. */
void orc_set_shard(orc_system* s, const int* rng_base, int64_t n_beads_total) {
    for (int a = 0; a < s->n_arch; ++a) s->arch[a].rng_base = rng_base[a];
    s->scale = n_beads_total > 0 ? (float)((double)s->n_cells / (double)n_beads_total) : 0.0f;
}

/* omega and the field energy of the given counts (the sum over all shards). */
void orc_field_from(orc_system* s, const uint32_t* counts) { field_update_from(s, counts, 1); }

/* One MC step per sweep, test.cpp:37-43: move, grid, then the field unless
 * the rule is "reference" and step % 10 == 0. */
void orc_step(orc_system* s, int n) {
    for (int i = 0; i < n; ++i) {
        s->step += 1;
        sweep_moves(s, (uint32_t)s->step);
        orc_reset_density(s);
        int upd = (s->field_rule == 1) || (s->step % 10 != 0);
        field_update(s, upd);
        if (s->avg && s->step % s->avg_every == 0) orc_average_sample(s);
    }
}

/* Time-averaged density: the counts of the final positions of every sweep s
 * with s % every == 0 are summed (average_field_unified, struct.h:234). */
void orc_set_fault(orc_system* s, int no_smc) { s->fault_no_smc = no_smc; }

void orc_average_start(orc_system* s, uint32_t every) {
    free(s->avg);
    s->avg = NULL;
    s->avg_every = every;
    s->avg_samples = 0;
    if (every) s->avg = (uint64_t*)calloc((size_t)(s->n_cells * s->n_types), sizeof(uint64_t));
}

void orc_average_sample(orc_system* s) {
    if (!s->avg) return;
    const int64_t n = s->n_cells * s->n_types;
    for (int64_t i = 0; i < n; ++i) s->avg[i] += s->counts[i];
    s->avg_samples += 1;
}

uint64_t orc_average_get(const orc_system* s, uint64_t* sums) {
    if (!s->avg) return 0;
    memcpy(sums, s->avg, sizeof(uint64_t) * (size_t)(s->n_cells * s->n_types));
    return s->avg_samples;
}

/* Chain observables in double.  R_e = last bead - first bead (test.cpp:47-68
 * uses beads 0 and 31); R_g^2 = mean |r - r_cm|^2 per chain; bonds once
 * (j > i); bead and centre-of-mass displacements from the reference
 * snapshot.  out[15] = means of re2 xyz, rg2 xyz, bond2 xyz (per bond),
 * msd xyz (per bead), msd_com xyz (per chain); NaN where undefined. */
void orc_analysis_reference(orc_system* s) {
    size_t nb = (size_t)s->n_beads;
    if (!s->rx) {
        s->rx = (float*)malloc(nb * sizeof(float));
        s->ry = (float*)malloc(nb * sizeof(float));
        s->rz = (float*)malloc(nb * sizeof(float));
    }
    memcpy(s->rx, s->x, nb * sizeof(float));
    memcpy(s->ry, s->y, nb * sizeof(float));
    memcpy(s->rz, s->z, nb * sizeof(float));
}

int orc_analyze(const orc_system* s, int arch, double* out) {
    if (arch < 0 || arch >= s->n_arch) return -1;
    const orc_arch* a = &s->arch[arch];
    const int L = a->length;
    double acc[15] = {0};
    int64_t n_bonds = 0;
    for (int c = 0; c < a->n_chains; ++c) {
        const int64_t b0 = a->bead_base + (int64_t)c * L;
        const float *X = s->x + b0, *Y = s->y + b0, *Z = s->z + b0;
        double cx = 0, cy = 0, cz = 0, rcx = 0, rcy = 0, rcz = 0;
        for (int b = 0; b < L; ++b) { cx += X[b]; cy += Y[b]; cz += Z[b]; }
        cx /= L; cy /= L; cz /= L;
        double gx = 0, gy = 0, gz = 0;
        for (int b = 0; b < L; ++b) {
            double ux = (double)X[b] - cx, uy = (double)Y[b] - cy, uz = (double)Z[b] - cz;
            gx += ux * ux; gy += uy * uy; gz += uz * uz;
        }
        double ex = (double)X[L - 1] - (double)X[0], ey = (double)Y[L - 1] - (double)Y[0], ez = (double)Z[L - 1] - (double)Z[0];
        acc[0] += ex * ex; acc[1] += ey * ey; acc[2] += ez * ez;
        acc[3] += gx / L; acc[4] += gy / L; acc[5] += gz / L;
        for (int b = 0; b < L; ++b)
            for (int d = 0; d < a->deg[b]; ++d) {
                int j = a->nbr[b * ORC_MAX_DEG + d];
                if (j <= b) continue;
                double bx = (double)X[j] - (double)X[b], by = (double)Y[j] - (double)Y[b], bz = (double)Z[j] - (double)Z[b];
                acc[6] += bx * bx; acc[7] += by * by; acc[8] += bz * bz;
                if (c == 0) n_bonds += 1;
            }
        if (s->rx) {
            for (int b = 0; b < L; ++b) {
                double ux = (double)X[b] - (double)s->rx[b0 + b], uy = (double)Y[b] - (double)s->ry[b0 + b],
                       uz = (double)Z[b] - (double)s->rz[b0 + b];
                acc[9] += ux * ux; acc[10] += uy * uy; acc[11] += uz * uz;
                rcx += s->rx[b0 + b]; rcy += s->ry[b0 + b]; rcz += s->rz[b0 + b];
            }
            double dx = cx - rcx / L, dy = cy - rcy / L, dz = cz - rcz / L;
            acc[12] += dx * dx; acc[13] += dy * dy; acc[14] += dz * dz;
        }
    }
    const double nan = 0.0 / 0.0;
    const double nc = a->n_chains ? (double)a->n_chains : nan;
    const double nbd = n_bonds ? (double)n_bonds * a->n_chains : nan;
    const double nbe = a->n_chains ? (double)a->n_chains * L : nan;
    for (int k = 0; k < 3; ++k) {
        out[k] = acc[k] / nc;
        out[3 + k] = acc[3 + k] / nc;
        out[6 + k] = acc[6 + k] / nbd;
        out[9 + k] = s->rx ? acc[9 + k] / nbe : nan;
        out[12 + k] = s->rx ? acc[12 + k] / nc : nan;
    }
    return 0;
}

/* Statistics; the bond energy is that of the current positions, computed on
 * demand (as the engine does). */
void orc_get_stats(const orc_system* s, orc_stats* out) {
    *out = s->st;
    out->step = s->step;
    double eb = 0.0;
    for (int a = 0; a < s->n_arch; ++a) {
        const orc_arch* ar = &s->arch[a];
        for (int c = 0; c < ar->n_chains; ++c) {
            int64_t b0 = ar->bead_base + (int64_t)c * ar->length;
            eb += chain_bond_energy(s, ar, s->x + b0, s->y + b0, s->z + b0);
        }
    }
    out->e_bond = eb;
}
