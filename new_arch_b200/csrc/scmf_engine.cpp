// Host engine of libscmf: specs, systems, work plans, the plain and batched
// step loops, and the C ABI entry points of include/scmf.h except file I/O
// (scmf_files.cpp) and serving (scmf_server.cpp).
//
// The reference's host orchestration (smc.cu:3-72, mesh.cu:161-248,
// mesh_mpi.cpp:4-27, test.cpp:37-43) launches one kernel at a time with a
// cudaDeviceSynchronize after each and a P2P/MPI density reduction.  Here a
// sweep is two launches on one stream (fused move+grid, then field) with no
// host round trip, optionally replayed from a CUDA graph; the step counter,
// the counts double buffer and the statistics live on the device.
#include "scmf_engine.h"

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <mutex>

namespace scmf {

static thread_local std::string g_last_error;

scmf_status fail(scmf_status code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

void clear_error() { g_last_error.clear(); }
const char* last_error_cstr() { return g_last_error.c_str(); }

#define CK(expr)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (expr);                                                                   \
        if (e_ != cudaSuccess) return fail(SCMF_E_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)

#define CKL(expr)                                                                                      \
    do {                                                                                               \
        int e_ = (expr);                                                                               \
        if (e_ != 0)                                                                                   \
            return fail(SCMF_E_CUDA, "%s: %s", #expr, cudaGetErrorString((cudaError_t)e_));          \
    } while (0)

scmf_status dev_alloc(void** p, size_t bytes, cudaStream_t st) {
    static std::once_flag once;
    std::call_once(once, [] {
        int dev = 0;
        cudaMemPool_t pool;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        cudaGetLastError();
    });
    bytes = (std::max<size_t>(bytes, 16) + 255) / 256 * 256;
    cudaError_t e = cudaMallocAsync(p, bytes, st);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? SCMF_E_NOMEM : SCMF_E_CUDA, "cudaMallocAsync(%zu): %s", bytes,
                    cudaGetErrorString(e));
    }
    return SCMF_OK;
}

void dev_free(void* p, cudaStream_t st) {
    if (p) cudaFreeAsync(p, st);
}

// ceil(2^32 / n): for i * n < 2^32, i / n == umulhi(i, magic).  n == 1 has no
// 32-bit magic; the kernels test for it.
uint32_t magic_for(uint32_t n) {
    if (n <= 1) return 0u;
    return (uint32_t)((((uint64_t)1 << 32) + n - 1) / n);
}

scmf_status validate_spec(const scmf_spec& s) {
    if (s.n_types < 1 || s.n_types > kMaxTypes) return fail(SCMF_E_INVALID, "n_mono_types %d not in [1,%d]", s.n_types, kMaxTypes);
    if (s.nx < 1 || s.ny < 1 || s.nz < 1) return fail(SCMF_E_INVALID, "grid %d x %d x %d invalid", s.nx, s.ny, s.nz);
    if ((int64_t)s.nx * s.ny * s.nz > ((int64_t)1 << 30)) return fail(SCMF_E_INVALID, "grid too large");
    // the FP32 cell fold is exact while |x / dx| < 2^22: keep whole boxes well inside that
    if (s.nx > (1 << 20) || s.ny > (1 << 20) || s.nz > (1 << 20))
        return fail(SCMF_E_INVALID, "grid axis longer than %d cells", 1 << 20);
    if (!(s.lx > 0 && s.ly > 0 && s.lz > 0)) return fail(SCMF_E_INVALID, "box lengths must be positive");
    if ((int)s.xn.size() != s.n_types * s.n_types) return fail(SCMF_E_INVALID, "xn matrix not set");
    if (s.p.reference_nbeads < 1) return fail(SCMF_E_INVALID, "reference_nbeads must be >= 1");
    if (!(s.p.smc_a >= 0) || !std::isfinite(s.p.harmonic_normb)) return fail(SCMF_E_INVALID, "bad smc_a / harmonic_normb");
    if (s.p.count_bits != 16 && s.p.count_bits != 32) return fail(SCMF_E_INVALID, "count_bits must be 16 or 32");
    if (s.p.hamiltonian != SCMF_HAM_SCMF0 && s.p.hamiltonian != SCMF_HAM_LITERAL) return fail(SCMF_E_INVALID, "unknown hamiltonian");
    if (s.p.field_rule != SCMF_FIELD_REFERENCE && s.p.field_rule != SCMF_FIELD_EVERY) return fail(SCMF_E_INVALID, "unknown field rule");
    if (s.archs.empty()) return fail(SCMF_E_INVALID, "spec has no polymer architecture");
    int64_t beads = 0, chains = 0;
    for (const auto& a : s.archs) {
        if (a.length < 1 || a.length > kMaxLength) return fail(SCMF_E_INVALID, "chain length %d not in [1,%d]", a.length, kMaxLength);
        if (a.n_chains < 0) return fail(SCMF_E_INVALID, "negative chain count %d", a.n_chains);
        beads += (int64_t)a.length * a.n_chains;
        chains += a.n_chains;
    }
    if (beads <= 0) return fail(SCMF_E_INVALID, "system has no beads");
    if (beads >= ((int64_t)1 << 31) || chains >= ((int64_t)1 << 31)) return fail(SCMF_E_INVALID, "too many beads");
    if (s.p.count_bits == 16 && beads >= 65536)
        return fail(SCMF_E_INVALID, "16-bit counts need fewer than 65536 beads (%lld)", (long long)beads);
    return SCMF_OK;
}

scmf_status prepare_archs(const scmf_spec& s, std::vector<ArchHost>* out, int64_t* n_beads, int* n_chains) {
    out->clear();
    int64_t nb = 0;
    int nc = 0;
    for (const auto& a : s.archs) {
        ArchHost h;
        h.length = a.length;
        h.n_chains = a.n_chains;
        h.chain_base = nc;
        h.bead_base = nb;
        h.init_sigma = (float)(a.init_sigma > 0 ? a.init_sigma : (a.length > 1 ? 1.0 / std::sqrt(3.0 * (a.length - 1.0)) : 0.0));
        const int L = a.length;
        h.beads.assign(L, BeadInfo{});
        std::vector<std::vector<char>> adj(L, std::vector<char>(L, 0));
        for (size_t b = 0; b + 1 < a.bonds.size(); b += 2) {
            int i = a.bonds[b], j = a.bonds[b + 1];
            if (i < 0 || j < 0 || i >= L || j >= L || i == j) return fail(SCMF_E_INVALID, "bond (%d,%d) out of range", i, j);
            adj[i][j] = adj[j][i] = 1;
        }
        for (int i = 0; i < L; ++i) {
            if (a.type[i] < 0 || a.type[i] >= s.n_types) return fail(SCMF_E_INVALID, "monomer type %d out of range", a.type[i]);
            BeadInfo& bi = h.beads[i];
            bi.type = (uint8_t)a.type[i];
            int d = 0;
            for (int j = 0; j < L; ++j)
                if (adj[i][j]) {
                    if (d >= kMaxDeg) return fail(SCMF_E_INVALID, "bead %d has more than %d bonds", i, kMaxDeg);
                    bi.nbr[d++] = (uint16_t)j;
                }
            bi.deg = (uint8_t)d;
            h.max_deg = std::max(h.max_deg, d);
        }
        // greedy colouring in index order
        int ncol = 0;
        for (int i = 0; i < L; ++i) {
            unsigned used = 0;
            for (int d = 0; d < h.beads[i].deg; ++d) {
                int j = h.beads[i].nbr[d];
                if (j < i) used |= 1u << h.beads[j].color;
            }
            int c = 0;
            while (used & (1u << c)) ++c;
            if (c >= kMaxColors) return fail(SCMF_E_INVALID, "architecture needs more than %d colours", kMaxColors);
            h.beads[i].color = (uint8_t)c;
            ncol = std::max(ncol, c + 1);
        }
        h.n_colors = ncol;
        h.linear = true;
        for (int i = 0; i < L && h.linear; ++i) {
            const BeadInfo& bi = h.beads[i];
            const int want = (i > 0) + (i + 1 < L);
            if (bi.deg != want || bi.color != (i & 1)) h.linear = false;
            if (bi.deg >= 1 && i > 0 && bi.nbr[0] != i - 1) h.linear = false;
            if (i + 1 < L && bi.nbr[bi.deg - 1] != i + 1) h.linear = false;
        }
        h.color_beads.clear();
        for (int c = 0; c < ncol; ++c) {
            h.color_off[c] = (int)h.color_beads.size();
            for (int i = 0; i < L; ++i)
                if (h.beads[i].color == c) h.color_beads.push_back((uint16_t)i);
        }
        h.color_off[ncol] = (int)h.color_beads.size();
        nb += (int64_t)L * a.n_chains;
        nc += a.n_chains;
        out->push_back(std::move(h));
    }
    *n_beads = nb;
    *n_chains = nc;
    return SCMF_OK;
}

static size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

static size_t count_words(const scmf_spec& s) {
    const size_t cells = (size_t)s.nx * s.ny * s.nz * s.n_types;
    return s.p.count_bits == 16 ? (cells + 1) / 2 : cells;
}

size_t system_device_bytes(const scmf_spec& s) {
    int64_t beads = 0, chains = 0, arch_bytes = 0;
    for (const auto& a : s.archs) {
        beads += (int64_t)a.length * a.n_chains;
        chains += a.n_chains;
        arch_bytes += round_up((size_t)a.length * (sizeof(BeadInfo) + 3) + 16, 256);
    }
    const size_t cells = (size_t)s.nx * s.ny * s.nz * s.n_types;
    size_t b = 3 * round_up((size_t)(beads + 4) * 4, 256) + round_up((size_t)chains * 4, 256);
    b += 2 * round_up(count_words(s) * 4, 256) + round_up(cells * 4, 256);
    b += round_up(sizeof(SysDev), 256) + round_up(s.archs.size() * sizeof(ArchDev), 256) + arch_bytes;
    b += (size_t)chains / 8 * sizeof(MoveTile) + 64 * 1024;  // work lists
    return b;
}

void field_coefficients(int n, const double* xn, int nref, int hamiltonian, float* cf) {
    const double inv_n = 1.0 / (double)nref;
    for (int i = 0; i < kMaxTypes * kMaxTypes; ++i) cf[i] = 0.0f;
    for (int t = 0; t < n; ++t)
        for (int u = 0; u < n; ++u) {
            const double v = xn[t + n * u];
            float c;
            if (t == u) c = (float)(v * inv_n);
            else if (hamiltonian == SCMF_HAM_SCMF0) c = (float)(-0.5 * v * inv_n);
            else c = (float)(v * inv_n);
            cf[t + n * u] = c;
        }
}

// 0: every axis a power of two (the move kernels may compile only the mask
// fold), 1: some axis is not.
int flat_threads_for(int tpc, int threads_move) {
    // lcm(tpc, 32): a block of that many threads holds whole chains with no idle lane
    int a = tpc, b = 32;
    while (b) {
        const int r = a % b;
        a = b;
        b = r;
    }
    const int l = tpc / a * 32;
    return l <= 256 ? l : std::max(32, threads_move);
}

int fold_kind_of(const scmf_spec& s) {
    const int dims[3] = {s.nx, s.ny, s.nz};
    bool pow2 = true;
    for (int n : dims) pow2 = pow2 && (n & (n - 1)) == 0;
    return pow2 ? 0 : 1;
}

void fill_sysdev_constants(const scmf_spec& s, int64_t n_beads, SysDev* d) {
    d->stop_step = 0xFFFFFFFFu;
    d->om_max_key = 0u;            // identities of the running max / min
    d->om_min_key = 0xFFFFFFFFu;
    d->omega_span = INFINITY;      // no bound until a field step computes one
    d->n_types = s.n_types;
    d->nx = s.nx; d->ny = s.ny; d->nz = s.nz;
    d->n_cells = (int64_t)s.nx * s.ny * s.nz;
    d->n_beads = n_beads;
    // derived constants (init_config.cu:480-484, 565-567, 785, 807-808) rounded to FP32
    d->inv_dx = (float)((double)s.nx / s.lx);
    d->inv_dy = (float)((double)s.ny / s.ly);
    d->inv_dz = (float)((double)s.nz / s.lz);
    d->lx = (float)s.lx; d->ly = (float)s.ly; d->lz = (float)s.lz;
    d->scale = (float)((double)d->n_cells / (double)n_beads);
    d->k = (float)s.p.harmonic_normb;
    d->k2 = (float)(2.0 * s.p.harmonic_normb);
    d->A = (float)s.p.smc_a;
    d->R = (float)std::sqrt(2.0 * s.p.smc_a);
    for (int g = 0; g <= kMaxDeg; ++g) {
        d->cdeg[g] = d->k2 * (float)g;
        d->ac4deg[g] = (d->A * d->cdeg[g]) * 0.25f;
    }
    field_coefficients(s.n_types, s.xn.data(), s.p.reference_nbeads, s.p.hamiltonian, d->cf);
    d->hamiltonian = s.p.hamiltonian;
    d->field_rule = s.p.field_rule;
    d->count16 = s.p.count_bits == 16 ? 1 : 0;
    d->n_arch = (int)s.archs.size();
    d->seed_lo = (uint32_t)s.p.seed;
    d->seed_hi = (uint32_t)(s.p.seed >> 32);
}

scmf_tune default_tune() {
    scmf_tune t{};
    t.chains_per_tile = 0;
    t.threads_move = 128;  // 4 warps: CTAs retire and refill at a finer grain than 8-warp CTAs
    t.cells_per_tile = 0;
    t.threads_field = 256;
    t.persistent_ctas = 0;
    t.use_graph = 1;
    return t;
}

scmf_tune resolve_tune(const scmf_tune* t) {
    scmf_tune r = default_tune();
    if (!t) return r;
    if (t->chains_per_tile > 0) r.chains_per_tile = t->chains_per_tile;
    if (t->threads_move > 0) r.threads_move = std::min(256, std::max(32, t->threads_move / 32 * 32));
    if (t->cells_per_tile > 0) r.cells_per_tile = t->cells_per_tile;
    if (t->threads_field > 0) r.threads_field = std::min(256, std::max(32, t->threads_field / 32 * 32));
    r.persistent_ctas = std::max(0, t->persistent_ctas);
    r.use_graph = t->use_graph;
    r.beads_per_tile = std::max(0, std::min(t->beads_per_tile, kMaxTileBeads));
    return r;
}


void DevPlan::release() {
    if (graph) cudaGraphExecDestroy(graph);
    if (graph_src) cudaGraphDestroy(graph_src);
    if (side) {
        cudaStreamSynchronize(side);
        cudaStreamDestroy(side);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    side = nullptr;
    ev_fork = ev_join = nullptr;
    void* ptrs[] = {d_move, d_field, d_close, d_acc, d_ef, d_eb, d_flat_list, d_warp_list};
    for (void* p : ptrs) dev_free(p, stream);
    d_flat_list = nullptr;
    d_warp_list = nullptr;
    n_flat = n_warp = 0;
    graph = nullptr;
    graph_src = nullptr;
    d_move = nullptr;
    d_field = nullptr;
    d_close = nullptr;
    d_acc = nullptr;
    d_ef = nullptr;
    d_eb = nullptr;
    n_move = n_field = n_sys = 0;
}

scmf_status DevPlan::upload(const Plan& p, const scmf_tune& t, cudaStream_t st) {
    release();
    stream = st;
    tune = t;
    n_move = (int)p.move.size();
    n_field = (int)p.field.size();
    max_tile_beads = p.max_tile_beads;
    max_length = p.max_length;
    n_types_uniform = p.n_types_uniform;
    max_chains = p.max_chains;
    linear = p.linear;
    fold_kind = p.fold_kind;
    flat_threads = p.flat_threads > 0 ? p.flat_threads : t.threads_move;
    one_seed = p.one_seed && !p.close.empty();
    one_seed_hi = p.one_seed_hi && !p.close.empty();
    seed = p.seed;
    n_sys = (int)p.close.size();
    lean = n_sys == 1 && p.lean_ok && p.fold_kind == 0 && p.linear;
    warp_even = p.warp_even && p.linear && p.max_length <= 64;
    sc = p.sc;
    std::vector<int32_t> fl, wl;
    for (size_t i = 0; i < p.move.size(); ++i) (p.tile_flat[i] ? fl : wl).push_back((int32_t)i);
    n_flat = (int)fl.size();
    n_warp = (int)wl.size();
    if (n_flat > 0 && n_warp > 0 && p.linear && p.max_length <= 64) {
        CK(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    }
    const size_t nm = std::max<size_t>(1, p.move.size()), nf = std::max<size_t>(1, p.field.size());
    scmf_status rc;
    if ((rc = dev_alloc((void**)&d_move, nm * sizeof(MoveTile), st)) ||
        (rc = dev_alloc((void**)&d_field, nf * sizeof(FieldTile), st)) ||
        (rc = dev_alloc((void**)&d_close, std::max<size_t>(1, p.close.size()) * sizeof(SysClose), st)) ||
        (rc = dev_alloc((void**)&d_acc, nm * kMaxWarps * sizeof(unsigned), st)) ||
        (rc = dev_alloc((void**)&d_ef, nf * sizeof(double), st)) || (rc = dev_alloc((void**)&d_eb, nm * sizeof(double), st)) ||
        (rc = dev_alloc((void**)&d_flat_list, std::max<size_t>(1, fl.size()) * sizeof(int32_t), st)) ||
        (rc = dev_alloc((void**)&d_warp_list, std::max<size_t>(1, wl.size()) * sizeof(int32_t), st)))
        return rc;
    if (!fl.empty()) CK(cudaMemcpyAsync(d_flat_list, fl.data(), fl.size() * 4, cudaMemcpyHostToDevice, st));
    if (!wl.empty()) CK(cudaMemcpyAsync(d_warp_list, wl.data(), wl.size() * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(d_acc, 0, nm * kMaxWarps * sizeof(unsigned), st));
    CK(cudaMemcpyAsync(d_move, p.move.data(), p.move.size() * sizeof(MoveTile), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_field, p.field.data(), p.field.size() * sizeof(FieldTile), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_close, p.close.data(), p.close.size() * sizeof(SysClose), cudaMemcpyHostToDevice, st));
    // the host vectors may go away after return: wait for the (pageable) copies
    CK(cudaStreamSynchronize(st));
    return SCMF_OK;
}

LaunchShape DevPlan::move_shape() const {
    LaunchShape sh{};
    sh.blocks = tune.persistent_ctas > 0 ? std::min(tune.persistent_ctas, n_move) : 0;
    sh.threads = tune.threads_move;
    sh.n_types = n_types_uniform;
    sh.linear = linear ? 1 : 0;
    sh.max_chains = max_chains;
    sh.flat_list = d_flat_list;
    sh.n_flat = n_flat;
    sh.warp_list = d_warp_list;
    sh.n_warp = n_warp;
    sh.fold = fold_kind;
    sh.flat_threads = flat_threads;
    sh.keyed = one_seed ? kKeysBoth : (one_seed_hi ? kKeysHigh : kKeysNone);
    sh.keys = philox_schedule((uint32_t)seed, (uint32_t)(seed >> 32));
    sh.lean = lean && one_seed && n_flat == 0 ? 1 : 0;
    sh.warp_even = warp_even ? 1 : 0;
    sh.sc = sc;
    return sh;
}

LaunchShape DevPlan::field_shape() const {
    LaunchShape sh{};
    sh.blocks = tune.persistent_ctas > 0 ? std::min(tune.persistent_ctas, n_field) : 0;
    sh.threads = tune.threads_field;
    sh.n_types = n_types_uniform;
    sh.linear = linear ? 1 : 0;
    return sh;
}

scmf_status DevPlan::enqueue_close(int mode, cudaStream_t st) const {
    CKL(launch_close(d_close, n_sys, d_acc, warps_per_tile(), d_ef, d_eb, mode, st));
    return SCMF_OK;
}

scmf_status DevPlan::enqueue_sweep(cudaStream_t st) const {
    const scmf_status rc = enqueue_move(st);
    return rc ? rc : enqueue_field(st);
}

scmf_status DevPlan::enqueue_move(cudaStream_t st) const {
    if (side && n_warp > 0 && n_flat > 0) {
        LaunchShape warp = move_shape(), flat = move_shape();
        warp.part = 1;
        flat.part = 2;
        CK(cudaEventRecord(ev_fork, st));
        CK(cudaStreamWaitEvent(side, ev_fork, 0));
        CKL(launch_sweep(kMoveGrid, d_move, n_move, max_tile_beads, max_length, flat, d_acc, side));
        CK(cudaEventRecord(ev_join, side));
        CKL(launch_sweep(kMoveGrid, d_move, n_move, max_tile_beads, max_length, warp, d_acc, st));
        CK(cudaStreamWaitEvent(st, ev_join, 0));
    } else {
        CKL(launch_sweep(kMoveGrid, d_move, n_move, max_tile_beads, max_length, move_shape(), d_acc, st));
    }
    return SCMF_OK;
}

scmf_status DevPlan::enqueue_field(cudaStream_t st) const {
    CKL(launch_field(true, 0, d_field, n_field, field_shape(), d_ef, kSweepClose, st));
    return SCMF_OK;
}

scmf_status DevPlan::run_sweeps(cudaStream_t st, int n) {
    if (n <= 0) return SCMF_OK;
    if (tune.use_graph) {
        if (!graph) {
            CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            scmf_status rc = enqueue_sweep(st);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(st, &g);
            if (rc != SCMF_OK) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (e != cudaSuccess) return fail(SCMF_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
            graph_src = g;
            CK(cudaGraphInstantiate(&graph, g, 0));
        }
        for (int i = 0; i < n; ++i) CK(cudaGraphLaunch(graph, st));
        return SCMF_OK;
    }
    for (int i = 0; i < n; ++i) {
        scmf_status rc = enqueue_sweep(st);
        if (rc) return rc;
    }
    return SCMF_OK;
}

scmf_status fetch_sysdev(const scmf_system* s, SysDev* out) {
    CK(cudaMemcpyAsync(out, s->d_sys, sizeof(SysDev), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return SCMF_OK;
}

}  // namespace scmf

using namespace scmf;

// Work tiles of this system appended to a plan.
scmf_status scmf_system::append_plan(const scmf_tune& t, Plan* p) {
    // systems below ~2.4M beads: four tiles per SM (measured best over the 256-system mix
    // against two and six per SM with 4-warp CTAs)
    const int sms = sm_count();
    const int64_t target_small = std::max<int64_t>(1, n_beads / (4 * sms));
    const size_t first_tile = p->move.size();
    const size_t first_field = p->field.size();
    p->fold_kind = std::max(p->fold_kind, fold_kind_of(spec));
    // the lean kernel indexes beads and cells (times types) with 32-bit integers
    p->lean_ok = p->lean_ok && n_beads < (1ll << 31) && (int64_t)n_cells * spec.n_types < (1ll << 31);
    if (p->close.empty()) {
        p->seed = spec.p.seed;
        SysDev h{};
        fill_sysdev_constants(spec, n_beads, &h);
        SysConsts& c = p->sc;
        c.x = x;
        c.y = y;
        c.z = z;
        c.chain_id = chain_id;
        c.omega = omega;
        c.n_cells = h.n_cells;
        c.k2 = h.k2;
        c.A = h.A;
        c.R = h.R;
        c.inv_dx = h.inv_dx;
        c.inv_dy = h.inv_dy;
        c.inv_dz = h.inv_dz;
        c.nx = h.nx;
        c.ny = h.ny;
        c.nz = h.nz;
        for (int g = 0; g < 3; ++g) {
            c.cdeg[g] = h.cdeg[g];
            c.ac4deg[g] = h.ac4deg[g];
        }
        c.sys = d_sys;
        c.n_arch = 0;
        for (size_t a = 0; a < archs.size(); ++a) {
            if (archs[a].n_chains == 0) continue;
            if (c.n_arch == kLeanMaxArch) {
                p->lean_ok = false;
                break;
            }
            LeanArch& la = c.arch[c.n_arch++];
            la.types = h_arch[a].types;
            la.length = archs[a].length;
            la.n_chains = archs[a].n_chains;
            la.chain0 = archs[a].chain_base;
            la.bead0 = (int32_t)archs[a].bead_base;
            la.rng0 = archs[a].rng_base;  // chain_id[chain_base + c] = rng_base + c (storage order is never permuted)
            la.pad = 0;
        }
    } else {
        if (p->seed != spec.p.seed) p->one_seed = false;
        if ((p->seed >> 32) != (spec.p.seed >> 32)) p->one_seed_hi = false;
    }
    for (size_t a = 0; a < archs.size(); ++a) {
        const ArchHost& A = archs[a];
        if (A.n_chains == 0) continue;
        const bool explicit_cpt = t.beads_per_tile <= 0 && t.chains_per_tile > 0;
        int cpt = t.beads_per_tile > 0 ? std::max(1, t.beads_per_tile / A.length) : t.chains_per_tile;
        if (cpt <= 0) {
            const int64_t target = std::min<int64_t>(4096, std::max<int64_t>(A.length, target_small));
            cpt = (int)std::max<int64_t>(1, target / A.length);
        }
        if (!explicit_cpt && A.linear && A.length <= 64) {
            // whole iterations of the register kernel: a CTA moves cpi chains per
            // iteration, and a tile that is not a multiple of cpi ends on a mostly
            // idle one (measured 2.5 % on the large system)
            const int tpc = (A.length + 1) / 2;
            const int threads = 32 % tpc ? flat_threads_for(tpc, t.threads_move) : std::max(32, t.threads_move);
            const int cpi = 32 % tpc ? std::max(1, threads / tpc) : (32 / tpc) * (threads / 32);
            cpt = std::max(cpi, (cpt + cpi / 2) / cpi * cpi);
        }
        cpt = std::max(1, std::min(cpt, kMaxTileBeads / A.length));
        for (int c = 0; c < A.n_chains; c += cpt) {
            MoveTile mt;
            mt.sys = d_sys;
            mt.arch = d_arch + a;
            mt.chain0 = A.chain_base + c;
            mt.n_chains = std::min(cpt, A.n_chains - c);
            mt.bead0 = A.bead_base + (int64_t)c * A.length;
            mt.n_tiles_sys = 0;
            mt.arch_index = (int32_t)a;
            p->move.push_back(mt);
            const bool flat = A.linear && A.length <= 64 && 32 % ((A.length + 1) / 2) != 0;
            p->tile_flat.push_back(flat ? 1 : 0);
            if (flat) {
                const int ft = flat_threads_for((A.length + 1) / 2, t.threads_move);
                p->flat_threads = p->flat_threads == 0 || p->flat_threads == ft ? ft : -1;  // -1: archs disagree
            }
            p->max_tile_beads = std::max(p->max_tile_beads, mt.n_chains * A.length);
            p->max_chains = std::max(p->max_chains, mt.n_chains);
        }
        p->max_length = std::max(p->max_length, A.length);
        p->lean_ok = p->lean_ok && A.linear && A.length % 2 == 0 && A.length <= 64 && 32 % (A.length / 2) == 0;
        // the multi-system lean kernel reads bead pairs as float2: every warp-wise
        // architecture must have an even length and start at an even bead (an
        // odd-length architecture with an odd chain count before it would shift
        // it by one); otherwise the register kernel, which checks, runs them
        if (A.linear && A.length <= 64 && 32 % ((A.length + 1) / 2) == 0)
            p->warp_even = p->warp_even && A.length % 2 == 0 && A.bead_base % 2 == 0;
        p->max_deg = std::max(p->max_deg, A.max_deg);
        p->linear = p->linear && A.linear;
    }
    for (size_t i = first_tile; i < p->move.size(); ++i) p->move[i].n_tiles_sys = (int32_t)(p->move.size() - first_tile);
    int64_t cpt_cells = t.cells_per_tile;
    if (cpt_cells <= 0) cpt_cells = std::min<int64_t>(8192, std::max<int64_t>(1024, n_cells / (4 * sms)));
    cpt_cells = (cpt_cells + 3) & ~(int64_t)3;
    const int ntile = (int)((n_cells + cpt_cells - 1) / cpt_cells);
    for (int i = 0; i < ntile; ++i) {
        FieldTile ft;
        ft.sys = d_sys;
        ft.cell0 = (int64_t)i * cpt_cells;
        ft.n_cells = (int)std::min<int64_t>(cpt_cells, n_cells - ft.cell0);
        ft.n_tiles_sys = ntile;
        ft.first_tile = (int32_t)first_field;
        ft.pad = 0;
        p->field.push_back(ft);
    }
    SysClose cl;
    cl.sys = d_sys;
    cl.move_first = (int32_t)first_tile;
    cl.move_count = (int32_t)(p->move.size() - first_tile);
    cl.field_first = (int32_t)first_field;
    cl.field_count = (int32_t)(p->field.size() - first_field);
    p->close.push_back(cl);
    if (p->n_types_uniform == 0 && p->field.size() == (size_t)ntile) p->n_types_uniform = spec.n_types;
    else if (p->n_types_uniform != spec.n_types) p->n_types_uniform = 0;
    // round the smem tile up so float4 staging stays aligned
    p->max_tile_beads = (p->max_tile_beads + 3) & ~3;
    return SCMF_OK;
}

