// C ABI entry points for specs, systems and batches (include/scmf.h).
#include <cmath>
#include <cstddef>
#include <cstring>
#include <algorithm>
#include <numeric>

#include "scmf_engine.h"

using namespace scmf;

#define CK(expr)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (expr);                                                                   \
        if (e_ != cudaSuccess) return fail(SCMF_E_CUDA, "%s: %s", #expr, cudaGetErrorString(e_)); \
    } while (0)

#define CKL(expr)                                                                             \
    do {                                                                                      \
        int e_ = (expr);                                                                      \
        if (e_ != 0) return fail(SCMF_E_CUDA, "%s: %s", #expr, cudaGetErrorString((cudaError_t)e_)); \
    } while (0)

#define RET(expr)                        \
    do {                                 \
        scmf_status r_ = (expr);         \
        if (r_ != SCMF_OK) return r_;    \
    } while (0)

namespace {

size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

template <typename T>
scmf_status dalloc(T** p, size_t bytes, size_t* total, cudaStream_t st) {
    bytes = round_up(std::max<size_t>(bytes, 16), 256);
    scmf_status rc = dev_alloc((void**)p, bytes, st);
    if (rc) return rc;
    *total += bytes;
    return SCMF_OK;
}

void free_system(scmf_system* s) {
    if (!s) return;
    s->plan.release();
    void* ptrs[] = {s->x, s->y, s->z, s->chain_id, s->counts[0], s->counts[1], s->omega, s->d_sys, s->d_arch,
                    s->d_arch_blob, s->d_aos, s->d_u32, s->d_avg, s->d_ref, s->d_obs, s->d_check, s->d_total};
    for (void* p : ptrs) dev_free(p, s->stream);
    if (s->copy_stream) {
        cudaStreamSynchronize(s->copy_stream);
        cudaStreamDestroy(s->copy_stream);
        for (auto e : s->chunk_ev)
            if (e) cudaEventDestroy(e);
    }
    if (s->own_stream && s->stream) {
        cudaStreamSynchronize(s->stream);
        cudaStreamDestroy(s->stream);
    }
    delete s;
}

}  // namespace

namespace scmf {

scmf_status alloc_scratch(void** p, size_t bytes, cudaStream_t st) {
    size_t dummy = 0;
    return dalloc(p, bytes, &dummy, st);
}

size_t counts_bytes(const scmf_system* s) {
    const size_t cells = (size_t)s->n_cells * s->spec.n_types;
    return s->spec.p.count_bits == 16 ? ((cells + 1) / 2) * 4 : cells * 4;
}

// Clear both counts buffers, make counts[0] current and grid the current
// positions into it (init_array + coord_to_density, mesh.cu:161-190).
scmf_status regrid(scmf_system* s) {
    CK(cudaMemsetAsync(s->counts[0], 0, counts_bytes(s), s->stream));
    CK(cudaMemsetAsync(s->counts[1], 0, counts_bytes(s), s->stream));
    CK(cudaMemsetAsync((char*)s->d_sys + offsetof(SysDev, cur), 0, sizeof(uint32_t), s->stream));
    LaunchShape sh = s->plan.move_shape();
    sh.blocks = 0;
    CKL(launch_sweep(kGridOnly, s->plan.d_move, s->plan.n_move, s->plan.max_tile_beads, s->plan.max_length, sh,
                     s->plan.d_acc, s->stream));
    s->counts_stale = false;
    return SCMF_OK;
}

// Fused sweeps move counts cell to cell and so need counts that are the grid
// of the positions; only a move-only call (scmf_smc_move) leaves them behind.
scmf_status fresh_counts(scmf_system* s) { return s->counts_stale ? regrid(s) : SCMF_OK; }

scmf_status field_now(scmf_system* s) {
    LaunchShape sh = s->plan.field_shape();
    sh.blocks = 0;
    CKL(launch_field(false, 1, s->plan.d_field, s->plan.n_field, sh, s->plan.d_ef, kCloseField, s->stream));
    return SCMF_OK;
}

scmf_status ensure_aos(scmf_system* s) {
    if (s->d_aos) return SCMF_OK;
    size_t dummy = 0;
    return dalloc(&s->d_aos, (size_t)s->n_beads * 3 * sizeof(float), &dummy, s->stream);
}

scmf_status set_stop_step(scmf_system* s, uint32_t stop_step) {
    CK(cudaMemcpyAsync((char*)s->d_sys + offsetof(SysDev, stop_step), &stop_step, 4, cudaMemcpyHostToDevice,
                       s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return SCMF_OK;
}

scmf_status check_error_word(const scmf_system* s) {
    SysDev d;
    RET(fetch_sysdev(s, &d));
    if (d.error_word) return fail(SCMF_E_DEVICE, "kernel error word 0x%x", d.error_word);
    return SCMF_OK;
}

}  // namespace scmf

extern "C" {

const char* scmf_last_error(void) { return last_error_cstr(); }
const char* scmf_version(void) { return "scmf-b200 0.1 (sm_100a)"; }

// ------------------------------------------------------------------ spec
scmf_status scmf_spec_create(int32_t n, int32_t nx, int32_t ny, int32_t nz, double lx, double ly, double lz,
                             scmf_spec** out) {
    if (!out) return fail(SCMF_E_INVALID, "out is NULL");
    if (n < 1 || n > kMaxTypes) return fail(SCMF_E_INVALID, "n_mono_types %d not in [1,%d]", n, kMaxTypes);
    if (nx < 1 || ny < 1 || nz < 1) return fail(SCMF_E_INVALID, "bad grid");
    if (!(lx > 0 && ly > 0 && lz > 0)) return fail(SCMF_E_INVALID, "bad box");
    scmf_spec* s = new scmf_spec;
    s->n_types = n;
    s->nx = nx; s->ny = ny; s->nz = nz;
    s->lx = lx; s->ly = ly; s->lz = lz;
    s->xn.assign((size_t)n * n, 0.0);
    s->p.reference_nbeads = 1;
    s->p.harmonic_normb = 1.0;
    s->p.smc_a = 0.0;
    s->p.seed = 0;
    s->p.hamiltonian = SCMF_HAM_SCMF0;
    s->p.field_rule = SCMF_FIELD_EVERY;
    s->p.count_bits = 32;
    *out = s;
    return SCMF_OK;
}

scmf_status scmf_spec_set_xn(scmf_spec* s, const double* xn, int32_t n) {
    if (!s || !xn || n != s->n_types) return fail(SCMF_E_INVALID, "xn size must be n_mono_types^2");
    s->xn.assign(xn, xn + (size_t)n * n);
    return SCMF_OK;
}

scmf_status scmf_spec_set_params(scmf_spec* s, const scmf_params* p) {
    if (!s || !p) return fail(SCMF_E_INVALID, "NULL argument");
    s->p = *p;
    return SCMF_OK;
}

scmf_status scmf_spec_add_arch(scmf_spec* s, int32_t length, int32_t n_chains, const int32_t* mono_type,
                               int32_t n_bonds, const int32_t* bonds, double init_sigma) {
    if (!s || !mono_type || length < 1 || length > kMaxLength || n_chains < 0 || n_bonds < 0 ||
        (n_bonds > 0 && !bonds))
        return fail(SCMF_E_INVALID, "bad architecture arguments");
    scmf_spec::Arch a;
    a.length = length;
    a.n_chains = n_chains;
    a.type.assign(mono_type, mono_type + length);
    for (int i = 0; i < length; ++i)
        if (a.type[i] < 0 || a.type[i] >= s->n_types) return fail(SCMF_E_INVALID, "monomer type %d out of range", a.type[i]);
    if (n_bonds) a.bonds.assign(bonds, bonds + 2 * (size_t)n_bonds);
    for (int v : a.bonds)
        if (v < 0 || v >= length) return fail(SCMF_E_INVALID, "bond index %d out of range", v);
    a.init_sigma = init_sigma;
    s->archs.push_back(std::move(a));
    return SCMF_OK;
}

scmf_status scmf_spec_get_info(const scmf_spec* s, scmf_spec_info* o) {
    if (!s || !o) return fail(SCMF_E_INVALID, "NULL argument");
    std::memset(o, 0, sizeof *o);
    int64_t nb = 0;
    int nc = 0;
    for (const auto& a : s->archs) {
        nb += (int64_t)a.length * a.n_chains;
        nc += a.n_chains;
    }
    o->n_beads = nb;
    o->n_cells = (int64_t)s->nx * s->ny * s->nz;
    o->n_chains = nc;
    o->n_types = s->n_types;
    o->n_arch = (int32_t)s->archs.size();
    o->nx = s->nx; o->ny = s->ny; o->nz = s->nz;
    o->lx = s->lx; o->ly = s->ly; o->lz = s->lz;
    o->field_scaling = nb > 0 ? (double)o->n_cells / (double)nb : 0.0;
    o->harmonic_normb = s->p.harmonic_normb;
    o->smc_a = s->p.smc_a;
    o->smc_r = std::sqrt(2.0 * s->p.smc_a);
    o->reference_nbeads = s->p.reference_nbeads;
    o->count_bits = s->p.count_bits;
    return SCMF_OK;
}

scmf_status scmf_spec_get_params(const scmf_spec* s, scmf_params* out) {
    if (!s || !out) return fail(SCMF_E_INVALID, "NULL argument");
    *out = s->p;
    return SCMF_OK;
}

scmf_status scmf_spec_get_xn(const scmf_spec* s, double* xn, int32_t n) {
    if (!s || !xn || n != s->n_types) return fail(SCMF_E_INVALID, "bad arguments");
    std::memcpy(xn, s->xn.data(), sizeof(double) * n * n);
    return SCMF_OK;
}

scmf_status scmf_spec_get_arch(const scmf_spec* s, int32_t idx, int32_t* length, int32_t* n_chains,
                               int32_t* mono_type, int32_t type_cap, int32_t* bonds, int32_t bond_cap,
                               int32_t* n_bonds, double* init_sigma) {
    if (!s || idx < 0 || idx >= (int)s->archs.size()) return fail(SCMF_E_INVALID, "architecture index out of range");
    const auto& a = s->archs[idx];
    if (length) *length = a.length;
    if (n_chains) *n_chains = a.n_chains;
    if (n_bonds) *n_bonds = (int32_t)(a.bonds.size() / 2);
    if (init_sigma) *init_sigma = a.init_sigma;
    if (mono_type && type_cap >= a.length) std::memcpy(mono_type, a.type.data(), sizeof(int32_t) * a.length);
    if (bonds && bond_cap >= (int)a.bonds.size()) std::memcpy(bonds, a.bonds.data(), sizeof(int32_t) * a.bonds.size());
    return SCMF_OK;
}

scmf_status scmf_spec_copy(const scmf_spec* s, scmf_spec** out) {
    if (!s || !out) return fail(SCMF_E_INVALID, "NULL argument");
    *out = new scmf_spec(*s);
    return SCMF_OK;
}

void scmf_spec_destroy(scmf_spec* s) { delete s; }

scmf_status scmf_debug_math(uint32_t key_lo, uint32_t key_hi, int32_t n, uint32_t* words, float* logs,
                            float* normals) {
    if (n < 0 || !words || !logs || !normals) return fail(SCMF_E_INVALID, "bad arguments");
    if (n == 0) return SCMF_OK;
    void* d = nullptr;
    const size_t bytes = (size_t)n * (4 * 4 + 4 + 3 * 4);
    CK(cudaMalloc(&d, bytes));
    uint32_t* dw = (uint32_t*)d;
    float* dl = (float*)(dw + 4 * (size_t)n);
    float* dn = dl + n;
    int e = launch_debug_math(key_lo, key_hi, n, dw, dl, dn, nullptr);
    if (e == 0) e = (int)cudaDeviceSynchronize();
    if (e == 0) {
        cudaMemcpy(words, dw, 16 * (size_t)n, cudaMemcpyDeviceToHost);
        cudaMemcpy(logs, dl, 4 * (size_t)n, cudaMemcpyDeviceToHost);
        cudaMemcpy(normals, dn, 12 * (size_t)n, cudaMemcpyDeviceToHost);
    }
    cudaFree(d);
    if (e) return fail(SCMF_E_CUDA, "debug kernel: %s", cudaGetErrorString((cudaError_t)e));
    return SCMF_OK;
}

// ---------------------------------------------------------------- system
// Chains [first[a], first[a] + count[a]) of each architecture a form chain shard
// `shard` of `n_shards`: every architecture's chains are split into n_shards
// contiguous, near-equal runs (the reference splits chains over GPUs the same
// way, init_config.cu:220-222).
static void shard_chains(const scmf_spec& spec, int shard, int n_shards, std::vector<int>* first,
                         std::vector<int>* count) {
    first->clear();
    count->clear();
    for (const auto& a : spec.archs) {
        const int64_t lo = (int64_t)a.n_chains * shard / n_shards, hi = (int64_t)a.n_chains * (shard + 1) / n_shards;
        first->push_back((int)lo);
        count->push_back((int)(hi - lo));
    }
}

static scmf_status create_system(const scmf_spec* spec, bool is_shard, int shard, int n_shards, void* stream,
                                 scmf_system** out) {
    if (!spec || !out) return fail(SCMF_E_INVALID, "NULL argument");
    *out = nullptr;
    RET(validate_spec(*spec));
    if (n_shards < 1 || shard < 0 || shard >= n_shards) return fail(SCMF_E_INVALID, "shard %d of %d", shard, n_shards);
    if (is_shard && spec->p.count_bits != 32) return fail(SCMF_E_INVALID, "chain shards keep 32-bit counts");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        return fail(SCMF_E_CUDA, "no CUDA device available");
    }
    if (int e = configure_kernels()) return fail(SCMF_E_CUDA, "kernel configuration: %s", cudaGetErrorString((cudaError_t)e));
    scmf_system* s = new scmf_system;
    s->spec = *spec;
    s->is_shard = is_shard;
    s->shard = shard;
    s->n_shards = n_shards;
    std::vector<int> first, count;
    shard_chains(*spec, shard, n_shards, &first, &count);
    int64_t whole_beads = 0;
    for (size_t a = 0; a < spec->archs.size(); ++a) {
        whole_beads += (int64_t)spec->archs[a].length * spec->archs[a].n_chains;
        s->spec.archs[a].n_chains = count[a];
    }
    s->n_beads_total = whole_beads;
    scmf_status rc = prepare_archs(s->spec, &s->archs, &s->n_beads, &s->n_chains);
    if (!rc && is_shard && s->n_beads == 0) rc = fail(SCMF_E_INVALID, "shard %d of %d holds no chains", shard, n_shards);
    if (rc) {
        delete s;
        return rc;
    }
    // random-stream ids: a chain keeps the id it has in the whole system
    for (size_t a = 0, base = 0; a < s->archs.size(); base += spec->archs[a].n_chains, ++a)
        s->archs[a].rng_base = (int)base + first[a];
    s->n_cells = (int64_t)spec->nx * spec->ny * spec->nz;
    cudaGetDevice(&s->device);
    auto bail = [&](scmf_status r) {
        free_system(s);
        return r;
    };
    if (stream) {
        s->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
            return bail(fail(SCMF_E_CUDA, "cudaStreamCreate failed"));
        s->own_stream = true;
    }
    size_t tot = 0;
    const size_t nbp = (size_t)((s->n_beads + 3) & ~(int64_t)3);
    const size_t cells_t = (size_t)s->n_cells * spec->n_types;
    cudaStream_t st = s->stream;
    if ((rc = dalloc(&s->x, nbp * 4, &tot, st)) || (rc = dalloc(&s->y, nbp * 4, &tot, st)) ||
        (rc = dalloc(&s->z, nbp * 4, &tot, st)) || (rc = dalloc(&s->chain_id, (size_t)s->n_chains * 4, &tot, st)) ||
        (rc = dalloc(&s->counts[0], counts_bytes(s), &tot, st)) ||
        (rc = dalloc(&s->counts[1], counts_bytes(s), &tot, st)) || (rc = dalloc(&s->omega, cells_t * 4, &tot, st)) ||
        (rc = dalloc(&s->d_sys, sizeof(SysDev), &tot, st)) ||
        (rc = dalloc(&s->d_arch, s->archs.size() * sizeof(ArchDev), &tot, st)) ||
        (is_shard && (rc = dalloc(&s->d_total, cells_t * 4, &tot, st))))
        return bail(rc);
    // architecture tables
    size_t blob = 0;
    auto arch_bytes = [](int L) { return round_up((size_t)L * (sizeof(BeadInfo) + sizeof(uint16_t) + 1) + 16, 256); };
    for (const auto& a : s->archs) blob += arch_bytes(a.length);
    if ((rc = dalloc(&s->d_arch_blob, blob, &tot, st))) return bail(rc);
    s->device_bytes = tot;
    std::vector<char> hblob(blob, 0);
    size_t off = 0;
    for (const auto& a : s->archs) {
        ArchDev d{};
        std::memcpy(hblob.data() + off, a.beads.data(), a.length * sizeof(BeadInfo));
        d.beads = (const BeadInfo*)((char*)s->d_arch_blob + off);
        const size_t off2 = off + (size_t)a.length * sizeof(BeadInfo);
        std::memcpy(hblob.data() + off2, a.color_beads.data(), a.length * sizeof(uint16_t));
        d.color_beads = (const uint16_t*)((char*)s->d_arch_blob + off2);
        const size_t off3 = off2 + (size_t)a.length * sizeof(uint16_t);
        for (int i = 0; i < a.length; ++i) hblob[off3 + i] = (char)a.beads[i].type;
        d.types = (const uint8_t*)((char*)s->d_arch_blob + off3);
        off += arch_bytes(a.length);
        d.length = a.length;
        d.n_colors = a.n_colors;
        for (int c = 0; c <= a.n_colors; ++c) d.color_off[c] = a.color_off[c];
        for (int c = 0; c < a.n_colors; ++c) {
            const uint32_t nc = (uint32_t)(a.color_off[c + 1] - a.color_off[c]);
            d.color_magic[c] = magic_for(nc);
        }
        d.len_magic = magic_for((uint32_t)a.length);
        d.tpc_magic = magic_for((uint32_t)((a.length + 1) / 2));
        d.n_chains = a.n_chains;
        d.chain_base = a.chain_base;
        d.rng_base = a.rng_base;
        d.bead_base = a.bead_base;
        d.init_sigma = a.init_sigma;
        s->h_arch.push_back(d);
    }
    if (cudaMemcpyAsync(s->d_arch_blob, hblob.data(), blob, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(s->d_arch, s->h_arch.data(), s->h_arch.size() * sizeof(ArchDev), cudaMemcpyHostToDevice, st) !=
            cudaSuccess)
        return bail(fail(SCMF_E_CUDA, "upload of architecture tables failed"));
    std::vector<uint32_t> ids(s->n_chains);
    for (const auto& a : s->archs)
        for (int c = 0; c < a.n_chains; ++c) ids[a.chain_base + c] = (uint32_t)(a.rng_base + c);
    SysDev h{};
    fill_sysdev_constants(s->spec, s->n_beads_total, &h);  // field scaling n_cells / beads of the whole system
    h.n_beads = s->n_beads;
    h.field_counts = s->d_total;
    h.x = s->x; h.y = s->y; h.z = s->z;
    h.chain_id = s->chain_id;
    h.counts[0] = s->counts[0];
    h.counts[1] = s->counts[1];
    h.omega = s->omega;
    if (cudaMemcpyAsync(s->chain_id, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(s->d_sys, &h, sizeof h, cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemsetAsync(s->x, 0, nbp * 4, st) != cudaSuccess || cudaMemsetAsync(s->y, 0, nbp * 4, st) != cudaSuccess ||
        cudaMemsetAsync(s->z, 0, nbp * 4, st) != cudaSuccess ||
        cudaMemsetAsync(s->counts[0], 0, counts_bytes(s), st) != cudaSuccess ||
        cudaMemsetAsync(s->counts[1], 0, counts_bytes(s), st) != cudaSuccess ||
        cudaMemsetAsync(s->omega, 0, cells_t * 4, st) != cudaSuccess ||
        (s->d_total && cudaMemsetAsync(s->d_total, 0, cells_t * 4, st) != cudaSuccess))
        return bail(fail(SCMF_E_CUDA, "initialisation of device buffers failed"));
    Plan p;
    const scmf_tune t = default_tune();
    // upload() waits for the stream, so the host staging above may go out of scope
    if ((rc = s->append_plan(t, &p)) || (rc = s->plan.upload(p, t, st))) return bail(rc);
    *out = s;
    return SCMF_OK;
}

scmf_status scmf_system_create(const scmf_spec* spec, void* stream, scmf_system** out) {
    return create_system(spec, false, 0, 1, stream, out);
}

scmf_status scmf_system_create_shard(const scmf_spec* spec, int32_t shard, int32_t n_shards, void* stream,
                                     scmf_system** out) {
    return create_system(spec, true, shard, n_shards, stream, out);
}

scmf_status scmf_shard_chains(const scmf_spec* spec, int32_t shard, int32_t n_shards, int32_t* first,
                              int32_t* count, int32_t n_arch) {
    if (!spec || !first || !count) return fail(SCMF_E_INVALID, "NULL argument");
    if (n_shards < 1 || shard < 0 || shard >= n_shards) return fail(SCMF_E_INVALID, "shard %d of %d", shard, n_shards);
    if (n_arch != (int32_t)spec->archs.size()) return fail(SCMF_E_INVALID, "the spec has %zu architectures", spec->archs.size());
    std::vector<int> f, c;
    shard_chains(*spec, shard, n_shards, &f, &c);
    for (int a = 0; a < n_arch; ++a) {
        first[a] = f[a];
        count[a] = c[a];
    }
    return SCMF_OK;
}

static scmf_status shard_only(const scmf_system* s) {
    if (!s) return fail(SCMF_E_INVALID, "NULL system");
    if (!s->is_shard) return fail(SCMF_E_STATE, "not a chain shard (scmf_system_create_shard)");
    return SCMF_OK;
}

scmf_status scmf_shard_init_coords(scmf_system* s, uint32_t* d_partial) {
    RET(shard_only(s));
    if (!d_partial) return fail(SCMF_E_INVALID, "NULL counts buffer");
    CKL(launch_init_coords(s->d_sys, s->d_arch, (int)s->archs.size(), s->n_chains, s->stream));
    RET(regrid(s));
    CKL(launch_copy_counts(s->d_sys, d_partial, s->n_cells * s->spec.n_types, s->stream));
    return SCMF_OK;
}

scmf_status scmf_shard_move(scmf_system* s, uint32_t* d_partial) {
    RET(shard_only(s));
    if (!d_partial) return fail(SCMF_E_INVALID, "NULL counts buffer");
    RET(fresh_counts(s));
    RET(s->plan.enqueue_move(s->stream));
    CKL(launch_copy_counts(s->d_sys, d_partial, s->n_cells * s->spec.n_types, s->stream));
    return SCMF_OK;
}

scmf_status scmf_shard_field(scmf_system* s, const uint32_t* d_total, int32_t close_sweep) {
    RET(shard_only(s));
    if (!d_total) return fail(SCMF_E_INVALID, "NULL counts buffer");
    CK(cudaMemcpyAsync(s->d_total, d_total, (size_t)s->n_cells * s->spec.n_types * 4, cudaMemcpyDeviceToDevice,
                       s->stream));
    if (close_sweep) return s->plan.enqueue_field(s->stream);
    return field_now(s);
}

void scmf_system_destroy(scmf_system* s) {
    if (!s) return;
    if (s->batch_refs > 0) {  // a batch's plan still points at it: free with the last batch
        s->destroy_pending = true;
        return;
    }
    cudaStreamSynchronize(s->stream);
    free_system(s);
}

scmf_status scmf_system_get_info(const scmf_system* s, scmf_spec_info* out) {
    if (!s) return fail(SCMF_E_INVALID, "NULL system");
    return scmf_spec_get_info(&s->spec, out);
}

scmf_status scmf_system_stream(const scmf_system* s, void** st) {
    if (!s || !st) return fail(SCMF_E_INVALID, "NULL argument");
    *st = (void*)s->stream;
    return SCMF_OK;
}

scmf_status scmf_init_coords(scmf_system* s) {
    if (s && s->is_shard) return fail(SCMF_E_STATE, "a chain shard moves through scmf_shard_move / scmf_shard_field");
    if (!s) return fail(SCMF_E_INVALID, "NULL system");
    CKL(launch_init_coords(s->d_sys, s->d_arch, (int)s->archs.size(), s->n_chains, s->stream));
    RET(regrid(s));
    RET(field_now(s));
    CK(cudaStreamSynchronize(s->stream));
    return check_error_word(s);
}

// Positions from host AoS in chunks: chunk k's host-to-device copy runs on the
// copy stream while the system stream converts and grids chunk k - 1, so the
// conversion and the gridding hide behind the transfer (the first sweep cannot:
// its moves read the field of all the new positions).
static scmf_status upload_chunked(scmf_system* s, const float* xyz) {
    constexpr int kChunks = 8;
    if (!s->copy_stream) {
        CK(cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking));
        for (auto& e : s->chunk_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    CK(cudaMemsetAsync(s->counts[0], 0, counts_bytes(s), s->stream));
    CK(cudaMemsetAsync(s->counts[1], 0, counts_bytes(s), s->stream));
    CK(cudaMemsetAsync((char*)s->d_sys + offsetof(SysDev, cur), 0, sizeof(uint32_t), s->stream));
    // the staging buffer is free once the system stream's earlier work is done
    CK(cudaEventRecord(s->chunk_ev[0], s->stream));
    CK(cudaStreamWaitEvent(s->copy_stream, s->chunk_ev[0], 0));
    const int64_t n = s->n_beads, per = (n + kChunks - 1) / kChunks;
    for (int k = 0; k < kChunks; ++k) {
        const int64_t i0 = std::min<int64_t>(n, k * per), i1 = std::min<int64_t>(n, i0 + per);
        if (i1 <= i0) break;
        CK(cudaMemcpyAsync(s->d_aos + 3 * i0, xyz + 3 * i0, (size_t)(i1 - i0) * 3 * sizeof(float),
                           cudaMemcpyHostToDevice, s->copy_stream));
        CK(cudaEventRecord(s->chunk_ev[k], s->copy_stream));
        CK(cudaStreamWaitEvent(s->stream, s->chunk_ev[k], 0));
        CKL(launch_aos_chunk(s->d_aos, s->d_sys, s->d_arch, (int)s->archs.size(), i0, i1, s->stream));
    }
    s->counts_stale = false;
    return SCMF_OK;
}

scmf_status scmf_set_coords(scmf_system* s, const float* xyz, size_t n) {
    if (s && s->is_shard) return fail(SCMF_E_STATE, "a chain shard moves through scmf_shard_move / scmf_shard_field");
    if (!s || !xyz) return fail(SCMF_E_INVALID, "NULL argument");
    if (n != (size_t)s->n_beads * 3) return fail(SCMF_E_INVALID, "expected %lld floats, got %zu", (long long)s->n_beads * 3, n);
    RET(ensure_aos(s));
    RET(upload_chunked(s, xyz));
    RET(field_now(s));
    CK(cudaStreamSynchronize(s->stream));
    return check_error_word(s);
}

scmf_status scmf_get_coords(const scmf_system* cs, float* xyz, size_t n) {
    scmf_system* s = const_cast<scmf_system*>(cs);
    if (!s || !xyz) return fail(SCMF_E_INVALID, "NULL argument");
    if (n != (size_t)s->n_beads * 3) return fail(SCMF_E_INVALID, "expected %lld floats, got %zu", (long long)s->n_beads * 3, n);
    RET(ensure_aos(s));
    CKL(launch_soa_to_aos(s->d_aos, s->d_sys, s->d_arch, (int)s->archs.size(), s->n_beads, s->stream));
    CK(cudaMemcpyAsync(xyz, s->d_aos, n * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return SCMF_OK;
}

scmf_status scmf_set_step(scmf_system* s, uint64_t step) {
    if (!s) return fail(SCMF_E_INVALID, "NULL system");
    if (step >= 0xFFFFFFF0ull) return fail(SCMF_E_INVALID, "step out of range");
    const uint32_t v = (uint32_t)step;
    CK(cudaMemcpyAsync((char*)s->d_sys + offsetof(SysDev, step), &v, 4, cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return SCMF_OK;
}

scmf_status scmf_step_async(scmf_system* s, int32_t n) {
    if (s && s->is_shard) return fail(SCMF_E_STATE, "a chain shard moves through scmf_shard_move / scmf_shard_field");
    if (!s || n < 0) return fail(SCMF_E_INVALID, "bad argument");
    RET(fresh_counts(s));
    return s->plan.run_sweeps(s->stream, n);
}

scmf_status scmf_step(scmf_system* s, int32_t n) {
    RET(scmf_step_async(s, n));
    CK(cudaStreamSynchronize(s->stream));
    return check_error_word(s);
}

// n fused sweeps of a plan enqueued launch by launch, each bracketed by CUDA
// events on `st`: the summed device time of the move launches (both tile kinds
// when the plan forks them), of the field launches, and from the first launch
// to the end of the last.
static scmf_status profile_sweeps(const DevPlan& p, cudaStream_t st, int32_t n, float* ms_move, float* ms_field,
                                  float* ms_total) {
    *ms_move = 0.0f;
    *ms_field = 0.0f;
    *ms_total = 0.0f;
    if (n == 0) return SCMF_OK;
    std::vector<cudaEvent_t> ev(3 * (size_t)n, nullptr);
    scmf_status rc = SCMF_OK;
    for (auto& e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) rc = fail(SCMF_E_CUDA, "cudaEventCreate failed");
    for (int i = 0; i < n && !rc; ++i) {
        cudaEventRecord(ev[3 * i], st);
        rc = p.enqueue_move(st);
        cudaEventRecord(ev[3 * i + 1], st);
        if (!rc) rc = p.enqueue_field(st);
        cudaEventRecord(ev[3 * i + 2], st);
    }
    if (!rc && cudaStreamSynchronize(st) != cudaSuccess) rc = fail(SCMF_E_CUDA, "sweep failed");
    for (int i = 0; i < n && !rc; ++i) {
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, ev[3 * i], ev[3 * i + 1]);
        cudaEventElapsedTime(&b, ev[3 * i + 1], ev[3 * i + 2]);
        *ms_move += a;
        *ms_field += b;
    }
    if (!rc) cudaEventElapsedTime(ms_total, ev[0], ev[3 * (size_t)n - 1]);
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    return rc;
}

scmf_status scmf_step_profiled(scmf_system* s, int32_t n, float* ms_move, float* ms_field, float* ms_total) {
    if (s && s->is_shard) return fail(SCMF_E_STATE, "a chain shard moves through scmf_shard_move / scmf_shard_field");
    if (!s || n < 0 || !ms_move || !ms_field || !ms_total) return fail(SCMF_E_INVALID, "bad argument");
    RET(fresh_counts(s));
    RET(profile_sweeps(s->plan, s->stream, n, ms_move, ms_field, ms_total));
    return check_error_word(s);
}

scmf_status scmf_smc_move(scmf_system* s, int32_t n) {
    if (s && s->is_shard) return fail(SCMF_E_STATE, "a chain shard moves through scmf_shard_move / scmf_shard_field");
    if (!s || n < 0) return fail(SCMF_E_INVALID, "bad argument");
    const LaunchShape sh = s->plan.move_shape();
    for (int i = 0; i < n; ++i) {
        CKL(launch_sweep(kMoveOnly, s->plan.d_move, s->plan.n_move, s->plan.max_tile_beads, s->plan.max_length, sh,
                         s->plan.d_acc, s->stream));
        RET(s->plan.enqueue_close(kCloseMove | kCloseAdvance, s->stream));
    }
    if (n > 0) s->counts_stale = true;  // like the reference, counts wait for reset_density_fields
    CK(cudaStreamSynchronize(s->stream));
    return check_error_word(s);
}

scmf_status scmf_reset_density_fields(scmf_system* s) {
    if (s && s->is_shard) return fail(SCMF_E_STATE, "a chain shard moves through scmf_shard_move / scmf_shard_field");
    if (!s) return fail(SCMF_E_INVALID, "NULL system");
    RET(regrid(s));
    CK(cudaStreamSynchronize(s->stream));
    return check_error_word(s);
}

scmf_status scmf_update_omega_fields_scmf0(scmf_system* s) {
    if (s && s->is_shard) return fail(SCMF_E_STATE, "a chain shard moves through scmf_shard_move / scmf_shard_field");
    if (!s) return fail(SCMF_E_INVALID, "NULL system");
    RET(field_now(s));
    CK(cudaStreamSynchronize(s->stream));
    return SCMF_OK;
}

scmf_status scmf_synchronize(scmf_system* s) {
    if (!s) return fail(SCMF_E_INVALID, "NULL system");
    CK(cudaStreamSynchronize(s->stream));
    return SCMF_OK;
}

scmf_status scmf_get_counts(const scmf_system* cs, uint32_t* out, size_t n) {
    scmf_system* s = const_cast<scmf_system*>(cs);
    if (!s || !out) return fail(SCMF_E_INVALID, "NULL argument");
    const size_t want = (size_t)s->n_cells * s->spec.n_types;
    if (n != want) return fail(SCMF_E_INVALID, "expected %zu counts, got %zu", want, n);
    SysDev d;
    RET(fetch_sysdev(s, &d));
    if (s->spec.p.count_bits == 16) {
        if (!s->d_u32) {
            size_t dummy = 0;
            RET(dalloc(&s->d_u32, want * 4, &dummy, s->stream));
        }
        CKL(launch_unpack_counts16(s->d_sys, s->d_u32, (int64_t)want, s->stream));
        CK(cudaMemcpyAsync(out, s->d_u32, want * 4, cudaMemcpyDeviceToHost, s->stream));
    } else {
        CK(cudaMemcpyAsync(out, s->counts[d.cur & 1u], want * 4, cudaMemcpyDeviceToHost, s->stream));
    }
    CK(cudaStreamSynchronize(s->stream));
    return SCMF_OK;
}

scmf_status scmf_get_omega(const scmf_system* s, float* out, size_t n) {
    if (!s || !out) return fail(SCMF_E_INVALID, "NULL argument");
    const size_t want = (size_t)s->n_cells * s->spec.n_types;
    if (n != want) return fail(SCMF_E_INVALID, "expected %zu values, got %zu", want, n);
    CK(cudaMemcpyAsync(out, s->omega, want * 4, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return SCMF_OK;
}

scmf_status scmf_set_omega(scmf_system* s, const float* in, size_t n) {
    if (!s || !in) return fail(SCMF_E_INVALID, "NULL argument");
    const size_t want = (size_t)s->n_cells * s->spec.n_types;
    if (n != want) return fail(SCMF_E_INVALID, "expected %zu values, got %zu", want, n);
    CK(cudaMemcpyAsync(s->omega, in, want * 4, cudaMemcpyHostToDevice, s->stream));
    // the caller's omega has no known span: the move kernels read every trial's
    // omega until the next field step computes one
    const float no_span = INFINITY;
    CK(cudaMemcpyAsync((char*)s->d_sys + offsetof(SysDev, omega_span), &no_span, sizeof no_span,
                       cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return SCMF_OK;
}

scmf_status scmf_get_sweep_stats(const scmf_system* s, scmf_stats* o) {
    if (!s || !o) return fail(SCMF_E_INVALID, "NULL argument");
    SysDev d;
    RET(fetch_sysdev(s, &d));
    std::memset(o, 0, sizeof *o);
    o->step = d.step;
    o->last_accepts = d.last_accepts;
    o->total_accepts = d.total_accepts;
    o->total_moves = d.total_moves;
    o->e_bond = d.e_bond_step == d.step + 1u ? d.e_bond : std::nan("");
    o->e_field = d.e_field;
    o->error_word = d.error_word;
    return SCMF_OK;
}

scmf_status scmf_step_stats(scmf_system* s, int32_t n, scmf_stats* o) {
    if (s && s->is_shard) return fail(SCMF_E_STATE, "a chain shard moves through scmf_shard_move / scmf_shard_field");
    if (!s || !o || n < 0) return fail(SCMF_E_INVALID, "bad argument");
    RET(fresh_counts(s));
    RET(s->plan.run_sweeps(s->stream, n));
    SysDev d;
    RET(fetch_sysdev(s, &d));  // queued behind the sweeps: one wait for both
    if (d.error_word) return fail(SCMF_E_DEVICE, "kernel error word 0x%x", d.error_word);
    std::memset(o, 0, sizeof *o);
    o->step = d.step;
    o->last_accepts = d.last_accepts;
    o->total_accepts = d.total_accepts;
    o->total_moves = d.total_moves;
    o->e_bond = d.e_bond_step == d.step + 1u ? d.e_bond : std::nan("");
    o->e_field = d.e_field;
    o->error_word = d.error_word;
    return SCMF_OK;
}

scmf_status scmf_step_stats_async(scmf_system* s, int32_t n, scmf_stats* host_out) {
    if (s && s->is_shard) return fail(SCMF_E_STATE, "a chain shard moves through scmf_shard_move / scmf_shard_field");
    if (!s || !host_out || n < 0) return fail(SCMF_E_INVALID, "bad argument");
    RET(fresh_counts(s));
    RET(s->plan.run_sweeps(s->stream, n));
    CKL(launch_stats_out(s->d_sys, s->stream));
    CK(cudaMemcpyAsync(host_out, (const char*)s->d_sys + offsetof(SysDev, stats_out), sizeof(scmf_stats),
                       cudaMemcpyDeviceToHost, s->stream));
    return SCMF_OK;
}

scmf_status scmf_get_stats(const scmf_system* cs, scmf_stats* o) {
    scmf_system* s = const_cast<scmf_system*>(cs);
    if (!s || !o) return fail(SCMF_E_INVALID, "NULL argument");
    SysDev d;
    RET(fetch_sysdev(s, &d));
    if (d.e_bond_step != d.step + 1u) {  // bond energy is computed on demand
        CKL(launch_bond_energy(s->plan.d_move, s->plan.n_move, s->plan.move_shape(), s->plan.d_eb, s->stream));
        RET(s->plan.enqueue_close(kCloseBond, s->stream));
        RET(fetch_sysdev(s, &d));
    }
    std::memset(o, 0, sizeof *o);
    o->step = d.step;
    o->last_accepts = d.last_accepts;
    o->total_accepts = d.total_accepts;
    o->total_moves = d.total_moves;
    o->e_bond = d.e_bond;
    o->e_field = d.e_field;
    o->error_word = d.error_word;
    return SCMF_OK;
}

// --------------------------------------------------------------- batches
scmf_status scmf_batch_create(scmf_system* const* systems, int32_t n, const scmf_tune* tune, void* stream,
                              scmf_batch** out) {
    for (int32_t i = 0; systems && i < n; ++i)
        if (systems[i] && systems[i]->is_shard) return fail(SCMF_E_STATE, "chain shards do not join batches");
    if (!systems || n < 1 || !out) return fail(SCMF_E_INVALID, "bad arguments");
    *out = nullptr;
    scmf_batch* b = new scmf_batch;
    for (int i = 0; i < n; ++i) {
        if (!systems[i]) {
            delete b;
            return fail(SCMF_E_INVALID, "system %d is NULL", i);
        }
        for (int j = 0; j < i; ++j)
            if (systems[j] == systems[i]) {
                delete b;
                return fail(SCMF_E_INVALID, "system %d appears twice", i);
            }
        if (systems[i]->destroy_pending) {
            delete b;
            return fail(SCMF_E_INVALID, "system %d has been destroyed", i);
        }
        b->systems.push_back(systems[i]);
    }
    for (auto* s : b->systems) ++s->batch_refs;  // released by scmf_batch_destroy
    if (stream) {
        b->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
            b->stream = nullptr;
            scmf_batch_destroy(b);
            return fail(SCMF_E_CUDA, "cudaStreamCreate failed");
        }
        b->own_stream = true;
    }
    const scmf_tune t = resolve_tune(tune);
    Plan p;
    for (auto* s : b->systems) s->append_plan(t, &p);
    scmf_status rc = b->plan.upload(p, t, b->stream);
    if (rc) {
        scmf_batch_destroy(b);
        return rc;
    }
    *out = b;
    return SCMF_OK;
}

static scmf_status batch_sync_members(scmf_batch* b) {
    for (auto* s : b->systems) CK(cudaStreamSynchronize(s->stream));
    return SCMF_OK;
}

scmf_status scmf_batch_step_async(scmf_batch* b, int32_t n) {
    if (!b || n < 0) return fail(SCMF_E_INVALID, "bad argument");
    for (auto* s : b->systems) {
        RET(fresh_counts(s));
        if (s->stream != b->stream) CK(cudaStreamSynchronize(s->stream));
    }
    return b->plan.run_sweeps(b->stream, n);
}

scmf_status scmf_batch_step(scmf_batch* b, int32_t n) {
    RET(scmf_batch_step_async(b, n));
    CK(cudaStreamSynchronize(b->stream));
    return SCMF_OK;
}

scmf_status scmf_batch_step_profiled(scmf_batch* b, int32_t n, float* ms_move, float* ms_field, float* ms_total) {
    if (!b || n < 0 || !ms_move || !ms_field || !ms_total) return fail(SCMF_E_INVALID, "bad argument");
    for (auto* s : b->systems) {
        RET(fresh_counts(s));
        if (s->stream != b->stream) CK(cudaStreamSynchronize(s->stream));
    }
    RET(profile_sweeps(b->plan, b->stream, n, ms_move, ms_field, ms_total));
    for (auto* s : b->systems) RET(check_error_word(s));
    return SCMF_OK;
}

scmf_status scmf_batch_tune_trials(const scmf_batch* b, scmf_tune_trial* out, int32_t max, int32_t* n) {
    if (!b || !n || max < 0 || (max > 0 && !out)) return fail(SCMF_E_INVALID, "bad arguments");
    *n = (int32_t)b->trials.size();
    for (int32_t i = 0; i < *n && i < max; ++i) {
        std::memset(&out[i], 0, sizeof out[i]);
        out[i].tune = b->trials[i].first;
        out[i].ms = b->trials[i].second;
    }
    return SCMF_OK;
}

scmf_status scmf_batch_get_tune(const scmf_batch* b, scmf_tune* out) {
    if (!b || !out) return fail(SCMF_E_INVALID, "NULL argument");
    *out = b->plan.tune;
    return SCMF_OK;
}

void scmf_batch_destroy(scmf_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    b->plan.release();
    if (b->stream) cudaStreamSynchronize(b->stream);  // the plan's stream-ordered frees
    if (b->own_stream) cudaStreamDestroy(b->stream);
    for (auto* s : b->systems)
        if (--s->batch_refs == 0 && s->destroy_pending) {
            s->destroy_pending = false;
            scmf_system_destroy(s);
        }
    delete b;
}

scmf_status scmf_batch_run(scmf_system* const* systems, int32_t n, int32_t n_sweeps, const scmf_tune* tune) {
    scmf_batch* b = nullptr;
    RET(scmf_batch_create(systems, n, tune, nullptr, &b));
    scmf_status rc = scmf_batch_step(b, n_sweeps);
    scmf_batch_destroy(b);
    return rc;
}

// Snapshot of the mutable device state of one system (autotune trials run on
// the live buffers and are undone from here).
struct Snapshot {
    float* xyz = nullptr;
    uint32_t* cnt = nullptr;
    float* om = nullptr;
    SysDev sd{};
};

static scmf_status snap_take(scmf_system* s, Snapshot* sn, cudaStream_t st) {
    const size_t nb = (size_t)s->n_beads * 4, cb = counts_bytes(s), ob = (size_t)s->n_cells * s->spec.n_types * 4;
    size_t dummy = 0;
    RET(dalloc(&sn->xyz, 3 * nb, &dummy, st));
    RET(dalloc(&sn->cnt, 2 * cb, &dummy, st));
    RET(dalloc(&sn->om, ob, &dummy, st));
    CK(cudaMemcpyAsync(sn->xyz, s->x, nb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync((char*)sn->xyz + nb, s->y, nb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync((char*)sn->xyz + 2 * nb, s->z, nb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(sn->cnt, s->counts[0], cb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync((char*)sn->cnt + cb, s->counts[1], cb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(sn->om, s->omega, ob, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(&sn->sd, s->d_sys, sizeof(SysDev), cudaMemcpyDeviceToHost, st));
    return SCMF_OK;
}

static scmf_status snap_restore(scmf_system* s, Snapshot* sn, cudaStream_t st) {
    const size_t nb = (size_t)s->n_beads * 4, cb = counts_bytes(s), ob = (size_t)s->n_cells * s->spec.n_types * 4;
    CK(cudaMemcpyAsync(s->x, sn->xyz, nb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s->y, (char*)sn->xyz + nb, nb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s->z, (char*)sn->xyz + 2 * nb, nb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s->counts[0], sn->cnt, cb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s->counts[1], (char*)sn->cnt + cb, cb, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s->omega, sn->om, ob, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s->d_sys, &sn->sd, sizeof(SysDev), cudaMemcpyHostToDevice, st));
    CK(cudaStreamSynchronize(st));
    return SCMF_OK;
}

static void snap_free(Snapshot* sn, cudaStream_t st) {
    dev_free(sn->xyz, st);
    dev_free(sn->cnt, st);
    dev_free(sn->om, st);
    sn->xyz = nullptr;
    sn->cnt = nullptr;
    sn->om = nullptr;
}

// Project-written autotuner: times a small grid of (threads per move CTA,
// chains per tile, persistent CTAs) and then (cells per field tile) on the
// batch's own systems, restoring their state after every trial.
scmf_status scmf_batch_autotune(scmf_batch* b, int32_t sweeps, scmf_tune* out) {
    if (!b || sweeps < 1) return fail(SCMF_E_INVALID, "bad arguments");
    RET(batch_sync_members(b));
    std::vector<Snapshot> snaps(b->systems.size());
    scmf_status rc = SCMF_OK;
    for (size_t i = 0; i < b->systems.size() && !rc; ++i) rc = snap_take(b->systems[i], &snaps[i], b->stream);
    if (!rc && cudaStreamSynchronize(b->stream) != cudaSuccess) rc = fail(SCMF_E_CUDA, "snapshot failed");
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto trial = [&](const scmf_tune& t, float* ms) -> scmf_status {
        DevPlan dp;
        Plan p;
        for (auto* s : b->systems) s->append_plan(t, &p);
        RET(dp.upload(p, t, b->stream));
        scmf_status r = dp.run_sweeps(b->stream, 1);  // warm-up (and graph capture)
        if (!r) {
            cudaEventRecord(e0, b->stream);
            r = dp.run_sweeps(b->stream, sweeps);
            cudaEventRecord(e1, b->stream);
        }
        if (!r && cudaEventSynchronize(e1) != cudaSuccess) r = fail(SCMF_E_CUDA, "trial failed");
        if (!r) cudaEventElapsedTime(ms, e0, e1);
        dp.release();
        for (size_t i = 0; i < b->systems.size() && !r; ++i) r = snap_restore(b->systems[i], &snaps[i], b->stream);
        return r;
    };
    scmf_tune best = b->plan.tune;
    float best_ms = 1e30f;
    b->trials.clear();
    if (!rc) {
        const int tile_beads[] = {1024, 2048, 4096, 8192};
        const int threads[] = {64, 128, 256};
        const int persist[] = {0, sm_count() * 4};
        for (int tb : tile_beads)
            for (int th : threads)
                for (int pc : persist) {
                    if (rc) break;
                    scmf_tune t = b->plan.tune;
                    t.chains_per_tile = 0;
                    t.beads_per_tile = tb;
                    t.threads_move = th;
                    t.persistent_ctas = pc;
                    float ms = 0;
                    rc = trial(t, &ms);
                    if (!rc) b->trials.push_back({t, ms});
                    if (!rc && ms < best_ms) {
                        best_ms = ms;
                        best = t;
                    }
                }
        const int cells[] = {2048, 8192, 32768};
        scmf_tune base = best;
        for (int c : cells) {
            if (rc) break;
            scmf_tune t = base;
            t.cells_per_tile = c;
            float ms = 0;
            rc = trial(t, &ms);
            if (!rc) b->trials.push_back({t, ms});
            if (!rc && ms < best_ms) {
                best_ms = ms;
                best = t;
            }
        }
    }
    for (auto& sn : snaps) snap_free(&sn, b->stream);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    Plan p;
    for (auto* s : b->systems) s->append_plan(best, &p);
    RET(b->plan.upload(p, best, b->stream));
    if (out) *out = best;
    return SCMF_OK;
}

}  // extern "C"
