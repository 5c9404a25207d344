// Time-averaged density, binary checkpoints and chain observables
// (include/scmf.h): the state around the hot path that a long run needs.
//
//   averaging   average_field_unified (struct.h:234, init_config.cu:770) and
//               io_out_aver_density (io.cpp:57-94).  The accumulator is
//               filled inside the fused field step (k_field) and the sample
//               count advanced by k_close, so scmf_step's captured graph
//               carries it without extra launches.
//   checkpoint  exact resume: positions bit for bit, omega, step, statistics
//               and averaging state.  The reference restarts through the
//               lossy coord.dat (init_config.cu:930-987).
//   analysis    end-to-end distance (test.cpp:47-68) and the Ana_Info
//               analyses (struct.h:65-75) as device reductions.
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <vector>

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

constexpr char kMagic[8] = {'S', 'C', 'M', 'F', 'C', 'K', 'P', 'T'};
constexpr uint32_t kVersion = 1;
static_assert(sizeof(scmf_checkpoint_header) == 128, "checkpoint header must stay 128 bytes");

// FNV-1a, 64-bit (Fowler, Noll, Vo): offset basis 14695981039346656037,
// prime 1099511628211.
struct Fnv {
    uint64_t h = 14695981039346656037ull;
    void add(const void* p, size_t n) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        for (size_t i = 0; i < n; ++i) {
            h ^= b[i];
            h *= 1099511628211ull;
        }
    }
    template <typename T>
    void put(T v) { add(&v, sizeof v); }
};

uint64_t spec_hash(const scmf_spec& s) {
    Fnv f;
    f.put<int32_t>(s.n_types);
    f.put<int32_t>(s.nx); f.put<int32_t>(s.ny); f.put<int32_t>(s.nz);
    f.put<double>(s.lx); f.put<double>(s.ly); f.put<double>(s.lz);
    for (double v : s.xn) f.put<double>(v);
    f.put<int32_t>(s.p.reference_nbeads);
    f.put<double>(s.p.harmonic_normb);
    f.put<double>(s.p.smc_a);
    f.put<int32_t>(s.p.hamiltonian);
    f.put<int32_t>(s.p.field_rule);
    f.put<int32_t>((int32_t)s.archs.size());
    for (const auto& a : s.archs) {
        f.put<int32_t>(a.length);
        f.put<int32_t>(a.n_chains);
        for (int t : a.type) f.put<int32_t>(t);
        f.put<int32_t>((int32_t)a.bonds.size());
        for (int b : a.bonds) f.put<int32_t>(b);
    }
    return f.h;
}

size_t cells_total(const scmf_system* s) { return (size_t)s->n_cells * s->spec.n_types; }

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) fclose(f);
    }
};

scmf_status read_exact(FILE* f, void* p, size_t n, const char* path, Fnv* h) {
    if (fread(p, 1, n, f) != n) return fail(SCMF_E_PARSE, "%s: truncated checkpoint", path);
    if (h) h->add(p, n);
    return SCMF_OK;
}

scmf_status read_header(FILE* f, const char* path, scmf_checkpoint_header* h) {
    char magic[8];
    if (fread(magic, 1, 8, f) != 8 || std::memcmp(magic, kMagic, 8) != 0)
        return fail(SCMF_E_PARSE, "%s: not an scmf checkpoint", path);
    if (fread(h, 1, sizeof *h, f) != sizeof *h) return fail(SCMF_E_PARSE, "%s: truncated checkpoint header", path);
    if (h->version != kVersion) return fail(SCMF_E_PARSE, "%s: checkpoint version %u (expected %u)", path, h->version, kVersion);
    if (h->n_types < 1 || h->n_types > kMaxTypes || h->n_beads < 0 || h->n_cells < 1)
        return fail(SCMF_E_PARSE, "%s: corrupt checkpoint header", path);
    const uint64_t cells = (uint64_t)h->n_cells * (uint64_t)h->n_types;
    const uint64_t want = 12ull * (uint64_t)h->n_beads + 4ull * cells + (h->avg_every ? 8ull * cells : 0ull);
    if (h->payload_bytes != want)
        return fail(SCMF_E_PARSE, "%s: payload of %llu bytes, header implies %llu", path,
                    (unsigned long long)h->payload_bytes, (unsigned long long)want);
    return SCMF_OK;
}

}  // namespace

extern "C" {

// ------------------------------------------------------------- averaging
scmf_status scmf_average_start(scmf_system* s, uint32_t every) {
    if (!s) return fail(SCMF_E_INVALID, "NULL system");
    const size_t bytes = cells_total(s) * sizeof(unsigned long long);
    if (every == 0) {
        CK(cudaMemsetAsync((char*)s->d_sys + offsetof(SysDev, avg), 0, sizeof(void*), s->stream));
        CK(cudaMemsetAsync((char*)s->d_sys + offsetof(SysDev, avg_samples), 0, 8, s->stream));
        CK(cudaMemsetAsync((char*)s->d_sys + offsetof(SysDev, avg_every), 0, 4, s->stream));
        if (s->d_avg) {
            dev_free(s->d_avg, s->stream);
            s->d_avg = nullptr;
        }
        CK(cudaStreamSynchronize(s->stream));
        return SCMF_OK;
    }
    if (!s->d_avg) RET(alloc_scratch((void**)&s->d_avg, bytes, s->stream));
    CK(cudaMemsetAsync(s->d_avg, 0, bytes, s->stream));
    unsigned long long* p = s->d_avg;
    const unsigned long long zero = 0ull;
    CK(cudaMemcpyAsync((char*)s->d_sys + offsetof(SysDev, avg_every), &every, 4, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync((char*)s->d_sys + offsetof(SysDev, avg_samples), &zero, 8, cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync((char*)s->d_sys + offsetof(SysDev, avg), &p, sizeof p, cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return SCMF_OK;
}

scmf_status scmf_average_sample(scmf_system* s) {
    if (!s) return fail(SCMF_E_INVALID, "NULL system");
    if (!s->d_avg) return fail(SCMF_E_STATE, "averaging is not started (scmf_average_start)");
    CKL(launch_average_sample(s->d_sys, (int64_t)cells_total(s), s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return SCMF_OK;
}

scmf_status scmf_average_get(const scmf_system* s, uint64_t* sums, size_t n, uint64_t* n_samples) {
    if (!s || !sums || !n_samples) return fail(SCMF_E_INVALID, "NULL argument");
    if (n != cells_total(s)) return fail(SCMF_E_INVALID, "expected %zu sums, got %zu", cells_total(s), n);
    if (!s->d_avg) return fail(SCMF_E_STATE, "averaging is not started (scmf_average_start)");
    SysDev d;
    RET(fetch_sysdev(s, &d));
    CK(cudaMemcpyAsync(sums, s->d_avg, n * sizeof(uint64_t), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    *n_samples = d.avg_samples;
    return SCMF_OK;
}

scmf_status scmf_write_average_density(const scmf_system* s, const char* path, int64_t step) {
    if (!s) return fail(SCMF_E_INVALID, "NULL system");
    const int n = s->spec.n_types;
    const size_t nc = (size_t)s->n_cells;
    std::vector<uint64_t> sums(nc * n);
    std::vector<float> om(nc * n);
    uint64_t samples = 0;
    RET(scmf_average_get(s, sums.data(), sums.size(), &samples));
    if (samples == 0) return fail(SCMF_E_STATE, "no density samples accumulated yet");
    RET(scmf_get_omega(s, om.data(), om.size()));
    char name[64];
    if (!path) {
        if (step < 1000000)
            snprintf(name, sizeof name, "density_aver_%d.dat", (int)step);
        else
            snprintf(name, sizeof name, "density_aver_%ge+06.dat", (double)step / 1000000);
        path = name;
    }
    FILE* f = fopen(path, "w");
    if (!f) return fail(SCMF_E_IO, "cannot open %s: %s", path, strerror(errno));
    const double scale = (double)nc / (double)s->n_beads;
    fprintf(f, "Nx=%d, Ny=%d, Nz=%d\n", s->spec.nx, s->spec.ny, s->spec.nz);
    fprintf(f, "dx=%g, dy=%g, dz=%g\n", s->spec.lx / s->spec.nx, s->spec.ly / s->spec.ny, s->spec.lz / s->spec.nz);
    for (size_t c = 0; c < nc; ++c) {
        for (int t = 0; t < n; ++t) fprintf(f, "%g ", (double)sums[c + t * nc] / (double)samples * scale);
        for (int t = 0; t < n; ++t) fprintf(f, "%g ", (double)om[c + t * nc]);
        fprintf(f, "\n");
    }
    if (fclose(f) != 0) return fail(SCMF_E_IO, "write to %s failed", path);
    return SCMF_OK;
}

// ------------------------------------------------------------ checkpoints
scmf_status scmf_spec_hash(const scmf_spec* spec, uint64_t* out) {
    if (!spec || !out) return fail(SCMF_E_INVALID, "NULL argument");
    *out = spec_hash(*spec);
    return SCMF_OK;
}

scmf_status scmf_checkpoint_write(const scmf_system* cs, const char* path) {
    scmf_system* s = const_cast<scmf_system*>(cs);
    if (!s || !path) return fail(SCMF_E_INVALID, "NULL argument");
    const size_t cells = cells_total(s);
    SysDev d;
    RET(fetch_sysdev(s, &d));
    std::vector<float> xyz((size_t)s->n_beads * 3);
    std::vector<float> om(cells);
    std::vector<uint64_t> avg(d.avg ? cells : 0);
    RET(scmf_get_coords(s, xyz.data(), xyz.size()));
    RET(scmf_get_omega(s, om.data(), om.size()));
    if (d.avg) {
        CK(cudaMemcpyAsync(avg.data(), s->d_avg, cells * 8, cudaMemcpyDeviceToHost, s->stream));
        CK(cudaStreamSynchronize(s->stream));
    }
    scmf_checkpoint_header h{};
    h.version = kVersion;
    h.n_types = s->spec.n_types;
    h.nx = s->spec.nx; h.ny = s->spec.ny; h.nz = s->spec.nz;
    h.n_chains = s->n_chains;
    h.n_arch = (int32_t)s->spec.archs.size();
    h.avg_every = d.avg ? d.avg_every : 0u;
    h.n_beads = s->n_beads;
    h.n_cells = s->n_cells;
    h.seed = s->spec.p.seed;
    h.spec_hash = spec_hash(s->spec);
    h.step = d.step;
    h.last_accepts = d.last_accepts;
    h.total_accepts = d.total_accepts;
    h.total_moves = d.total_moves;
    h.e_field = d.e_field;
    h.avg_samples = d.avg ? d.avg_samples : 0ull;
    h.payload_bytes = xyz.size() * 4 + om.size() * 4 + avg.size() * 8;
    Fnv fh;
    fh.add(xyz.data(), xyz.size() * 4);
    fh.add(om.data(), om.size() * 4);
    fh.add(avg.data(), avg.size() * 8);
    h.payload_hash = fh.h;
    File f;
    f.f = fopen(path, "wb");
    if (!f.f) return fail(SCMF_E_IO, "cannot open %s: %s", path, strerror(errno));
    bool ok = fwrite(kMagic, 1, 8, f.f) == 8 && fwrite(&h, 1, sizeof h, f.f) == sizeof h &&
              fwrite(xyz.data(), 4, xyz.size(), f.f) == xyz.size() && fwrite(om.data(), 4, om.size(), f.f) == om.size() &&
              fwrite(avg.data(), 8, avg.size(), f.f) == avg.size();
    const int rc = fclose(f.f);
    f.f = nullptr;
    if (!ok || rc != 0) return fail(SCMF_E_IO, "write to %s failed", path);
    return SCMF_OK;
}

scmf_status scmf_checkpoint_info(const char* path, scmf_checkpoint_header* out) {
    if (!path || !out) return fail(SCMF_E_INVALID, "NULL argument");
    File f;
    f.f = fopen(path, "rb");
    if (!f.f) return fail(SCMF_E_IO, "cannot open %s: %s", path, strerror(errno));
    scmf_checkpoint_header h;
    RET(read_header(f.f, path, &h));
    Fnv fh;
    std::vector<unsigned char> buf(1 << 20);
    uint64_t left = h.payload_bytes;
    while (left) {
        const size_t n = (size_t)std::min<uint64_t>(left, buf.size());
        RET(read_exact(f.f, buf.data(), n, path, &fh));
        left -= n;
    }
    if (fh.h != h.payload_hash) return fail(SCMF_E_PARSE, "%s: checkpoint checksum mismatch", path);
    if (fgetc(f.f) != EOF) return fail(SCMF_E_PARSE, "%s: trailing bytes after the checkpoint payload", path);
    *out = h;
    return SCMF_OK;
}

scmf_status scmf_checkpoint_read(scmf_system* s, const char* path) {
    if (!s || !path) return fail(SCMF_E_INVALID, "NULL argument");
    if (s->is_shard) return fail(SCMF_E_STATE, "checkpoints hold whole systems, not chain shards");
    File f;
    f.f = fopen(path, "rb");
    if (!f.f) return fail(SCMF_E_IO, "cannot open %s: %s", path, strerror(errno));
    scmf_checkpoint_header h;
    RET(read_header(f.f, path, &h));
    if (h.n_beads != s->n_beads || h.n_cells != s->n_cells || h.n_types != s->spec.n_types || h.nx != s->spec.nx ||
        h.ny != s->spec.ny || h.nz != s->spec.nz || h.n_chains != s->n_chains)
        return fail(SCMF_E_INVALID, "%s: checkpoint of a different system (%lld beads, %lld cells)", path,
                    (long long)h.n_beads, (long long)h.n_cells);
    if (h.spec_hash != spec_hash(s->spec)) return fail(SCMF_E_INVALID, "%s: checkpoint of a different spec", path);
    if (h.seed != s->spec.p.seed)
        return fail(SCMF_E_INVALID, "%s: checkpoint seed %llu differs from the system's %llu", path,
                    (unsigned long long)h.seed, (unsigned long long)s->spec.p.seed);
    if (h.step >= 0xFFFFFFF0ull) return fail(SCMF_E_PARSE, "%s: step out of range", path);
    const size_t cells = cells_total(s);
    std::vector<float> xyz((size_t)s->n_beads * 3);
    std::vector<float> om(cells);
    std::vector<uint64_t> avg(h.avg_every ? cells : 0);
    Fnv fh;
    RET(read_exact(f.f, xyz.data(), xyz.size() * 4, path, &fh));
    RET(read_exact(f.f, om.data(), om.size() * 4, path, &fh));
    RET(read_exact(f.f, avg.data(), avg.size() * 8, path, &fh));
    if (fh.h != h.payload_hash) return fail(SCMF_E_PARSE, "%s: checkpoint checksum mismatch", path);
    // positions, then the counts of those positions (cur = 0), then omega as saved
    RET(ensure_aos(s));
    CK(cudaMemcpyAsync(s->d_aos, xyz.data(), xyz.size() * 4, cudaMemcpyHostToDevice, s->stream));
    CKL(launch_aos_to_soa(s->d_aos, s->d_sys, s->d_arch, (int)s->archs.size(), s->n_beads, s->stream));
    RET(regrid(s));
    CK(cudaMemcpyAsync(s->omega, om.data(), cells * 4, cudaMemcpyHostToDevice, s->stream));
    SysDev d;
    RET(fetch_sysdev(s, &d));  // also waits for the copies above
    d.step = (uint32_t)h.step;
    d.last_accepts = h.last_accepts;
    d.total_accepts = h.total_accepts;
    d.total_moves = h.total_moves;
    d.e_field = h.e_field;
    d.e_bond_step = 0u;
    d.omega_span = INFINITY;  // omega came from the file: no span until the next field step
    for (int i = 0; i < kSlots; ++i) d.slot_acc[i] = 0ull;
    if (h.avg_every) {
        if (!s->d_avg) RET(alloc_scratch((void**)&s->d_avg, cells * 8, s->stream));
        CK(cudaMemcpyAsync(s->d_avg, avg.data(), cells * 8, cudaMemcpyHostToDevice, s->stream));
        d.avg = s->d_avg;
        d.avg_every = h.avg_every;
        d.avg_samples = h.avg_samples;
    } else {
        if (s->d_avg) {
            dev_free(s->d_avg, s->stream);
            s->d_avg = nullptr;
        }
        d.avg = nullptr;
        d.avg_every = 0u;
        d.avg_samples = 0ull;
    }
    CK(cudaMemcpyAsync(s->d_sys, &d, sizeof d, cudaMemcpyHostToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return check_error_word(s);
}

// ------------------------------------------------------------- validation
scmf_status scmf_validate(scmf_system* s, scmf_validation* out) {
    if (!s || !out) return fail(SCMF_E_INVALID, "NULL argument");
    std::memset(out, 0, sizeof *out);
    constexpr int kCounters = 4;
    if (!s->d_check)
        RET(alloc_scratch((void**)&s->d_check, (kCounters + kMaxTypes) * sizeof(unsigned long long), s->stream));
    CK(cudaMemsetAsync(s->d_check, 0, (kCounters + kMaxTypes) * sizeof(unsigned long long), s->stream));
    SysDev d;
    RET(fetch_sysdev(s, &d));
    const uint32_t cur = d.cur & 1u;
    const size_t cb = counts_bytes(s);
    // a fresh gridding of the positions into the idle counts buffer (zero
    // between calls), compared word by word with the current counts; the idle
    // buffer is cleared again afterwards
    const uint32_t other = cur ^ 1u;
    CK(cudaMemsetAsync(s->counts[other], 0, cb, s->stream));
    CK(cudaMemcpyAsync((char*)s->d_sys + offsetof(SysDev, cur), &other, 4, cudaMemcpyHostToDevice, s->stream));
    LaunchShape sh = s->plan.move_shape();
    sh.blocks = 0;
    CKL(launch_sweep(kGridOnly, s->plan.d_move, s->plan.n_move, s->plan.max_tile_beads, s->plan.max_length, sh,
                     s->plan.d_acc, s->stream));
    CK(cudaMemcpyAsync((char*)s->d_sys + offsetof(SysDev, cur), &cur, 4, cudaMemcpyHostToDevice, s->stream));
    CKL(launch_validate_positions(s->d_sys, s->n_beads, s->d_check, s->stream));
    CKL(launch_validate_cells(s->d_sys, s->counts[cur], s->counts[other], (int64_t)(cb / 4),
                              (int64_t)cells_total(s), s->d_check, s->d_check + kCounters, s->stream));
    CK(cudaMemsetAsync(s->counts[other], 0, cb, s->stream));
    unsigned long long h[kCounters + kMaxTypes];
    CK(cudaMemcpyAsync(h, s->d_check, sizeof h, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    out->nonfinite_positions = h[0];
    out->positions_out_of_range = h[1];
    out->count_mismatch_words = h[2];
    out->nonfinite_omega = h[3];
    std::vector<int64_t> per_type(s->spec.n_types, 0);
    for (const auto& a : s->archs)
        for (const auto& b : a.beads) per_type[b.type] += a.n_chains;
    int64_t err = 0;
    for (int t = 0; t < s->spec.n_types; ++t) err += std::llabs((int64_t)h[kCounters + t] - per_type[t]);
    out->count_sum_error = err;
    RET(fetch_sysdev(s, &d));
    out->error_word = d.error_word;
    if (out->nonfinite_positions || out->positions_out_of_range || out->count_mismatch_words ||
        out->nonfinite_omega || out->count_sum_error || out->error_word)
        return fail(SCMF_E_DEVICE,
                    "state check: %llu non-finite positions, %llu beyond the fold range, %llu count words differ "
                    "from the positions, %llu non-finite omega, count sum error %lld, error word 0x%x",
                    (unsigned long long)out->nonfinite_positions, (unsigned long long)out->positions_out_of_range,
                    (unsigned long long)out->count_mismatch_words, (unsigned long long)out->nonfinite_omega,
                    (long long)out->count_sum_error, out->error_word);
    return SCMF_OK;
}

// --------------------------------------------------------------- analysis
scmf_status scmf_analysis_reference(scmf_system* s) {
    if (!s) return fail(SCMF_E_INVALID, "NULL system");
    const size_t nb = (size_t)s->n_beads;
    if (!s->d_ref) RET(alloc_scratch((void**)&s->d_ref, nb * 3 * sizeof(float), s->stream));
    CK(cudaMemcpyAsync(s->d_ref, s->x, nb * 4, cudaMemcpyDeviceToDevice, s->stream));
    CK(cudaMemcpyAsync(s->d_ref + nb, s->y, nb * 4, cudaMemcpyDeviceToDevice, s->stream));
    CK(cudaMemcpyAsync(s->d_ref + 2 * nb, s->z, nb * 4, cudaMemcpyDeviceToDevice, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return SCMF_OK;
}

scmf_status scmf_analyze(const scmf_system* cs, scmf_observables* out, int32_t n_arch) {
    scmf_system* s = const_cast<scmf_system*>(cs);
    if (!s || !out) return fail(SCMF_E_INVALID, "NULL argument");
    if (n_arch != (int32_t)s->archs.size())
        return fail(SCMF_E_INVALID, "system has %d architectures, got room for %d", (int)s->archs.size(), n_arch);
    const DevPlan& p = s->plan;
    if (!s->d_obs) RET(alloc_scratch((void**)&s->d_obs, (size_t)std::max(1, p.n_move) * kObsSlots * sizeof(double), s->stream));
    CKL(launch_observables(p.d_move, p.n_move, s->d_ref, s->n_beads, s->d_obs, s->stream));
    std::vector<double> part((size_t)p.n_move * kObsSlots);
    std::vector<MoveTile> tiles(p.n_move);
    CK(cudaMemcpyAsync(part.data(), s->d_obs, part.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaMemcpyAsync(tiles.data(), p.d_move, tiles.size() * sizeof(MoveTile), cudaMemcpyDeviceToHost, s->stream));
    SysDev d;
    RET(fetch_sysdev(s, &d));  // waits for the copies above
    std::vector<double> sum((size_t)n_arch * kObsSlots, 0.0);
    for (int i = 0; i < p.n_move; ++i)  // tiles in plan order: a fixed summation order
        for (int k = 0; k < kObsSlots; ++k) sum[(size_t)tiles[i].arch_index * kObsSlots + k] += part[(size_t)i * kObsSlots + k];
    const double acc = d.total_moves && d.step ? (double)d.last_accepts / (double)s->n_beads : 0.0;
    const double nan = std::nan("");
    for (int a = 0; a < n_arch; ++a) {
        const ArchHost& A = s->archs[a];
        const scmf_spec::Arch& sa = s->spec.archs[a];
        scmf_observables& o = out[a];
        std::memset(&o, 0, sizeof o);
        o.arch = a;
        o.n_chains = A.n_chains;
        o.n_beads = (int64_t)A.n_chains * A.length;
        o.n_bonds = (int64_t)A.n_chains * (int64_t)(sa.bonds.size() / 2);
        const double* v = &sum[(size_t)a * kObsSlots];
        const double nc = A.n_chains > 0 ? (double)A.n_chains : nan;
        const double nbd = o.n_bonds > 0 ? (double)o.n_bonds : nan;
        const double nbe = o.n_beads > 0 ? (double)o.n_beads : nan;
        for (int c = 0; c < 3; ++c) {
            o.re2[c] = v[kObsRe + c] / nc;
            o.rg2[c] = v[kObsRg + c] / nc;
            o.bond2[c] = v[kObsBond + c] / nbd;
            o.msd[c] = s->d_ref ? v[kObsMsd + c] / nbe : nan;
            o.msd_com[c] = s->d_ref ? v[kObsMsdCom + c] / nc : nan;
        }
        o.re2[3] = o.re2[0] + o.re2[1] + o.re2[2];
        o.rg2[3] = o.rg2[0] + o.rg2[1] + o.rg2[2];
        o.bond2[3] = o.bond2[0] + o.bond2[1] + o.bond2[2];
        o.msd[3] = o.msd[0] + o.msd[1] + o.msd[2];
        o.msd_com[3] = o.msd_com[0] + o.msd_com[1] + o.msd_com[2];
        o.acc_ratio = acc;
    }
    return SCMF_OK;
}

}  // extern "C"
