// Host-side engine objects behind the C ABI (include/scmf.h).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "scmf.h"
#include "scmf_internal.h"

// A system specification (box, grid, interactions, architectures).  Plain
// host data; nothing here touches the GPU.
struct scmf_spec {
    int n_types = 0, nx = 0, ny = 0, nz = 0;
    double lx = 0, ly = 0, lz = 0;
    std::vector<double> xn;  // [t + n*s]
    scmf_params p{};
    struct Arch {
        int length = 0, n_chains = 0;
        std::vector<int> type;   // [length]
        std::vector<int> bonds;  // pairs
        double init_sigma = 0;   // per-component sigma of the initial random walk
    };
    std::vector<Arch> archs;
};

namespace scmf {

scmf_status fail(scmf_status code, const char* fmt, ...);
void clear_error();
const char* last_error_cstr();

// Architecture prepared for the device: adjacency in ascending index order,
// greedy colouring in index order, beads grouped by colour, division magics.
struct ArchHost {
    int length = 0, n_colors = 0, n_chains = 0, chain_base = 0, max_deg = 0;
    int rng_base = 0;  // random-stream id of the first chain (chain_base, or its id in the whole system)
    bool linear = false;  // bonds exactly (i, i+1): even/odd colouring, computed neighbours
    int64_t bead_base = 0;
    float init_sigma = 0;
    std::vector<BeadInfo> beads;
    std::vector<uint16_t> color_beads;
    int color_off[kMaxColors + 1] = {};
};

// Stream-ordered device memory (cudaMallocAsync / cudaFreeAsync on the
// device's default pool, kept cached): creating and destroying systems and
// plans never synchronises the device.
scmf_status dev_alloc(void** p, size_t bytes, cudaStream_t st);
void dev_free(void* p, cudaStream_t st);

scmf_status validate_spec(const scmf_spec& s);
scmf_status prepare_archs(const scmf_spec& s, std::vector<ArchHost>* out, int64_t* n_beads, int* n_chains);
uint32_t magic_for(uint32_t n);
size_t system_device_bytes(const scmf_spec& s);
void fill_sysdev_constants(const scmf_spec& s, int64_t n_beads, SysDev* d);
int fold_kind_of(const scmf_spec& s);  // 0: every grid axis a power of two, 1: otherwise
// Block size for chains of ceil(L/2) = tpc threads laid across warps:
// lcm(tpc, 32) when it is at most 256 (no idle lane), else threads_move.
int flat_threads_for(int tpc, int threads_move);

// Work decomposition of one or many systems for one launch shape.
struct Plan {
    std::vector<MoveTile> move;
    std::vector<FieldTile> field;
    std::vector<SysClose> close;   // tile ranges of every system
    int max_tile_beads = 0;
    int max_length = 0;
    int n_types_uniform = 0;
    int max_deg = 0;
    int max_chains = 0;   // most chains in one move tile
    bool linear = true;
    int fold_kind = 0;  // largest fold_kind_of() of the systems
    int flat_threads = 0;  // block size of the block-wide move launch (0: none yet, -1: archs disagree)
    std::vector<uint8_t> tile_flat;  // per move tile: chains run across warps (32 % ceil(L/2) != 0)
    uint64_t seed = 0;      // the systems' seed when they all share one
    bool one_seed = true;   // every system appended so far has `seed`
    bool one_seed_hi = true;  // ... or at least its upper 32 bits
    bool lean_ok = true;      // every architecture so far fits the lean move kernel
    bool warp_even = true;    // every warp-wise linear architecture so far has an even length
    SysConsts sc{};           // move constants of the first system appended
};

struct DevPlan {
    MoveTile* d_move = nullptr;
    FieldTile* d_field = nullptr;
    SysClose* d_close = nullptr;
    unsigned* d_acc = nullptr;   // accept count per (move tile, warp)
    double* d_ef = nullptr;      // field energy per field tile
    double* d_eb = nullptr;      // bond energy per move tile
    int n_move = 0, n_field = 0, n_sys = 0;
    int max_tile_beads = 0, max_length = 0, n_types_uniform = 0, max_chains = 0;
    bool linear = false;
    int32_t* d_flat_list = nullptr;  // tile indices for the block-wide register kernel
    int32_t* d_warp_list = nullptr;  // tile indices for the warp-wise register kernel
    int n_flat = 0, n_warp = 0;
    int fold_kind = 0;
    int flat_threads = 0;
    bool one_seed = false;     // every system of the plan has `seed`: move launches take its key schedule
    bool one_seed_hi = false;  // they share its upper 32 bits: the second key word's schedule
    uint64_t seed = 0;
    bool lean = false;  // one system that fits the lean move kernel (LaunchShape::lean)
    bool warp_even = false;  // LaunchShape::warp_even
    SysConsts sc{};
    scmf_tune tune{};
    cudaGraphExec_t graph = nullptr;
    cudaGraph_t graph_src = nullptr;
    cudaStream_t stream = nullptr;  // allocations of the plan are ordered on it
    // plans with both warp-wise and flat tiles run the two move launches side
    // by side (fork on ev_fork, join on ev_join) so neither waits for the
    // other's last partial wave
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    void release();
    scmf_status upload(const Plan& p, const scmf_tune& t, cudaStream_t st);
    LaunchShape move_shape() const;
    LaunchShape field_shape() const;
    int warps_per_tile() const { return tune.threads_move / 32; }
    // one fused sweep (move+grid, field, close) enqueued on `st`: the move
    // launches (two side by side when the plan has both tile kinds), then the
    // field launch whose last tile per system closes the sweep
    scmf_status enqueue_sweep(cudaStream_t st) const;
    scmf_status enqueue_move(cudaStream_t st) const;
    scmf_status enqueue_field(cudaStream_t st) const;
    scmf_status enqueue_close(int mode, cudaStream_t st) const;
    scmf_status run_sweeps(cudaStream_t st, int n);
};

scmf_tune default_tune();
scmf_tune resolve_tune(const scmf_tune* t);

}  // namespace scmf

struct scmf_system {
    scmf_spec spec;  // for a chain shard: the shard's own chain counts
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int device = 0;
    int64_t n_beads = 0, n_cells = 0;
    // chain shard `shard` of `n_shards` (n_shards == 1: a whole system); n_beads_total
    // is the whole system's bead count (the field scaling), d_total the summed counts
    // of all shards that its field step reads
    bool is_shard = false;  // made by scmf_system_create_shard (any n_shards, 1 included)
    int shard = 0, n_shards = 1;
    int64_t n_beads_total = 0;
    uint32_t* d_total = nullptr;
    int n_chains = 0;
    size_t device_bytes = 0;
    // device buffers
    float* x = nullptr;
    float* y = nullptr;
    float* z = nullptr;
    uint32_t* chain_id = nullptr;
    uint32_t* counts[2] = {nullptr, nullptr};
    float* omega = nullptr;
    scmf::SysDev* d_sys = nullptr;
    scmf::ArchDev* d_arch = nullptr;
    void* d_arch_blob = nullptr;
    float* d_aos = nullptr;      // staging for AoS coordinate transfers (lazy)
    // chunked uploads: copies on their own stream, one event per chunk (lazy)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t chunk_ev[8] = {};
    uint32_t* d_u32 = nullptr;   // staging for unpacked 16-bit counts (lazy)
    unsigned long long* d_avg = nullptr;  // time-averaged density accumulator (while averaging)
    float* d_ref = nullptr;      // reference snapshot for displacements, SoA (lazy)
    double* d_obs = nullptr;     // per-tile observable partials (lazy)
    unsigned long long* d_check = nullptr;  // validation counters (lazy)
    bool counts_stale = false;    // moved without counts (scmf_smc_move): regrid before a fused sweep
    int batch_refs = 0;           // batches whose plans point at this system
    bool destroy_pending = false; // destroyed by the caller while still in a batch
    std::vector<scmf::ArchHost> archs;
    std::vector<scmf::ArchDev> h_arch;  // host image of d_arch
    scmf::DevPlan plan;                  // default work plan of this system alone

    scmf_status append_plan(const scmf_tune& t, scmf::Plan* p);
};

struct scmf_batch {
    std::vector<scmf_system*> systems;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    scmf::DevPlan plan;
    std::vector<std::pair<scmf_tune, float>> trials;  // the last autotune's tunings and their times (ms)
};

namespace scmf {
scmf_status fetch_sysdev(const scmf_system* s, SysDev* out);
scmf_status current_counts(const scmf_system* s, uint32_t* host_out, size_t n);
scmf_status write_density_file(const scmf_system* s, const char* path, int64_t step);
// scmf_api.cpp helpers shared with scmf_state.cpp
scmf_status alloc_scratch(void** p, size_t bytes, cudaStream_t st);  // device buffer, 256-byte rounded
size_t counts_bytes(const scmf_system* s);
scmf_status regrid(scmf_system* s);         // counts of the current positions into counts[0], cur = 0
scmf_status fresh_counts(scmf_system* s);   // regrid if a move-only call left the counts stale
scmf_status field_now(scmf_system* s);      // omega of the current counts (always updated)
scmf_status ensure_aos(scmf_system* s);     // AoS staging buffer
scmf_status check_error_word(const scmf_system* s);
// Fused sweeps skip the system once its step reaches stop_step (served form).
scmf_status set_stop_step(scmf_system* s, uint32_t stop_step);
}  // namespace scmf
