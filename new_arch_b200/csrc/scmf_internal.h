// Internal data model shared by the host engine (C++) and the kernels (CUDA).
//
// HBM layout of one system (all cudaMalloc'd, owned by the system):
//   x, y, z      float[n_beads]       SoA bead coordinates, unwrapped (the box is
//                                      folded only when a cell index is taken,
//                                      device_function.cu:313-360).  Beads of a
//                                      chain are contiguous; chains are grouped
//                                      by architecture (init_config.cu:610-629).
//   chain_id     uint32[n_chains]     storage slot -> global chain id (the first
//                                      Philox counter word).  Storage order is the id
//                                      order within each architecture (chain_id[chain_base
//                                      + c] = rng_base + c), which the lean kernels use to
//                                      compute the id instead of loading it; the other
//                                      kernels read this table.
//   counts[2]    uint32[n_types*n_cells] (or uint16 pairs)  per-type cell counts,
//                                      [type][z][y][x].  counts[cur] is kept the
//                                      grid of the positions: a fused sweep
//                                      moves a count for each accepted move that
//                                      leaves its cell.  The other buffer is
//                                      zero between calls (validation scratch).
//   omega        float[n_types*n_cells]  quasi-instantaneous field.
// plus a SysDev descriptor in device memory holding constants, the sweep
// counter and the statistics accumulators.
#pragma once
#include <stdint.h>

#include "scmf.h"

namespace scmf {

constexpr int kMaxTypes = 8;
constexpr int kMaxDeg = 8;
constexpr int kMaxColors = 8;
constexpr int kMaxLength = 4096;    // beads per chain (16-bit neighbour indices)
constexpr int kMaxTileBeads = 8192;  // beads staged in shared memory per tile
constexpr int kMaxWarps = 8;         // warps per move CTA (256 threads at most)
constexpr int kSlots = 32;           // spread of the accept-count atomics
constexpr uint32_t kInitStep = 0xFFFFFFFFu;

// Per-bead architecture record.
struct BeadInfo {
    uint8_t type, deg, color, pad;
    uint16_t nbr[kMaxDeg];
};

// One polymer architecture of one system.
struct ArchDev {
    const BeadInfo* beads;       // [length]
    const uint16_t* color_beads; // [length], beads grouped by colour
    const uint8_t* types;        // [length], monomer type per bead
    int32_t length;
    int32_t n_colors;
    int32_t color_off[kMaxColors + 1];
    uint32_t color_magic[kMaxColors];  // ceil(2^32 / n_in_colour): i / n == umulhi(i, magic)
    uint32_t len_magic;          // ceil(2^32 / length)
    uint32_t tpc_magic;          // magic of ceil(length / 2): threads per chain in k_sweep_reg
    int32_t n_chains;
    int32_t chain_base;          // first storage slot of this architecture in the system
    int32_t rng_base;            // random-stream id of its first chain: chain_base, or for a chain
                                 // shard the id that chain has in the whole system
    int64_t bead_base;           // first bead of this architecture in the system arrays
    float init_sigma;
};

struct SysDev {
    float* x;
    float* y;
    float* z;
    uint32_t* chain_id;
    uint32_t* counts[2];
    float* omega;
    int64_t n_cells;
    int64_t n_beads;
    int32_t n_types, nx, ny, nz;
    float inv_dx, inv_dy, inv_dz, scale;
    float lx, ly, lz;
    float k, k2, A, R;
    float cdeg[kMaxDeg + 1];    // c = 2k deg
    float ac4deg[kMaxDeg + 1];  // A c / 4
    float cf[kMaxTypes * kMaxTypes];
    int32_t hamiltonian, field_rule, count16, n_arch;
    uint32_t seed_lo, seed_hi;
    // mutable state
    uint32_t step;        // completed sweeps
    uint32_t cur;         // counts[cur] holds the counts of the current positions
    uint32_t error_word;
    uint32_t pad0;
    unsigned long long slot_acc[kSlots];  // accepted moves of the running sweep, cleared by k_close
    // statistics of the last completed sweep
    unsigned long long last_accepts, total_accepts, total_moves;
    double e_bond, e_field;
    uint32_t e_bond_step;  // step at which e_bond was last computed (+1; 0 = never)
    uint32_t pad1;
    // time-averaged density (io.cpp:57-94): the fused sweep adds the new counts
    // into avg at every sweep s with s % avg_every == 0 (avg NULL = off)
    unsigned long long* avg;         // [n_types * n_cells]
    unsigned long long avg_samples;  // sweeps accumulated
    uint32_t avg_every;
    uint32_t field_done;  // field tiles of the running launch finished (the last one closes the sweep)
    // fused sweeps leave the system alone once step reaches stop_step (the
    // served form gives each request its own sweep count inside a shared
    // round); 0xFFFFFFFF everywhere else
    uint32_t stop_step;
    uint32_t pad2;
    // counts the field step reads: NULL means counts[cur] (the grid of this
    // system's own beads); a chain shard points it at the sum over all shards
    const uint32_t* field_counts;
    // the span of omega: every field step folds the largest and smallest
    // non-NaN omega of its cells into om_max_key / om_min_key (order-preserving
    // integer keys, reset by the block that closes the step) and publishes
    // omega_span = max - min, so that omega_t[a] - omega_t[b] >= -omega_span for
    // any two cells of a type.  The move kernels use it to reject trials
    // without reading omega; +inf (after creation, scmf_set_omega or a
    // checkpoint read) disables that until the next field step.
    uint32_t om_max_key, om_min_key;
    float omega_span;
    uint32_t pad3;
    // the statistics of the last sweep in the public layout, written by
    // k_stats_out for asynchronous reads (scmf_step_stats_async)
    scmf_stats stats_out;
};

// Work item of the move / grid kernel: a run of whole chains of one architecture.
struct MoveTile {
    SysDev* sys;
    const ArchDev* arch;
    int32_t chain0;       // first storage slot (system-wide chain index)
    int32_t n_chains;
    int64_t bead0;        // first bead (system arrays)
    int32_t n_tiles_sys;  // move tiles of this system in the launch
    int32_t arch_index;   // architecture of the tile within its system
};

// Work item of the field kernel: a run of cells of one system.
struct FieldTile {
    SysDev* sys;
    int64_t cell0;
    int32_t n_cells;
    int32_t n_tiles_sys;  // field tiles of this system in the launch
    int32_t first_tile;   // index of this system's first field tile in the launch
    int32_t pad;
};

enum SweepMode : int { kMoveOnly = 0, kMoveGrid = 1, kGridOnly = 2 };

// What k_close does for each system of a launch.
enum CloseMode : int {
    kCloseMove = 1, kCloseField = 2, kCloseBond = 4, kCloseAdvance = 16,
    kCloseAverage = 32,  // count a time-averaged density sample when the sweep took one
    kSweepClose = kCloseMove | kCloseField | kCloseAdvance | kCloseAverage
};

// Per-tile partial sums of the chain observables (k_observables), each over
// the chains of one move tile, in double.
enum ObsSlot : int {
    kObsRe = 0,     // end-to-end vector components squared, x y z (first to last bead)
    kObsRg = 3,     // radius of gyration components squared
    kObsBond = 6,   // bond vector components squared, summed over bonds
    kObsMsd = 9,    // bead displacement from the reference snapshot, squared
    kObsMsdCom = 12,  // chain centre-of-mass displacement, squared
    kObsSlots = 16
};

// The tile ranges of one system in a launch's work lists.
struct SysClose {
    SysDev* sys;
    int32_t move_first, move_count;
    int32_t field_first, field_count;
};

// Launchers (scmf_kernels.cu).  Every pointer is device memory.
// Round keys of Philox4x32-10 for one 64-bit key: round r XORs in
// (k0 + r * 0x9E3779B9, k1 + r * 0xBB67AE85) (mod 2^32).  Passed to a kernel
// by value, the schedule sits in the parameter constant bank, so each round's
// XOR reads its key there instead of advancing two key registers.
struct PhiloxKeys {
    uint32_t k[20];  // k[2r], k[2r + 1]: the two key words of round r
};

inline PhiloxKeys philox_schedule(uint32_t k0, uint32_t k1) {
    PhiloxKeys s;
    for (int r = 0; r < 10; ++r) {
        s.k[2 * r] = k0;
        s.k[2 * r + 1] = k1;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return s;
}

enum KeyMode { kKeysNone = 0, kKeysHigh = 1, kKeysBoth = 2 };

// Move constants of the one system of a launch, passed by value so that the
// single-system move kernel reads them from the parameter constant bank
// (instruction operands) instead of loading them from SysDev into registers.
// Fixed for the life of the system: device buffers and spec constants.
// One architecture of the system the lean move kernel moves: linear chains of
// an even length with length / 2 dividing 32.
struct LeanArch {
    const uint8_t* types;  // [length], monomer type per bead
    int32_t length;
    int32_t n_chains;
    int32_t chain0;        // first chain (index into chain_id)
    int32_t bead0;         // first bead
    int32_t rng0;          // random-stream id of the first chain (chain_id[chain0 + c] = rng0 + c)
    int32_t pad;
};
constexpr int kLeanMaxArch = 4;

struct SysConsts {
    float* x;
    float* y;
    float* z;
    const uint32_t* chain_id;
    const float* omega;
    int64_t n_cells;
    float k2, A, R, inv_dx, inv_dy, inv_dz;
    int32_t nx, ny, nz, pad;
    float cdeg[3], ac4deg[3];  // c = 2k deg and A c / 4 for 0, 1, 2 bonds
    SysDev* sys;
    int32_t n_arch, pad2;
    LeanArch arch[kLeanMaxArch];
};

struct LaunchShape {
    int blocks;    // 0 = one CTA per tile
    int threads;
    int smem;      // unused by the launchers (they size shared memory themselves)
    int n_types;   // field kernel: monomer types shared by all systems, 0 = mixed
    int linear;    // sweep kernel: every architecture is a linear chain
    int max_chains;  // sweep kernel: most chains in one tile
    // sweep kernel, linear chains of at most 64 beads: tiles whose ceil(L/2)
    // does not divide 32 (chains laid across warps) and the others, as lists
    // of tile indices; n_flat == 0 means every tile is a warp tile
    const int32_t* flat_list;
    int n_flat;
    const int32_t* warp_list;
    int n_warp;
    int part;        // 0: every tile; 1: warp tiles only; 2: flat tiles only
    int fold;        // 0: every system's grid axes are powers of two (mask-only fold)
    int flat_threads;  // block size of the block-wide launch (0: threads)
    // sweep kernel: kKeysBoth when every system of the launch has the seed of
    // `keys`, kKeysHigh when they share its upper 32 bits, else kKeysNone
    int keyed;
    PhiloxKeys keys;
    // the launch moves one system (constants `sc`) whose architectures are all
    // linear chains of an even length L <= 64 with L/2 dividing 32, on a grid of
    // power-of-two axes, with fewer than 2^31 beads: the lean move kernel runs
    int lean;
    SysConsts sc;
    // every architecture whose chains fill warps exactly (ceil(L/2) divides 32)
    // has an even length: those tiles run k_sweep_leanm
    int warp_even;
};

// Streaming multiprocessors of the current device (read once per device; 148
// on a B200), for grid and tile sizing.
int sm_count();

int launch_init_coords(SysDev* d_sys, const ArchDev* d_arch, int n_arch, int n_chains, void* stream);
// Writes the statistics of the last sweep into d_sys->stats_out (one thread).
int launch_stats_out(SysDev* d_sys, void* stream);
// Copies the current counts (counts[cur], 32-bit words) into dst.
int launch_copy_counts(const SysDev* d_sys, uint32_t* dst, int64_t n_words, void* stream);
// Move kernels add their accept counts into SysDev::slot_acc (32-way spread);
// the field kernel writes one energy per tile into ef_part, the bond-energy
// kernel one per move tile into eb_part; k_close sums and publishes them.
int launch_sweep(int mode, const MoveTile* tiles, int n_tiles, int max_tile_beads, int max_length,
                 LaunchShape shape, unsigned* acc_part, void* stream);
// close_mode != 0: the last field tile of every system closes it in the same
// launch (what k_close does with that mode), so a sweep is two launches.
int launch_field(bool fused, int force_update, const FieldTile* tiles, int n_tiles, LaunchShape shape,
                 double* ef_part, int close_mode, void* stream);
int launch_bond_energy(const MoveTile* tiles, int n_tiles, LaunchShape shape, double* eb_part, void* stream);
int launch_close(const SysClose* list, int n_sys, const unsigned* acc_part, int warps_per_tile,
                 const double* ef_part, const double* eb_part, int mode, void* stream);
int launch_aos_to_soa(const float* aos, SysDev* sys, const ArchDev* arch, int n_arch, int64_t n_beads,
                      void* stream);
// Storage beads [i0, i1) from AoS positions (storage order = chain order: the
// AoS bead of storage bead i is bead i), then their counts added into
// counts[0] (a cleared buffer): one chunk of a chunked coordinate upload.
int launch_aos_chunk(const float* aos, SysDev* sys, const ArchDev* arch, int n_arch, int64_t i0, int64_t i1,
                     void* stream);
int launch_soa_to_aos(float* aos, const SysDev* sys, const ArchDev* arch, int n_arch, int64_t n_beads,
                      void* stream);
int launch_unpack_counts16(const SysDev* sys, uint32_t* out, int64_t n, void* stream);
// Validation (scmf_validate): out[0] += non-finite positions, out[1] +=
// positions beyond the exact fold range; out[2] += differing count words of
// a and b, out[3] += non-finite omega; sums[t] += counts of type t.
int launch_validate_positions(const SysDev* sys, int64_t n_beads, unsigned long long* out, void* stream);
int launch_validate_cells(const SysDev* sys, const uint32_t* a, const uint32_t* b, int64_t n_words,
                          int64_t n_values, unsigned long long* out, unsigned long long* sums, void* stream);
// Adds the current counts into SysDev::avg and counts one sample.
int launch_average_sample(SysDev* sys, int64_t n, void* stream);
// Chain observables: kObsSlots partial sums per move tile into part; ref_xyz
// is the SoA reference snapshot (x, then y, then z; NULL = no displacements).
int launch_observables(const MoveTile* tiles, int n_tiles, const float* ref_xyz, int64_t n_beads_sys,
                       double* part, void* stream);
size_t sweep_smem_bytes(int max_tile_beads, int max_length);
// Field coefficients cf[t + n*s] in FP32 from xn[t + n*s] (double): diagonal
// xn/N_ref; off-diagonal -xn/(2 N_ref) (SCMF0) or xn/N_ref (literal).
void field_coefficients(int n, const double* xn, int nref, int hamiltonian, float* cf);
// Sets the thread's last-error message (scmf_engine.cpp); returns code.
scmf_status fail(scmf_status code, const char* fmt, ...);
int configure_kernels();
int launch_debug_math(uint32_t k0, uint32_t k1, int n, uint32_t* words, float* logs, float* normals, void* stream);

}  // namespace scmf
