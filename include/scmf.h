/*
 * scmf.h - C ABI of the B200 single-chain-in-mean-field (SCMF) polymer Monte
 * Carlo engine (libscmf.so).
 *
 * The reference (ren5885a/New_arch) has no plugin or FFI layer: its boundary is
 * a set of blocking host C++ functions that mutate a managed-memory `Phase`
 * struct, plus its file surface (configuration.dat, polymer.dat,
 * density_<step>.dat, coord.dat, out.vtk).  Each entry point below names the
 * reference function or file it replaces.
 *
 * Conventions
 *   - Every function returns scmf_status: 0 = ok, negative = error; the message
 *     of the last error on the calling thread is returned by scmf_last_error().
 *   - Plain pointers and sizes only.  Host buffers are owned by the caller;
 *     getters copy into them.  A system owns all of its device memory (no
 *     managed memory).
 *   - A system handle is not thread-safe.  The server is thread-safe for
 *     submit and poll.
 *   - Positions cross the ABI in the reference's AoS layout (x,y,z per bead,
 *     beads of one chain contiguous, chains grouped by architecture in the
 *     order they were added; init_config.cu:753, device_function.cu:104-114).
 *   - Counts and omega are laid out [type][z][y][x] (device_function.cuh:17-20,
 *     device_function.cu:359).
 */
#ifndef SCMF_H
#define SCMF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t scmf_status;

#define SCMF_OK 0
#define SCMF_E_INVALID (-1)   /* bad argument or size */
#define SCMF_E_CUDA (-2)      /* CUDA runtime error or no device */
#define SCMF_E_NOMEM (-3)     /* device or host allocation failed / over budget */
#define SCMF_E_IO (-4)        /* file could not be opened or written */
#define SCMF_E_PARSE (-5)     /* malformed configuration.dat / polymer.dat / coord.dat */
#define SCMF_E_STATE (-6)     /* call not allowed in the current state */
#define SCMF_E_TIMEOUT (-7)   /* a bounded wait ran out */
#define SCMF_E_DEVICE (-8)    /* a kernel reported an error word */
#define SCMF_E_CANCELLED (-9) /* a served request was cancelled before it finished */

#define SCMF_MAX_TYPES 8      /* monomer types */
#define SCMF_MAX_DEGREE 8     /* bonds per bead */
#define SCMF_MAX_LENGTH 4096  /* beads per chain */

/* hamiltonian */
#define SCMF_HAM_SCMF0 0      /* reference SCMF0, device_function.cu:373-412 */
#define SCMF_HAM_LITERAL 1    /* omega_T = [kN (sum phi - 1) + sum_{S!=T} chiN_TS phi_S] / N_ref */
/* field_rule */
#define SCMF_FIELD_REFERENCE 0  /* omega not recomputed when step % 10 == 0 (test.cpp:42) */
#define SCMF_FIELD_EVERY 1      /* omega recomputed after every sweep */

const char* scmf_last_error(void);
const char* scmf_version(void);

/* ------------------------------------------------------------------ spec */
/* A system specification: box, grid, interactions and polymer
 * architectures.  Replaces Read_polymer_config + initialize_values
 * (init_config.cu:210-451, 455-736) and their derived constants. */
typedef struct scmf_spec scmf_spec;

typedef struct scmf_params {
    int32_t reference_nbeads;  /* N_ref ("Polymer length unit", init_config.cu:267) */
    double harmonic_normb;     /* k of the harmonic bond energy k |r_i - r_j|^2 (init_config.cu:484) */
    double smc_a;              /* smart-MC A; R = sqrt(2A) (init_config.cu:807-808) */
    uint64_t seed;             /* Philox key */
    int32_t hamiltonian;       /* SCMF_HAM_* */
    int32_t field_rule;        /* SCMF_FIELD_* */
    int32_t count_bits;        /* 32, or 16 (only when total beads < 65536) */
    int32_t reserved;
} scmf_params;

typedef struct scmf_spec_info {
    int64_t n_beads;
    int64_t n_cells;
    int32_t n_chains;
    int32_t n_types;
    int32_t n_arch;
    int32_t nx, ny, nz;
    double lx, ly, lz;
    double field_scaling;      /* n_cells / n_beads (init_config.cu:785) */
    double harmonic_normb, smc_a, smc_r;
    int32_t reference_nbeads;
    int32_t count_bits;
} scmf_spec_info;

scmf_status scmf_spec_create(int32_t n_mono_types, int32_t nx, int32_t ny, int32_t nz,
                             double lx, double ly, double lz, scmf_spec** out);
/* xn[t + n*s] as in Phase_info_gpu::xn (init_config.cu:670-672): diagonal
 * kappaN, off-diagonal chiN. */
scmf_status scmf_spec_set_xn(scmf_spec* spec, const double* xn, int32_t n);
scmf_status scmf_spec_set_params(scmf_spec* spec, const scmf_params* p);
/* Adds n_chains chains of one architecture: mono_type[length], bonds as
 * n_bonds (i,j) pairs.  init_sigma <= 0 selects the reference's per-component
 * initial bond sigma 1/sqrt(3(length-1)) (device_function.cu:169-171). */
scmf_status scmf_spec_add_arch(scmf_spec* spec, int32_t length, int32_t n_chains,
                               const int32_t* mono_type, int32_t n_bonds, const int32_t* bonds,
                               double init_sigma);
/* Reference input files: configuration.dat (init_config.cu:487-512) and
 * polymer.dat (init_config.cu:214-340), parsed by the same literal patterns.
 * Derived constants follow init_config.cu:480-484, 807-808. */
scmf_status scmf_spec_load_files(const char* configuration_dat, const char* polymer_dat,
                                 uint64_t seed, scmf_spec** out);
scmf_status scmf_spec_get_info(const scmf_spec* spec, scmf_spec_info* out);
scmf_status scmf_spec_get_params(const scmf_spec* spec, scmf_params* out);
scmf_status scmf_spec_get_xn(const scmf_spec* spec, double* xn, int32_t n);
/* Architecture idx: mono_type[length] and bonds[2*n_bonds] are copied when the
 * capacities (in elements) suffice; length / n_bonds are always returned. */
scmf_status scmf_spec_get_arch(const scmf_spec* spec, int32_t idx, int32_t* length, int32_t* n_chains,
                               int32_t* mono_type, int32_t type_cap, int32_t* bonds, int32_t bond_cap,
                               int32_t* n_bonds, double* init_sigma);
scmf_status scmf_spec_copy(const scmf_spec* spec, scmf_spec** out);
void scmf_spec_destroy(scmf_spec* spec);

/* ---------------------------------------------------------------- system */
typedef struct scmf_system scmf_system;

typedef struct scmf_stats {
    uint64_t step;            /* completed sweeps */
    uint64_t last_accepts;    /* accepted moves in the last sweep */
    uint64_t total_accepts;
    uint64_t total_moves;
    double e_bond;            /* sum over bonds of k |r_i - r_j|^2 after the last sweep */
    double e_field;           /* sum_T sum_cells omega_T n_T after the last field step */
    uint32_t error_word;      /* nonzero if a kernel flagged an error */
    uint32_t reserved;
} scmf_stats;

/* Allocates and owns all device memory of the system (initialize_structure_GPU,
 * init_config.cu:737-854).  cuda_stream may be NULL for a private stream. */
scmf_status scmf_system_create(const scmf_spec* spec, void* cuda_stream, scmf_system** out);

/* ---------------------------------------------------- chain shards (one system on several GPUs)
 * The reference spreads one system's chains over GPUs (init_config.cu:220-222), sums the per-GPU
 * int density counts by P2P copies and MPI_Allreduce (mesh.cu:10-81, mesh_mpi.cpp:16) and gives
 * every GPU the summed field (mesh.cu:191-215).  A chain shard is that per-GPU part: chains
 * [first[a], first[a] + count[a]) of every architecture a (scmf_shard_chains), each keeping the
 * random stream of its id in the whole system, with the whole system's field scaling.  One sweep:
 *   scmf_shard_move(shard, d_partial)        moves the shard's beads; its counts (the grid of its own
 *                                            beads) are copied to d_partial
 *   all-reduce (sum) of d_partial over the shards, by the caller (NCCL over NVLink, or any sum)
 *   scmf_shard_field(shard, d_sum, 1)        omega of the summed counts (the same on every shard),
 *                                            the field energy, and the close of the sweep
 * After scmf_shard_init_coords(shard, d_partial) and the sum, scmf_shard_field(shard, d_sum, 0)
 * computes the starting field.  Positions, summed counts and omega are bit-identical to the whole
 * system's; accepted moves and bond energies are per shard (their sum is the system's).  Buffers
 * are n_types * n_cells uint32 words in device memory; every call is enqueued on the shard's stream
 * (order the caller's sum on that stream).  A shard refuses the whole-system step, init, coordinate,
 * reference-shaped, batch and checkpoint calls, and needs 32-bit counts. */
scmf_status scmf_system_create_shard(const scmf_spec* spec, int32_t shard, int32_t n_shards, void* cuda_stream,
                                     scmf_system** out);
/* first[a], count[a]: the chains of architecture a that shard `shard` of n_shards holds (host only). */
scmf_status scmf_shard_chains(const scmf_spec* spec, int32_t shard, int32_t n_shards, int32_t* first, int32_t* count,
                              int32_t n_arch);
scmf_status scmf_shard_init_coords(scmf_system* shard, uint32_t* d_partial);
scmf_status scmf_shard_move(scmf_system* shard, uint32_t* d_partial);
scmf_status scmf_shard_field(scmf_system* shard, const uint32_t* d_total, int32_t close_sweep);
/* A system that still belongs to a batch is freed when the last such batch is
 * destroyed; its handle must not be used after this call either way. */
void scmf_system_destroy(scmf_system* sys);
scmf_status scmf_system_get_info(const scmf_system* sys, scmf_spec_info* out);
scmf_status scmf_system_stream(const scmf_system* sys, void** cuda_stream);
/* Random-walk initial coordinates (initialize_coord, device_function.cu:140-207),
 * followed by the initial grid and field (test.cpp:21-23). */
scmf_status scmf_init_coords(scmf_system* sys);
/* Restart from host coordinates, AoS float[3*n_beads] (Generate_init_coord with
 * read_file=1, init_config.cu:930-987), followed by the initial grid + field. */
scmf_status scmf_set_coords(scmf_system* sys, const float* xyz, size_t n_floats);
scmf_status scmf_get_coords(const scmf_system* sys, float* xyz, size_t n_floats);
scmf_status scmf_set_step(scmf_system* sys, uint64_t step);   /* -Start_time (init.cpp:33) */
/* n_sweeps full MC steps: move -> grid -> field, the field skipped per the
 * field rule.  Replaces the body of the loop at test.cpp:37-43. */
scmf_status scmf_step(scmf_system* sys, int32_t n_sweeps);
/* The same, enqueued on the system's stream without waiting (for graphs of
 * the caller's own work and for timing with events on that stream). */
scmf_status scmf_step_async(scmf_system* sys, int32_t n_sweeps);
/* n_sweeps full MC steps enqueued kernel by kernel (no graph) with CUDA
 * events around every launch on the system's stream; returns after the last
 * sweep with the summed device time of the fused move+grid kernel, of the
 * field kernel, and the device time from the first launch to the end of the
 * last (milliseconds).  Same results as scmf_step. */
scmf_status scmf_step_profiled(scmf_system* sys, int32_t n_sweeps, float* ms_move, float* ms_field, float* ms_total);
/* Reference-shaped pieces of one step (blocking, like the originals): */
scmf_status scmf_smc_move(scmf_system* sys, int32_t n_sweeps);          /* smc_move, smc.cu:3-72 */
scmf_status scmf_reset_density_fields(scmf_system* sys);                /* reset_density_fields, mesh.cu:161-190 */
scmf_status scmf_update_omega_fields_scmf0(scmf_system* sys);           /* update_omega_fields_scmf0, mesh.cu:217-248 */
scmf_status scmf_synchronize(scmf_system* sys);
scmf_status scmf_get_counts(const scmf_system* sys, uint32_t* out, size_t n);
scmf_status scmf_get_omega(const scmf_system* sys, float* out, size_t n);
scmf_status scmf_set_omega(scmf_system* sys, const float* in, size_t n);
scmf_status scmf_get_stats(const scmf_system* sys, scmf_stats* out);
/* The statistics a sweep produces by itself (step, accepts, field energy) in
 * one small device-to-host read; e_bond is NaN unless it is current (it is
 * computed on demand by scmf_get_stats). */
scmf_status scmf_get_sweep_stats(const scmf_system* sys, scmf_stats* out);
/* scmf_step followed by scmf_get_sweep_stats with one device read and one
 * wait: the loop of a driver that reports every sweep (test.cpp:45-68 prints
 * per check step) costs one host round trip per call instead of three. */
scmf_status scmf_step_stats(scmf_system* sys, int32_t n_sweeps, scmf_stats* out);
/* The same without waiting: the sweeps and a copy of their statistics into
 * *host_out are enqueued on the system's stream, and *host_out is valid after
 * the next scmf_synchronize (or any other wait on that stream).  host_out
 * should be page-locked host memory (cudaHostAlloc / cudaHostRegister) for the
 * copy to run asynchronously, and must stay valid until then.  e_bond is NaN,
 * as in scmf_get_sweep_stats. */
scmf_status scmf_step_stats_async(scmf_system* sys, int32_t n_sweeps, scmf_stats* host_out);

/* Diagnostics: evaluates the device arithmetic (Philox4x32-10 with counter
 * (c0,c1,c2,c3) = (i, 0, 0, 0) and the given key, then log(u01(w.w)), the
 * Metropolis logarithm, and the three inverse-CDF normals of w.x, w.y, w.z)
 * for i < n on the GPU, for comparison with any host restatement.
 * words[4*n] (raw), logs[n], normals[3*n]. */
scmf_status scmf_debug_math(uint32_t key_lo, uint32_t key_hi, int32_t n, uint32_t* words, float* logs,
                            float* normals);

/* Field update that allocates nothing.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc: code that must not allocate while
 * it runs (work replayed inside a stream capture owned by someone else, a
 * latency-critical loop where an allocation could stall), or an application
 * that owns every byte of device memory and passes only pointers to its own
 * buffers.  It computes omega (SCMF0 or literal, as scmf_update_omega_fields_scmf0)
 * from caller-owned device counts d_counts[n_types*n_cells] into caller-owned
 * d_omega, and the field energy sum_T sum_cells omega_T n_T into the device
 * double *d_energy, enqueued on `stream`.  Its only scratch, the per-tile
 * energy partials, is a fixed array in the library's device memory: at most
 * 8,388,608 cells (2048 tiles of 4096); larger grids are rejected with
 * SCMF_E_INVALID.  Every GPU that loads the library holds that 16 KiB until
 * the process exits.  The first call in a device's context looks the array's
 * address up (cudaGetSymbolAddress) and keeps it with that context's id; the
 * first call after the context was re-created (cudaDeviceReset, or a primary
 * context released and retained again) looks it up anew.  Make those first
 * calls before any stream capture.  There is one array per device, shared by
 * every call on that device, and each call overwrites it: calls on the same
 * device that overlap on the GPU (from any stream or any host thread) race;
 * calls on different devices do not. */
scmf_status scmf_update_omega_noalloc(const uint32_t* d_counts, float* d_omega, int32_t n_types, int64_t n_cells,
                                      double field_scaling, const double* xn, int32_t reference_nbeads,
                                      int32_t hamiltonian, double* d_energy, void* stream);

/* --------------------------------------------------------------- output */
/* density_<step>.dat writer (io_out_density, io.cpp:4-56).  path NULL uses the
 * reference's file name rule in the current directory. */
scmf_status scmf_write_density(const scmf_system* sys, const char* path, int64_t step);
/* coord.dat writer (io_out_coord, io.cpp:95-118). */
scmf_status scmf_write_coords(const scmf_system* sys, const char* path);
/* coord.dat reader: skips skip_beads lines (init_config.cu:955-959), then reads
 * n_beads "%lg %lg %lg" lines into xyz (AoS float). */
scmf_status scmf_read_coords_file(const char* path, int64_t skip_beads, float* xyz, size_t n_floats);
/* density file -> out.vtk STRUCTURED_POINTS of phi_0 - phi_1 (vtk.c:4-81).
 * values_per_point = 6 reproduces vtk.c exactly (it reads six numbers per
 * grid point whatever the type count); 0 takes 2*n_types from the file. */
scmf_status scmf_vtk_convert(const char* density_path, const char* vtk_path, int32_t values_per_point);

/* ---------------------------------------------------- time-averaged density
 * Replaces average_field_unified (struct.h:234, allocated at
 * init_config.cu:770 and never filled) and io_out_aver_density (io.cpp:57-94).
 * While averaging is on, every sweep s with s % every == 0 adds the counts of
 * its final positions into a uint64 accumulator inside the fused field step
 * (no extra pass over the counts). */
/* every >= 1 starts (or restarts) averaging with a zeroed accumulator of
 * 8 * n_types * n_cells bytes; every = 0 stops it and frees the accumulator. */
scmf_status scmf_average_start(scmf_system* sys, uint32_t every);
/* Adds the current counts as one sample now (for drivers that call the
 * reference-shaped pieces instead of scmf_step). */
scmf_status scmf_average_sample(scmf_system* sys);
/* Sums [type][z][y][x] (n = n_types * n_cells) and the number of samples. */
scmf_status scmf_average_get(const scmf_system* sys, uint64_t* sums, size_t n, uint64_t* n_samples);
/* density_aver_<step>.dat (path NULL) in the density-file format: per cell the
 * mean phi_T = (sum_T / n_samples) * n_cells / n_beads of every type, then the
 * current omega_T, "%g " each. */
scmf_status scmf_write_average_density(const scmf_system* sys, const char* path, int64_t step);

/* ------------------------------------------------------------ checkpoints
 * A binary checkpoint holds everything the next sweep reads: positions (FP32,
 * bit for bit), omega, the step, the statistics and the averaging state, with
 * a checksum.  Reading it into a system of the same spec resumes the run
 * exactly (the random stream is stateless: it depends only on seed, chain,
 * bead and step).  Counts are recomputed from the positions on reading.  The
 * reference's restart (read_file=1, init_config.cu:930-987) goes through the
 * lossy "%g" coord.dat and recomputes omega, so it does not resume exactly. */
/* File layout (little endian): the 8 bytes "SCMFCKPT", this 128-byte header,
 * then the payload: positions float[3 * n_beads] (AoS, the order of
 * scmf_get_coords), omega float[n_types * n_cells], and when avg_every > 0 the
 * accumulator uint64[n_types * n_cells]. */
typedef struct scmf_checkpoint_header {
    uint32_t version;         /* 1 */
    int32_t n_types, nx, ny, nz;
    int32_t n_chains, n_arch;
    uint32_t avg_every;       /* 0: no accumulator stored */
    int64_t n_beads;
    int64_t n_cells;
    uint64_t seed;
    uint64_t spec_hash;       /* hash of every spec field that changes a trajectory (seed aside) */
    uint64_t step;
    uint64_t last_accepts, total_accepts, total_moves;
    double e_field;
    uint64_t avg_samples;
    uint64_t payload_bytes;
    uint64_t payload_hash;    /* FNV-1a 64 of the payload bytes */
} scmf_checkpoint_header;
scmf_status scmf_checkpoint_write(const scmf_system* sys, const char* path);
scmf_status scmf_checkpoint_read(scmf_system* sys, const char* path);
/* Reads and checks the header (and the payload checksum) without a system. */
scmf_status scmf_checkpoint_info(const char* path, scmf_checkpoint_header* out);
/* spec_hash a checkpoint of systems of this spec carries. */
scmf_status scmf_spec_hash(const scmf_spec* spec, uint64_t* out);

/* ------------------------------------------------------------- validation
 * The reference has no sanitizer or checks (bounds printf()s and one trap,
 * device_function.cu:159-160, 490-502, 610, 646-651).  scmf_validate checks
 * the state on the device and reports instead of trapping: non-finite
 * positions, positions beyond the exact range of the FP32 cell fold
 * (|x / dx| >= 2^22 on some axis; the cell index stays in range but is no
 * longer the floor), count words differing from a fresh gridding of the
 * positions (counts are stale between scmf_smc_move and
 * scmf_reset_density_fields), per-type counts not summing to that type's
 * beads, and non-finite omega.  Returns SCMF_E_DEVICE when any is nonzero. */
typedef struct scmf_validation {
    uint64_t nonfinite_positions;
    uint64_t positions_out_of_range;
    uint64_t count_mismatch_words;   /* 32-bit words of the counts array (16-bit counts come in pairs) */
    uint64_t nonfinite_omega;
    int64_t count_sum_error;         /* sum over types of |sum of counts - beads of the type| */
    uint32_t error_word;             /* the kernels' error word */
    uint32_t reserved;
} scmf_validation;
scmf_status scmf_validate(scmf_system* sys, scmf_validation* out);

/* --------------------------------------------------------------- analysis
 * Chain observables as device reductions (double), per architecture: the
 * reference's end-to-end distance (test.cpp:47-68, beads 0 and 31 of every
 * chain) generalised to first/last bead of any length, and the analyses its
 * Ana_Info names (struct.h:65-75: Re, Rg, bond anisotropy, acceptance ratio,
 * MSD) which it never computes. */
typedef struct scmf_observables {
    int32_t arch;             /* architecture index */
    int32_t n_chains;
    int64_t n_beads;
    int64_t n_bonds;
    double re2[4];            /* <R_e,x^2>, <R_e,y^2>, <R_e,z^2>, <|R_e|^2> over chains */
    double rg2[4];            /* <R_g^2> components and total over chains */
    double bond2[4];          /* <b_x^2>, <b_y^2>, <b_z^2>, <|b|^2> over bonds */
    double msd[4];            /* bead <|r - r_ref|^2> components and total (NaN: no reference) */
    double msd_com[4];        /* chain centre-of-mass displacement, same form */
    double acc_ratio;         /* accepted / attempted moves of the last sweep (whole system) */
    double reserved[3];
} scmf_observables;
/* Takes the current positions as the reference for displacements. */
scmf_status scmf_analysis_reference(scmf_system* sys);
/* Fills out[0 .. n_arch-1]; n_arch must equal the system's architecture count. */
scmf_status scmf_analyze(const scmf_system* sys, scmf_observables* out, int32_t n_arch);

/* -------------------------------------------------------------- batched */
/* Many independent systems advanced together: one persistent kernel per
 * phase over a work list of (system, chain tile) and (system, cell tile),
 * captured once in a CUDA graph.  No reference counterpart (the reference runs
 * one system per process). */
typedef struct scmf_batch scmf_batch;

typedef struct scmf_tune {
    int32_t chains_per_tile;   /* 0 = per-architecture default */
    int32_t threads_move;      /* 0 = default */
    int32_t cells_per_tile;    /* 0 = default */
    int32_t threads_field;     /* 0 = default */
    int32_t persistent_ctas;   /* 0 = one CTA per tile (no persistence) */
    int32_t use_graph;         /* 1 = capture one sweep in a CUDA graph */
    int32_t beads_per_tile;    /* > 0: chains per tile = max(1, beads_per_tile / length) for each
                                  architecture (takes precedence over chains_per_tile) */
    int32_t reserved;
} scmf_tune;

scmf_status scmf_batch_create(scmf_system* const* systems, int32_t n, const scmf_tune* tune,
                              void* cuda_stream, scmf_batch** out);
scmf_status scmf_batch_step(scmf_batch* b, int32_t n_sweeps);
/* The same, enqueued on the batch's stream without waiting. */
scmf_status scmf_batch_step_async(scmf_batch* b, int32_t n_sweeps);
/* scmf_step_profiled for a batch: its sweeps launch by launch with CUDA events
 * on the batch's stream; the move time covers both move launches of a plan
 * that runs them side by side.  Same results as scmf_batch_step. */
scmf_status scmf_batch_step_profiled(scmf_batch* b, int32_t n_sweeps, float* ms_move, float* ms_field,
                                     float* ms_total);
/* Times candidate tunings on snapshots of the batch's systems (their state is
 * restored afterwards) and installs the fastest; *out receives it. */
scmf_status scmf_batch_autotune(scmf_batch* b, int32_t sweeps_per_trial, scmf_tune* out);
/* One tuning the last scmf_batch_autotune timed, with the device time of its
 * timed sweeps (milliseconds). */
typedef struct {
    scmf_tune tune;
    float ms;
    int32_t reserved;
} scmf_tune_trial;
/* The trials of the batch's last autotune in the order they ran: *n receives
 * their number, out[0 .. min(*n, max)) the trials.  No counterpart in the
 * reference (it has no batched form). */
scmf_status scmf_batch_tune_trials(const scmf_batch* b, scmf_tune_trial* out, int32_t max, int32_t* n);
scmf_status scmf_batch_get_tune(const scmf_batch* b, scmf_tune* out);
void scmf_batch_destroy(scmf_batch* b);
/* create + step + destroy */
scmf_status scmf_batch_run(scmf_system* const* systems, int32_t n, int32_t n_sweeps, const scmf_tune* tune);

/* --------------------------------------------------------------- served */
/* A request loop with continuous batching: requests are admitted as device
 * memory (against hbm_budget_bytes) and slots free up, state stays resident
 * on the device between sweeps, and requests that arrive while others run
 * join the next round.  No reference counterpart. */
typedef struct scmf_server scmf_server;

typedef struct scmf_server_opts {
    uint64_t hbm_budget_bytes;
    int32_t max_active;         /* 0 = unlimited */
    int32_t sweeps_per_round;   /* 0 = default */
    int32_t use_graph;
    int32_t reserved;
} scmf_server_opts;

typedef struct scmf_result {
    uint64_t id;
    scmf_status status;         /* SCMF_OK, SCMF_E_CANCELLED, or the error that ended the request */
    int32_t n_sweeps;           /* requested */
    double e_bond, e_field;
    uint64_t accepts;
    int64_t n_beads;
    double t_submit, t_admit, t_done;   /* seconds on the server's monotonic clock (t_admit 0: never admitted) */
    int32_t sweeps_done;
    int32_t reserved;
} scmf_result;

scmf_status scmf_server_create(const scmf_server_opts* opts, scmf_server** out);
/* The server copies the spec.  counts_out (optional, uint32[n_types*n_cells])
 * must stay valid until the result has been polled. */
scmf_status scmf_server_submit(scmf_server* s, const scmf_spec* spec, int32_t n_sweeps,
                               uint32_t* counts_out, uint64_t* id_out);
/* Up to max results; waits up to wait_ms for at least one. */
scmf_status scmf_server_poll(scmf_server* s, scmf_result* out, int32_t max, int32_t* n_out, int32_t wait_ms);
scmf_status scmf_server_pending(scmf_server* s, int32_t* queued, int32_t* active, uint64_t* bytes_in_use);
/* Cancels a request: a queued one leaves the queue at once, an active one at
 * the next round boundary (its device memory is freed); either way one result
 * with status SCMF_E_CANCELLED and the sweeps done so far is delivered.
 * SCMF_E_INVALID if the id is unknown or its result is already delivered. */
scmf_status scmf_server_cancel(scmf_server* s, uint64_t id);
/* Waits until no request is queued or active: SCMF_OK, or SCMF_E_TIMEOUT
 * after timeout_ms (the requests keep running). */
scmf_status scmf_server_drain(scmf_server* s, int32_t timeout_ms);
double scmf_server_now(const scmf_server* s);
/* Stops the server: queued requests are dropped, running ones stop at their
 * round boundary, their device memory is freed, and results not yet polled
 * are discarded.  Drain first (scmf_server_drain) to finish outstanding work. */
void scmf_server_destroy(scmf_server* s);

#ifdef __cplusplus
}
#endif
#endif /* SCMF_H */
