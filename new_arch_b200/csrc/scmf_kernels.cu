// sm_100a kernels of the SCMF engine.
//
//   k_init_coords   random-walk chains (device_function.cu:140-207)
//   k_sweep_reg     one MC sweep of linear chains of up to 64 beads, positions
//                   in registers (a thread per bead pair): odd/even half-sweeps
//                   of smart-MC trials (device_function.cu:444-454, 509-799),
//                   moving one cell count for each accepted move that leaves
//                   its cell, so counts stay the grid of the positions
//                   (device_function.cu:471-508); or, in kGridOnly, a gridding
//                   pass from scratch
//   k_sweep_lean    the same sweep for one system of even-length chains on a
//                   power-of-two grid, constants in the parameter bank
//   k_sweep_leanm   its structure for many systems / any grid (even lengths)
//   k_sweep_linear  the same for longer linear chains, staged per warp in
//                   shared memory
//   k_sweep         the same for any bond graph (graph-colour half-sweeps)
//   k_field<fused>  counts -> omega (SCMF0, device_function.cu:373-412) with the
//                   field-energy reduction; in the fused step the block that
//                   finishes a system's last tile closes the sweep (step,
//                   statistics, averaging sample)
//   k_close, k_bond_energy, k_observables, k_validate_*, transposes: the
//                   reductions and checks around the step
//
// Built with --fmad=false -prec-div=true -prec-sqrt=true: positions and counts
// are bit-identical to the CPU oracle, whatever the tiling or launch shape.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "scmf.h"

#include "scmf_internal.h"
#include "scmf_math.cuh"
#include "scmf_normal_table.h"

namespace scmf {

// The inverse normal CDF table of normal_of, read-only in global memory.
__device__ __align__(16) const float g_normal_tab[SCMF_NORMAL_SEGS * 4] = {SCMF_NORMAL_TABLE_DATA};

__device__ __forceinline__ const float4* normal_table() { return reinterpret_cast<const float4*>(g_normal_tab); }

// Copies the table into a block's shared memory (all threads of the block
// call it; a barrier follows).
__device__ __forceinline__ void load_normal_table(float4* s_tab) {
    for (int i = threadIdx.x; i < SCMF_NORMAL_SEGS; i += blockDim.x) s_tab[i] = __ldg(normal_table() + i);
    __syncthreads();
}

// i / n via a multiply-high by magic = ceil(2^32 / n) (exact while i * n < 2^32).
__device__ __forceinline__ uint32_t div_magic(uint32_t i, uint32_t magic, int n) {
    return n == 1 ? i : __umulhi(i, magic);
}

// ------------------------------------------------------------------ init
__global__ void k_init_coords(SysDev* __restrict__ S, const ArchDev* __restrict__ archs, int n_arch,
                              int n_chains) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n_chains) return;
    int a = 0;
    while (a + 1 < n_arch && g >= archs[a + 1].chain_base) ++a;
    const ArchDev& A = archs[a];
    const int L = A.length;
    const int64_t b0 = A.bead_base + (int64_t)(g - A.chain_base) * L;
    const uint32_t gid = (uint32_t)(A.rng_base + (g - A.chain_base));  // the chain's random-stream id
    float* X = S->x + b0;
    float* Y = S->y + b0;
    float* Z = S->z + b0;
    const uint32_t k0 = S->seed_lo, k1 = S->seed_hi;
    uint32_t placed[kMaxLength / 32];
    for (int i = 0; i < (L + 31) / 32; ++i) placed[i] = 0u;
    for (int i = 0; i < L; ++i) {
        X[i] = 0.0f;
        Y[i] = 0.0f;
        Z[i] = 0.0f;
    }
    uint4 w = philox4x32_10(make_uint4(gid, 0u, kInitStep, 0u), k0, k1);
    X[0] = u01(w.x) * S->lx;
    Y[0] = u01(w.y) * S->ly;
    Z[0] = u01(w.z) * S->lz;
    placed[0] = 1u;
    for (int i = 0; i < L; ++i) {
        const BeadInfo bi = A.beads[i];
        for (int d = 0; d < bi.deg; ++d) {
            const int j = bi.nbr[d];
            if (placed[j >> 5] & (1u << (j & 31))) continue;
            float n0, n1, n2;
            normals3(philox4x32_10(make_uint4(gid, (uint32_t)j, kInitStep, 1u), k0, k1), normal_table(), n0, n1, n2);
            X[j] = X[i] + A.init_sigma * n0;
            Y[j] = Y[i] + A.init_sigma * n1;
            Z[j] = Z[i] + A.init_sigma * n2;
            placed[j >> 5] |= 1u << (j & 31);
        }
    }
}

// ------------------------------------------------------------------ sweep
struct MoveConsts {
    float k, k2, A, R, inv_dx, inv_dy, inv_dz;
    float span;  // SysDev::omega_span of the system (early rejection)
    int nx, ny, nz;
    bool pow2;   // every axis a power of two
    bool small;  // every axis of 2 to 256 cells (fold_magic)
};

__device__ __forceinline__ bool is_pow2(int n) { return (n & (n - 1)) == 0; }

__device__ __forceinline__ void load_fold(MoveConsts& c, const SysDev* S) {
    c.span = S->omega_span;
    c.nx = S->nx; c.ny = S->ny; c.nz = S->nz;
    c.pow2 = is_pow2(c.nx) && is_pow2(c.ny) && is_pow2(c.nz);
    c.small = c.nx >= 2 && c.ny >= 2 && c.nz >= 2 && c.nx <= 256 && c.ny <= 256 && c.nz <= 256;
}

// Offsets and magic multipliers of fold_magic for n = 0 .. 256 (filled once
// per device by configure_kernels).  Every lane of a warp reads the entry of
// the same n, which the constant cache broadcasts.
__constant__ int2 c_fold[257];

// FOLD = 0: every system of the launch has power-of-two axes, so only the
// mask fold is compiled in; FOLD = -1 picks the fold per system at run time.
template <int FOLD = -1>
__device__ __forceinline__ int cell_of(const MoveConsts& c, float x, float y, float z) {
    int ix, iy, iz;
    if (FOLD == 0 || c.pow2) {
        ix = fold_pow2(x, c.inv_dx, c.nx - 1);
        iy = fold_pow2(y, c.inv_dy, c.ny - 1);
        iz = fold_pow2(z, c.inv_dz, c.nz - 1);
    } else if (c.small) {
        const int2 fx = c_fold[c.nx], fy = c_fold[c.ny], fz = c_fold[c.nz];
        ix = fold_magic(x, c.inv_dx, c.nx, fx.x, (uint32_t)fx.y);
        iy = fold_magic(y, c.inv_dy, c.ny, fy.x, (uint32_t)fy.y);
        iz = fold_magic(z, c.inv_dz, c.nz, fz.x, (uint32_t)fz.y);
    } else {
        ix = fold(x, c.inv_dx, c.nx);
        iy = fold(y, c.inv_dy, c.ny);
        iz = fold(z, c.inv_dz, c.nz);
    }
    return ix + c.nx * (iy + c.ny * iz);
}


// Bond force f = 2k sum_j (q_j - p), one neighbour at a time in ascending
// bead order (fma per neighbour, as the oracle).
__device__ __forceinline__ void add_bond(float k2, float x, float y, float z, float qx, float qy, float qz, float& fx,
                                         float& fy, float& fz) {
    fx = __fmaf_rn(__fsub_rn(qx, x), k2, fx);
    fy = __fmaf_rn(__fsub_rn(qy, y), k2, fy);
    fz = __fmaf_rn(__fsub_rn(qz, z), k2, fz);
}

// Rejection before the omega reads.  Every field step publishes span >= the
// largest omega_t[a] - omega_t[b] (SysDev::omega_span), so, rounding being
// monotone, fl(w_new - w_old) >= -span and dE = fl(fl(w_new - w_old) + deb) >=
// fl(deb - span) =: lb.  A trial with -lb <= log_lower(u) <= log_f(u) has
// dE > 0 and log_f(u) >= -dE: the Metropolis test below rejects it whatever
// omega holds (and a NaN bound or energy rejects, as the test does).  At the
// benchmark acceptance (~0.5 %) about 2 % of trials pass this bound, so about
// half of the warps skip the cell folds, the two gathers and their L2 round
// trip altogether; the outcome of every trial is the oracle's.
__device__ __forceinline__ bool maybe_accepted(float deb, float span, float lf) {
    return -__fsub_rn(deb, span) > lf;
}

// The trial of a bead at (x,y,z) with bond force f.  With d = A f + R xi the
// displacement, the reference's bonded energy change plus smart-MC correction
// equals (A c / 4)(c |d|^2 - 2 f.d), c = 2k deg (the force at p + d is
// f - c d).  Same FP32 expression (explicit fma) as the oracle's move_bead().
// Returns whether the move is accepted; (px,py,pz) is the proposed position
// and cell_old / cell_new the cells of the old and proposed positions.
template <int FOLD = -1>
__device__ __forceinline__ bool trial_f(const MoveConsts& c, float x, float y, float z, float fx, float fy, float fz,
                                        float cc, float ac4, float n0, float n1, float n2, uint32_t aw,
                                        const float* __restrict__ w_t, float& px, float& py, float& pz, int& cell_old,
                                        int& cell_new) {
    const float A = c.A, R = c.R;
    const float dx = __fmaf_rn(A, fx, __fmul_rn(R, n0));
    const float dy = __fmaf_rn(A, fy, __fmul_rn(R, n1));
    const float dz = __fmaf_rn(A, fz, __fmul_rn(R, n2));
    px = __fadd_rn(x, dx);
    py = __fadd_rn(y, dy);
    pz = __fadd_rn(z, dz);
    const float d2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
    const float fd = __fmaf_rn(fx, dx, __fmaf_rn(fy, dy, __fmul_rn(fz, dz)));
    const float deb = __fmul_rn(ac4, __fmaf_rn(cc, d2, __fmul_rn(-2.0f, fd)));
    // Trials that the omega span already rejects skip the folds and gathers
    // (maybe_accepted; same outcome).  Otherwise: log(u) >= -23 ln2 > -17 for
    // every u the generator yields, so dE >= 17 rejects without the logarithm;
    // below that, log_f(u) >= log_lower(u) for every such u, so
    // -dE <= log_lower(u) rejects without it too (same outcome).
    bool acc = false;
    int c_old = 0, c_new = 0;
    if (maybe_accepted(deb, c.span, log_lower(u01(aw)))) {
        c_old = cell_of<FOLD>(c, x, y, z);
        c_new = cell_of<FOLD>(c, px, py, pz);
        const float dE = __fadd_rn(__fsub_rn(__ldg(w_t + c_new), __ldg(w_t + c_old)), deb);
        if (dE < 0.0f)
            acc = true;
        else if (dE < 17.0f)
            acc = -dE > log_lower(u01(aw)) && log_f(u01(aw)) < -dE;  // u recomputed: no register held across
    }
    cell_old = c_old;
    cell_new = c_new;
    return acc;
}

// One smart-MC trial (device_function.cu:637-717, 562-588, 444-454) of a bead
// at (x,y,z) with deg bonded neighbours q[0..deg) in ascending bead order.
template <int MAXDEG, int FOLD = -1>
__device__ __forceinline__ bool trial(const MoveConsts& c, float x, float y, float z, const float* qx,
                                      const float* qy, const float* qz, int deg, float cc, float ac4, float n0,
                                      float n1, float n2, uint32_t aw, const float* __restrict__ w_t, float& px,
                                      float& py, float& pz, int& cell_old, int& cell_new) {
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
#pragma unroll
    for (int d = 0; d < MAXDEG; ++d)
        if (d < deg) add_bond(c.k2, x, y, z, qx[d], qy[d], qz[d], fx, fy, fz);
    return trial_f<FOLD>(c, x, y, z, fx, fy, fz, cc, ac4, n0, n1, n2, aw, w_t, px, py, pz, cell_old, cell_new);
}

// Counts are kept as the grid of the current positions: a fused sweep moves
// one count from the old to the new cell of every accepted move that leaves
// its cell (typ = type * n_cells), instead of regridding every bead.
__device__ __forceinline__ void count_move(uint32_t* cnt, bool c16, int64_t typ, int c_old, int c_new) {
    const int64_t io = typ + c_old, in = typ + c_new;
    if (c16) {
        atomicSub(cnt + (io >> 1), 1u << ((io & 1) * 16));  // the cell holds this bead: no borrow
        atomicAdd(cnt + (in >> 1), 1u << ((in & 1) * 16));
    } else {
        atomicSub(cnt + io, 1u);
        atomicAdd(cnt + in, 1u);
    }
}

// KEYS (KeyMode): kKeysBoth when every system of the launch has the seed whose
// Philox round keys are in `keys` (a kernel parameter); kKeysHigh when they
// share its upper 32 bits, so that only the first key word is read from the
// tile's SysDev and advanced round by round; kKeysNone: both are.
template <int KEYS>
__device__ __forceinline__ uint4 philox_block(uint4 ctr, uint32_t k0, uint32_t k1, const PhiloxKeys& keys) {
    if (KEYS == kKeysBoth) return philox4x32_10(ctr, keys);
    if (KEYS == kKeysHigh) return philox4x32_10(ctr, k0, keys);
    return philox4x32_10(ctr, k0, k1);
}

// Philox block and normals of bead b of chain gc; returns its Metropolis word.
template <int KEYS>
__device__ __forceinline__ uint32_t bead_normals(uint32_t gc, int b, uint32_t step, uint32_t k0, uint32_t k1,
                                                 const PhiloxKeys& keys, float& n0, float& n1, float& n2) {
    const uint4 w = philox_block<KEYS>(make_uint4(gc, (uint32_t)b, step, 0u), k0, k1, keys);
    normals3(w, normal_table(), n0, n1, n2);
    return accept_word(w);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

size_t sweep_smem_bytes(int max_tile_beads, int max_length) {
    size_t b = (size_t)max_tile_beads * 3 * sizeof(float);
    b = (b + 15) & ~(size_t)15;
    b += (size_t)max_length * sizeof(BeadInfo);
    b = (b + 15) & ~(size_t)15;
    b += (size_t)max_length * sizeof(uint16_t);
    return (b + 15) & ~(size_t)15;
}

// One MC sweep over tiles of whole chains staged in shared memory.
//   MODE kMoveOnly / kMoveGrid / kGridOnly: moves; moves keeping counts[cur]
//   the grid of the positions (accepted moves that change cell move a count);
//   counts of the current positions added into counts[cur] (a cleared buffer).
//   LINEAR: every architecture of the launch is a linear chain (bonds i-i+1,
//   even beads colour 0, odd beads colour 1); neighbours are computed, not looked up.
//   Two 256-thread CTAs per SM leave it 128 registers and no spill (at 64 it
//   spilled ~400 B per thread and moved combs 12 % slower).
template <int MODE, bool LINEAR, int KEYS>
__global__ void __launch_bounds__(256, 2) k_sweep(const MoveTile* __restrict__ tiles, int n_tiles,
                                                   int max_tile_beads, int max_length, unsigned* __restrict__ acc_part,
                                                   const PhiloxKeys keys) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* sx = reinterpret_cast<float*>(smem_raw);
    float* sy = sx + max_tile_beads;
    float* sz = sy + max_tile_beads;
    size_t off = ((size_t)max_tile_beads * 3 * sizeof(float) + 15) & ~(size_t)15;
    BeadInfo* sinfo = reinterpret_cast<BeadInfo*>(smem_raw + off);
    off = (off + (size_t)max_length * sizeof(BeadInfo) + 15) & ~(size_t)15;
    uint16_t* scol = reinterpret_cast<uint16_t*>(smem_raw + off);
    uint8_t* stype = reinterpret_cast<uint8_t*>(sinfo);  // LINEAR: types only
    const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5;
    for (int ti = blockIdx.x; ti < n_tiles; ti += gridDim.x) {
        const MoveTile t = tiles[ti];
        SysDev* S = t.sys;
        if (MODE != kGridOnly && S->step >= S->stop_step) continue;  // block-uniform
        const ArchDev* Ap = t.arch;
        const int L = Ap->length;
        const int nb = t.n_chains * L;
        if (nb > max_tile_beads || L > max_length) {
            if (tid == 0) atomicOr(&S->error_word, 1u);
            continue;
        }
        MoveConsts c;
        c.k = S->k; c.k2 = S->k2; c.A = S->A; c.R = S->R;
        c.inv_dx = S->inv_dx; c.inv_dy = S->inv_dy; c.inv_dz = S->inv_dz;
        load_fold(c, S);
        const uint32_t len_magic = Ap->len_magic;
        for (int i = tid; i < L; i += T) {
            if (LINEAR) {
                stype[i] = Ap->beads[i].type;
            } else {
                sinfo[i] = Ap->beads[i];
                scol[i] = Ap->color_beads[i];
            }
        }
        float* gx = S->x + t.bead0;
        float* gy = S->y + t.bead0;
        float* gz = S->z + t.bead0;
        const bool vec = ((t.bead0 & 3) == 0) && ((nb & 3) == 0);
        if (vec) {
            const float4* vx = reinterpret_cast<const float4*>(gx);
            const float4* vy = reinterpret_cast<const float4*>(gy);
            const float4* vz = reinterpret_cast<const float4*>(gz);
            for (int i = tid; i < (nb >> 2); i += T) {
                const float4 a = __ldcs(vx + i), b = __ldcs(vy + i), d = __ldcs(vz + i);
                reinterpret_cast<float4*>(sx)[i] = a;
                reinterpret_cast<float4*>(sy)[i] = b;
                reinterpret_cast<float4*>(sz)[i] = d;
            }
        } else {
            for (int i = tid; i < nb; i += T) {
                sx[i] = gx[i];
                sy[i] = gy[i];
                sz[i] = gz[i];
            }
        }
        __syncthreads();

        if (MODE != kGridOnly) {
            const uint32_t step = S->step + 1u;
            const uint32_t k0 = S->seed_lo, k1 = S->seed_hi;
            const uint32_t* __restrict__ cid = S->chain_id + t.chain0;
            const float* __restrict__ omega = S->omega;
            const int64_t NC = S->n_cells;
            const float cc2 = S->cdeg[2], ac42 = S->ac4deg[2];
            uint32_t* cnt = S->counts[S->cur];
            const bool c16 = S->count16 != 0;
            unsigned nacc = 0;
            for (int col = 0; col < Ap->n_colors; ++col) {
                const int ncol = Ap->color_off[col + 1] - Ap->color_off[col];
                const uint32_t mg = Ap->color_magic[col];
                const int items = t.n_chains * ncol;
                for (int j = tid; j < items; j += T) {
                    const int cl = (int)div_magic((uint32_t)j, mg, ncol);
                    const int base = cl * L;
                    float qx[LINEAR ? 2 : kMaxDeg], qy[LINEAR ? 2 : kMaxDeg], qz[LINEAR ? 2 : kMaxDeg];
                    int b, deg, type;
                    if (LINEAR) {
                        b = 2 * (j - cl * ncol) + col;
                        type = stype[b];
                        deg = 0;
                        if (b > 0) {
                            qx[0] = sx[base + b - 1];
                            qy[0] = sy[base + b - 1];
                            qz[0] = sz[base + b - 1];
                            deg = 1;
                        }
                        if (b + 1 < L) {
                            qx[deg] = sx[base + b + 1];
                            qy[deg] = sy[base + b + 1];
                            qz[deg] = sz[base + b + 1];
                            ++deg;
                        }
                    } else {
                        b = scol[Ap->color_off[col] + (j - cl * ncol)];
                        const BeadInfo bi = sinfo[b];
                        type = bi.type;
                        deg = bi.deg;
#pragma unroll
                        for (int d = 0; d < kMaxDeg; ++d) {
                            if (d < deg) {
                                const int q = base + bi.nbr[d];
                                qx[d] = sx[q];
                                qy[d] = sy[q];
                                qz[d] = sz[q];
                            }
                        }
                    }
                    float n0, n1, n2;
                    const uint32_t aw = bead_normals<KEYS>(__ldg(cid + cl), b, step, k0, k1, keys, n0, n1, n2);
                    float px, py, pz;
                    int c_old, c_new;
                    const bool acc = trial<LINEAR ? 2 : kMaxDeg>(c, sx[base + b], sy[base + b], sz[base + b], qx, qy,
                                                                 qz, deg, deg == 2 ? cc2 : S->cdeg[deg],
                                                                 deg == 2 ? ac42 : S->ac4deg[deg], n0, n1, n2, aw,
                                                                 omega + (int64_t)type * NC, px, py, pz, c_old, c_new);
                    if (acc) {
                        sx[base + b] = px;
                        sy[base + b] = py;
                        sz[base + b] = pz;
                    }
                    nacc += acc ? 1u : 0u;
                    if (MODE == kMoveGrid && acc && c_new != c_old) count_move(cnt, c16, (int64_t)type * NC, c_old, c_new);
                }
                __syncthreads();
            }
            nacc = warp_sum(nacc);
            if (lane == 0 && nacc) atomicAdd(&S->slot_acc[(ti * kMaxWarps + warp) % kSlots], (unsigned long long)nacc);
        }

        if (MODE == kGridOnly) {
            uint32_t* cnt = S->counts[S->cur];
            const int64_t NC = S->n_cells;
            const bool c16 = S->count16 != 0;
            for (int i = tid; i < nb; i += T) {
                const int cl = (int)div_magic((uint32_t)i, len_magic, L);
                const int b = i - cl * L;
                const int type = LINEAR ? stype[b] : sinfo[b].type;
                const int64_t idx = (int64_t)type * NC + cell_of(c, sx[i], sy[i], sz[i]);
                if (c16)
                    atomicAdd(cnt + (idx >> 1), 1u << ((idx & 1) * 16));
                else
                    atomicAdd(cnt + idx, 1u);
            }
        }

        if (MODE != kGridOnly) {
            if (vec) {
                float4* vx = reinterpret_cast<float4*>(gx);
                float4* vy = reinterpret_cast<float4*>(gy);
                float4* vz = reinterpret_cast<float4*>(gz);
                for (int i = tid; i < (nb >> 2); i += T) {
                    __stcs(vx + i, reinterpret_cast<const float4*>(sx)[i]);
                    __stcs(vy + i, reinterpret_cast<const float4*>(sy)[i]);
                    __stcs(vz + i, reinterpret_cast<const float4*>(sz)[i]);
                }
            } else {
                for (int i = tid; i < nb; i += T) {
                    gx[i] = sx[i];
                    gy[i] = sy[i];
                    gz[i] = sz[i];
                }
            }
        }
        __syncthreads();
    }
}

// Linear chains, one warp per run of whole chains.  Each warp stages its
// chains in its own slice of shared memory in a parity-split layout (for chain
// cl: even beads at cl*L + b/2, odd beads at cl*L + h0 + b/2, h0 = ceil(L/2)),
// so the lanes of a half-sweep read consecutive words, and the warp needs no
// block barrier: load, even half-sweep, odd half-sweep, store, separated by
// __syncwarp.  Results are identical to k_sweep (same trial, same keys).
// Three 256-thread CTAs per SM leave it 80 registers and no spill (at 64 it
// spilled ~100 B per thread and moved chains of 128 beads 12 % slower).
template <int MODE, int KEYS>
__global__ void __launch_bounds__(256, 3) k_sweep_linear(const MoveTile* __restrict__ tiles,
                                                          const int32_t* __restrict__ list, int n_list,
                                                          int warp_beads, unsigned* __restrict__ acc_part,
                                                          const PhiloxKeys keys) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    // per warp: x, y, z of its chains (parity-split)
    float* sx = reinterpret_cast<float*>(smem_raw) + (size_t)warp * 3 * warp_beads;
    float* sy = sx + warp_beads;
    float* sz = sy + warp_beads;
    for (int li = blockIdx.x; li < n_list; li += gridDim.x) {
        const int ti = list ? __ldg(list + li) : li;
        const MoveTile t = tiles[ti];
        SysDev* S = t.sys;
        if (MODE != kGridOnly && S->step >= S->stop_step) continue;
        const ArchDev* Ap = t.arch;
        const int L = Ap->length;
        const int h0 = (L + 1) >> 1;
        const int cpw = (t.n_chains + nwarps - 1) / nwarps;
        const int c_begin = warp * cpw;
        const int nch = min(cpw, t.n_chains - c_begin);
        if (nch <= 0) {
            continue;
        }
        const int nb = nch * L;
        if (nb > warp_beads) {
            if (lane == 0) atomicOr(&S->error_word, 2u);
            continue;
        }
        MoveConsts c;
        c.k = S->k; c.k2 = S->k2; c.A = S->A; c.R = S->R;
        c.inv_dx = S->inv_dx; c.inv_dy = S->inv_dy; c.inv_dz = S->inv_dz;
        load_fold(c, S);
        const uint32_t len_magic = Ap->len_magic;
        const int64_t g0 = t.bead0 + (int64_t)c_begin * L;
        float* gx = S->x + g0;
        float* gy = S->y + g0;
        float* gz = S->z + g0;
        for (int i = lane; i < nb; i += 32) {
            const int cl = (int)div_magic((uint32_t)i, len_magic, L);
            const int b = i - cl * L;
            const int slot = cl * L + (b & 1) * h0 + (b >> 1);
            sx[slot] = __ldcs(gx + i);
            sy[slot] = __ldcs(gy + i);
            sz[slot] = __ldcs(gz + i);
        }
        const uint8_t* __restrict__ types = Ap->types;
        const int64_t NC = S->n_cells;
        uint32_t* cnt = S->counts[S->cur];
        const bool c16 = S->count16 != 0;
        __syncwarp();
        if (MODE != kGridOnly) {
            const uint32_t step = S->step + 1u;
            const uint32_t k0 = S->seed_lo, k1 = S->seed_hi;
            const uint32_t my_cid = lane < nch ? __ldg(S->chain_id + t.chain0 + c_begin + lane) : 0u;
            const float* __restrict__ omega = S->omega;
            const float cc1 = S->cdeg[1], ac41 = S->ac4deg[1], cc2 = S->cdeg[2], ac42 = S->ac4deg[2];
            unsigned nacc = 0;
#pragma unroll 1
            for (int col = 0; col < 2; ++col) {
                const int half = col == 0 ? h0 : (L >> 1);
                const uint32_t mg = Ap->color_magic[col];
                const int items = nch * half;
                const int own = col * h0, other = (1 - col) * h0;
                // lanes of one iteration share the loop bound: every lane runs the
                // shuffle below, inactive ones on a dummy item
                for (int j0 = 0; j0 < items; j0 += 32) {
                    const int j = j0 + lane;
                    const bool act = j < items;
                    const int jj = act ? j : 0;
                    const int cl = (int)div_magic((uint32_t)jj, mg, half);
                    const uint32_t gc = __shfl_sync(0xffffffffu, my_cid, cl & 31);
                    if (!act) continue;
                    const int k = jj - cl * half;
                    const int b = 2 * k + col;
                    const int base = cl * L;
                    const int me = base + own + k;
                    float qx[2], qy[2], qz[2];
                    int deg = 0;
                    if (b > 0) {
                        const int q = base + other + k - 1 + col;
                        qx[0] = sx[q];
                        qy[0] = sy[q];
                        qz[0] = sz[q];
                        deg = 1;
                    }
                    if (b + 1 < L) {
                        const int q = base + other + k + col;
                        qx[deg] = sx[q];
                        qy[deg] = sy[q];
                        qz[deg] = sz[q];
                        ++deg;
                    }
                    const int type = __ldg(types + b);
                    float n0, n1, n2;
                    const uint32_t aw = bead_normals<KEYS>(gc, b, step, k0, k1, keys, n0, n1, n2);
                    float px, py, pz;
                    int c_old, c_new;
                    const bool acc = trial<2>(c, sx[me], sy[me], sz[me], qx, qy, qz, deg, deg == 2 ? cc2 : cc1,
                                              deg == 2 ? ac42 : ac41, n0, n1, n2, aw, omega + (int64_t)type * NC, px,
                                              py, pz, c_old, c_new);
                    if (acc) {
                        sx[me] = px;
                        sy[me] = py;
                        sz[me] = pz;
                    }
                    nacc += acc ? 1u : 0u;
                    if (MODE == kMoveGrid && acc && c_new != c_old) count_move(cnt, c16, (int64_t)type * NC, c_old, c_new);
                }
                __syncwarp();
            }
            nacc = warp_sum(nacc);
            if (lane == 0 && nacc) atomicAdd(&S->slot_acc[(ti * kMaxWarps + warp) % kSlots], (unsigned long long)nacc);
        }
        if (MODE == kGridOnly) {
            for (int i = lane; i < nb; i += 32) {
                const int cl = (int)div_magic((uint32_t)i, len_magic, L);
                const int b = i - cl * L;
                const int slot = cl * L + (b & 1) * h0 + (b >> 1);
                const int64_t idx = (int64_t)__ldg(types + b) * NC + cell_of(c, sx[slot], sy[slot], sz[slot]);
                if (c16)
                    atomicAdd(cnt + (idx >> 1), 1u << ((idx & 1) * 16));
                else
                    atomicAdd(cnt + idx, 1u);
            }
        } else {
            for (int i = lane; i < nb; i += 32) {
                const int cl = (int)div_magic((uint32_t)i, len_magic, L);
                const int b = i - cl * L;
                const int slot = cl * L + (b & 1) * h0 + (b >> 1);
                __stcs(gx + i, sx[slot]);
                __stcs(gy + i, sy[slot]);
                __stcs(gz + i, sz[slot]);
            }
        }
        __syncwarp();
    }
}

// Linear chains of at most 64 beads, positions in registers.  Each thread owns
// the bead pair (2t, 2t+1) of one chain (ceil(L/2) threads per chain).  Even
// half-sweep: bead 2t moves against 2t-1 (the odd bead of lane-1, by shuffle)
// and 2t+1 (its own); odd half-sweep: bead 2t+1 moves against 2t (its own,
// already moved) and 2t+2 (the even bead of lane+1).  When ceil(L/2) divides
// 32, each warp holds whole chains: no shared memory, no block barrier.
// Otherwise (L = 48: 24 threads per chain would idle a quarter of every warp)
// the block holds as many whole chains as fit in all its threads, chains run
// across warp boundaries: a warp's first even bead reads its left neighbour
// from global memory (not yet moved, not yet stored), its last odd bead gets
// the moved right neighbour through shared memory after one block barrier per
// iteration; every chain still moves all its even beads before any odd bead.  Tiles are read and written with
// coalesced float2 accesses.  Same trial and keys as k_sweep.
// Register cap per instance.  80 (six 128-thread CTAs, 24 warps per SM) is
// what the general instances need without spilling; the instances that read
// their Philox round keys from the parameter bank fit in 72 without spilling,
// which gives seven CTAs (28 warps) per SM (large system 0.661 -> 0.621 ms,
// batched mix +4.4 %).  At 64 (32 warps) they spill 20-36 B.
constexpr int reg_cap(bool flat, int fold, int keys) {
    return (keys == kKeysBoth || (keys == kKeysHigh && fold != 0 && !flat)) ? 72 : 80;
}

template <int MODE, bool ANY_FLAT, int FOLD, int KEYS>
__global__ void __maxnreg__(reg_cap(ANY_FLAT, FOLD, KEYS)) k_sweep_reg(const MoveTile* __restrict__ tiles,
                                                                        const int32_t* __restrict__ list, int n_list,
                                                                        unsigned* __restrict__ acc_part,
                                                                        const PhiloxKeys keys) {
    // even bead of each warp's lane 0 after its move, double-buffered by
    // iteration parity: with one barrier per iteration a warp may write the
    // next iteration's slot while its left neighbour still reads this one
    __shared__ float s_first_even[2][kMaxWarps][3];
    __shared__ float4 s_ntab[SCMF_NORMAL_SEGS];
    if (MODE != kGridOnly) load_normal_table(s_ntab);
    // Every instance computes the odd bead's Philox block together with the
    // even bead's (two independent chains of rounds to interleave).  The keyed
    // instances, whose Philox key lives (at least half) in the parameter bank,
    // also add the even bead's bond forces one at a time (no local array); the
    // others spill that way and keep the two-entry array.  All give the same bits.
    constexpr bool kLean = KEYS != kKeysNone;
    int parity = 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int li = blockIdx.x; li < n_list; li += gridDim.x) {
        const int ti = list ? __ldg(list + li) : li;  // tile index in the plan
        const MoveTile t = tiles[ti];
        SysDev* S = t.sys;
        if (MODE != kGridOnly && S->step >= S->stop_step) continue;  // block-uniform
        const ArchDev* Ap = t.arch;
        const int L = Ap->length;
        const int tpc = (L + 1) >> 1;                        // threads per chain
        const bool flat = ANY_FLAT && (32 % tpc) != 0;       // chains run across warps (block-uniform)
        const int slot = flat ? (int)threadIdx.x : lane;     // pair slot in the block / in the warp
        const int cpw = flat ? (int)blockDim.x / tpc : 32 / tpc;  // chains per block / per warp iteration
        const int cs = (int)div_magic((uint32_t)slot, Ap->tpc_magic, tpc);
        const int tt = slot - cs * tpc;                      // pair index in the chain
        const int be = 2 * tt, bo = 2 * tt + 1;
        MoveConsts c;
        c.k = S->k; c.k2 = S->k2; c.A = S->A; c.R = S->R;
        c.inv_dx = S->inv_dx; c.inv_dy = S->inv_dy; c.inv_dz = S->inv_dz;
        load_fold(c, S);
        const int64_t NC = S->n_cells;
        // counts pointer and width: read here for gridding, and again at each (rare)
        // count move of the move modes, so that no register holds them across a sweep
        uint32_t* cnt = S->counts[S->cur];
        const bool c16 = S->count16 != 0;
        const float* __restrict__ omega = S->omega;
        const uint32_t step = S->step + 1u;
        const uint32_t k0 = S->seed_lo, k1 = S->seed_hi;
        const float cc1 = S->cdeg[1], ac41 = S->ac4deg[1], cc2 = S->cdeg[2], ac42 = S->ac4deg[2];
        const int type_e = cs < cpw ? __ldg(Ap->types + min(be, L - 1)) : 0;
        const int type_o = cs < cpw && bo < L ? __ldg(Ap->types + bo) : 0;
        const bool pair_aligned = ((t.bead0 & 1) == 0) && ((L & 1) == 0);
        unsigned nacc = 0;
        for (int cbase = flat ? 0 : warp * cpw; cbase < t.n_chains; cbase += flat ? cpw : nwarps * cpw) {
            const int chain = cbase + cs;
            const bool live = cs < cpw && chain < t.n_chains;
            const bool has_o = live && bo < L;
            const int64_t g = t.bead0 + (int64_t)chain * L + be;
            float xe = 0.0f, ye = 0.0f, ze = 0.0f, xo = 0.0f, yo = 0.0f, zo = 0.0f;
            uint32_t gc = 0u;
            if (live) {
                if (pair_aligned) {
                    const float2 vx = __ldcs(reinterpret_cast<const float2*>(S->x + g));
                    const float2 vy = __ldcs(reinterpret_cast<const float2*>(S->y + g));
                    const float2 vz = __ldcs(reinterpret_cast<const float2*>(S->z + g));
                    xe = vx.x; xo = vx.y;
                    ye = vy.x; yo = vy.y;
                    ze = vz.x; zo = vz.y;
                } else {
                    xe = __ldcs(S->x + g);
                    ye = __ldcs(S->y + g);
                    ze = __ldcs(S->z + g);
                    if (has_o) {
                        xo = __ldcs(S->x + g + 1);
                        yo = __ldcs(S->y + g + 1);
                        zo = __ldcs(S->z + g + 1);
                    }
                }
                gc = __ldg(S->chain_id + t.chain0 + chain);
            }
            if (MODE == kGridOnly) {
                if (live) {
                    const int64_t ie = (int64_t)type_e * NC + cell_of<FOLD>(c, xe, ye, ze);
                    if (c16) atomicAdd(cnt + (ie >> 1), 1u << ((ie & 1) * 16)); else atomicAdd(cnt + ie, 1u);
                }
                if (has_o) {
                    const int64_t io = (int64_t)type_o * NC + cell_of<FOLD>(c, xo, yo, zo);
                    if (c16) atomicAdd(cnt + (io >> 1), 1u << ((io & 1) * 16)); else atomicAdd(cnt + io, 1u);
                }
                continue;
            }
            uint4 wo = make_uint4(0u, 0u, 0u, 0u);  // the odd bead's Philox block
            // even half-sweep
            {
                float lx = __shfl_up_sync(0xffffffffu, xo, 1);
                float ly = __shfl_up_sync(0xffffffffu, yo, 1);
                float lz = __shfl_up_sync(0xffffffffu, zo, 1);
                if (flat && lane == 0 && warp > 0 && live && tt > 0) {
                    // the previous warp's last odd bead, not yet moved: positions of this
                    // iteration are stored only after the barrier below, so global memory
                    // still holds its start-of-sweep value (read through L2)
                    lx = __ldcg(S->x + g - 1);
                    ly = __ldcg(S->y + g - 1);
                    lz = __ldcg(S->z + g - 1);
                }
                if (live) {
                    // neighbours in ascending bead order: 2t-1 (if any), then 2t+1 (if any),
                    // one at a time (kLean) or through a two-entry array (in a 24 B stack
                    // frame; the other instances spill 16-32 B without it).  Same fma sequence.
                    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
                    float qx[2], qy[2], qz[2];
                    int deg = 0;
                    if (kLean) {
                        if (tt > 0) add_bond(c.k2, xe, ye, ze, lx, ly, lz, fx, fy, fz);
                        if (has_o) add_bond(c.k2, xe, ye, ze, xo, yo, zo, fx, fy, fz);
                        deg = (tt > 0 ? 1 : 0) + (has_o ? 1 : 0);
                    } else {
                        if (tt > 0) { qx[0] = lx; qy[0] = ly; qz[0] = lz; deg = 1; }
                        if (has_o) { qx[deg] = xo; qy[deg] = yo; qz[deg] = zo; ++deg; }
                    }
                    const uint4 w = philox_block<KEYS>(make_uint4(gc, (uint32_t)be, step, 0u), k0, k1, keys);
                    wo = philox_block<KEYS>(make_uint4(gc, (uint32_t)bo, step, 0u), k0, k1, keys);
                    float n0, n1, n2;
                    normals3(w, s_ntab, n0, n1, n2);
                    float px, py, pz;
                    int c_old, c_new;
                    const float cc = deg == 2 ? cc2 : (deg == 1 ? cc1 : 0.0f);
                    const float ac4 = deg == 2 ? ac42 : (deg == 1 ? ac41 : 0.0f);
                    const float* w_e = omega + (int64_t)type_e * NC;
                    const bool acc = kLean ? trial_f<FOLD>(c, xe, ye, ze, fx, fy, fz, cc, ac4, n0, n1, n2,
                                                           accept_word(w), w_e, px, py, pz, c_old, c_new)
                                           : trial<2, FOLD>(c, xe, ye, ze, qx, qy, qz, deg, cc, ac4, n0, n1, n2,
                                                            accept_word(w), w_e, px, py, pz, c_old, c_new);
                    if (acc) { xe = px; ye = py; ze = pz; }
                    nacc += acc ? 1u : 0u;
                    if (MODE == kMoveGrid && acc && c_new != c_old)
                        count_move(S->counts[S->cur], S->count16 != 0, (int64_t)type_e * NC, c_old, c_new);
                }
            }
            // odd half-sweep
            {
                float rx = __shfl_down_sync(0xffffffffu, xe, 1);
                float ry = __shfl_down_sync(0xffffffffu, ye, 1);
                float rz = __shfl_down_sync(0xffffffffu, ze, 1);
                if (flat) {
                    if (lane == 0) {
                        s_first_even[parity][warp][0] = xe;
                        s_first_even[parity][warp][1] = ye;
                        s_first_even[parity][warp][2] = ze;
                    }
                    __syncthreads();
                    if (lane == 31 && warp + 1 < nwarps) {
                        rx = s_first_even[parity][warp + 1][0];
                        ry = s_first_even[parity][warp + 1][1];
                        rz = s_first_even[parity][warp + 1][2];
                    }
                    parity ^= 1;
                }
                if (has_o) {
                    float qx[2], qy[2], qz[2];
                    qx[0] = xe; qy[0] = ye; qz[0] = ze;
                    int deg = 1;
                    if (bo + 1 < L) { qx[1] = rx; qy[1] = ry; qz[1] = rz; deg = 2; }
                    float n0, n1, n2;
                    normals3(wo, s_ntab, n0, n1, n2);
                    float px, py, pz;
                    int c_old, c_new;
                    const bool acc = trial<2, FOLD>(c, xo, yo, zo, qx, qy, qz, deg, deg == 2 ? cc2 : cc1,
                                              deg == 2 ? ac42 : ac41, n0, n1, n2, accept_word(wo),
                                              omega + (int64_t)type_o * NC, px, py, pz, c_old, c_new);
                    if (acc) { xo = px; yo = py; zo = pz; }
                    nacc += acc ? 1u : 0u;
                    if (MODE == kMoveGrid && acc && c_new != c_old)
                        count_move(S->counts[S->cur], S->count16 != 0, (int64_t)type_o * NC, c_old, c_new);
                }
            }
            if (live) {
                if (pair_aligned) {
                    __stcs(reinterpret_cast<float2*>(S->x + g), make_float2(xe, xo));
                    __stcs(reinterpret_cast<float2*>(S->y + g), make_float2(ye, yo));
                    __stcs(reinterpret_cast<float2*>(S->z + g), make_float2(ze, zo));
                } else {
                    __stcs(S->x + g, xe);
                    __stcs(S->y + g, ye);
                    __stcs(S->z + g, ze);
                    if (has_o) {
                        __stcs(S->x + g + 1, xo);
                        __stcs(S->y + g + 1, yo);
                        __stcs(S->z + g + 1, zo);
                    }
                }
            }
        }
        if (MODE != kGridOnly) {
            nacc = warp_sum(nacc);
            if (lane == 0 && nacc) atomicAdd(&S->slot_acc[(ti * kMaxWarps + warp) % kSlots], (unsigned long long)nacc);
        }
    }
}

// Lean move kernel for launches of one system whose architectures are linear
// chains of an even length L <= 64 with L/2 dividing 32, on a grid of
// power-of-two axes (LaunchShape::lean; the large system and the blend are
// such launches).  Same sweep, trials and random numbers as k_sweep_reg, with
// less work per trial:
//  * the system's constants (positions, omega, chain ids, k, A, R, cell
//    inverses, grid, per-degree c and A c / 4, the architectures' chain and
//    bead ranges) come from the parameter bank (SysConsts), the Philox round
//    keys too;
//  * every pair has an odd bead, so the even/odd branches go away; a missing
//    bond neighbour at a chain end is replaced by the bead itself, whose term
//    fma(+0, 2k, f) leaves the force bit for bit as if it were skipped (the
//    force starts at +0 and can only be -0 from a -0 sum, which RN never
//    gives here);
//  * lanes beyond an architecture's last chain (a partial last group) repeat
//    that chain and store nothing, so every lane runs the same code;
//  * the Metropolis logarithm and the count moves sit under warp-uniform
//    branches (__any_sync); the outcome of every trial is unchanged;
//  * a trial whose bonded energy change alone exceeds what the omega span
//    and its uniform allow is rejected before the cell folds and the omega
//    gathers (maybe_accepted), which about half of the warps then skip.
// Persistent: one CTA of kLeanThreads (28 warps, 72 registers each: the SM's
// whole register file) per SM.  Each warp strides over the groups of 32/(L/2)
// chains of every architecture, so no tile tail is left, and loads the next
// group's pairs while it moves the current one.  The CTA keeps kLeanCopies
// copies of the normal table in shared memory, entry-interleaved, and lane l
// reads copy l % 8: the eight lanes of one 16-byte shared-memory phase then
// always read eight different bank groups (with one copy, random segments made
// 2.3 wavefronts of every phase).  Bead and cell indices are 32-bit (the plan
// checks the sizes).
constexpr int kLeanThreads = 896;
constexpr int kLeanCopies = 8;
constexpr size_t kLeanSmem = (size_t)SCMF_NORMAL_SEGS * kLeanCopies * sizeof(float4);


// One trial of the bead at (x, y, z) with bond force f, updated in place when
// accepted (lanes with live false never move): the proposal, its cells and
// the omega reads are formed only in warps where some lane passes the span
// bound.  Returns whether the move was accepted.
__device__ __forceinline__ bool trial_lean(const MoveConsts& c, float& x, float& y, float& z, float fx, float fy,
                                           float fz, float cc, float ac4, float n0, float n1, float n2, uint32_t aw,
                                           float span, bool live, const float* __restrict__ w_t, int& cell_old,
                                           int& cell_new) {
    const float A = c.A, R = c.R;
    const float dx = __fmaf_rn(A, fx, __fmul_rn(R, n0));
    const float dy = __fmaf_rn(A, fy, __fmul_rn(R, n1));
    const float dz = __fmaf_rn(A, fz, __fmul_rn(R, n2));
    const float d2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
    const float fd = __fmaf_rn(fx, dx, __fmaf_rn(fy, dy, __fmul_rn(fz, dz)));
    const float deb = __fmul_rn(ac4, __fmaf_rn(cc, d2, __fmul_rn(-2.0f, fd)));
    const float u = u01(aw);
    bool acc = false;
    cell_old = cell_new = 0;
    if (__any_sync(0xffffffffu, maybe_accepted(deb, span, log_lower(u)))) {
        const float px = __fadd_rn(x, dx), py = __fadd_rn(y, dy), pz = __fadd_rn(z, dz);
        cell_old = cell_of<0>(c, x, y, z);
        cell_new = cell_of<0>(c, px, py, pz);
        const float dE = __fadd_rn(__fsub_rn(__ldg(w_t + cell_new), __ldg(w_t + cell_old)), deb);
        // accept if dE < 0; else if log(u) < -dE (log_lower decides without the
        // logarithm for all but a few trials in a thousand; dE >= 17 fails
        // -dE > log_lower(u) >= -16, so no separate bound is needed)
        acc = dE < 0.0f;
        const bool near = !acc && -dE > log_lower(u);
        if (__any_sync(0xffffffffu, near)) acc = acc || (near && log_f(u) < -dE);
        acc = acc && live;
        if (acc) {
            x = px;
            y = py;
            z = pz;
        }
    }
    return acc;
}

template <int MODE>
__global__ void __maxnreg__(72) k_sweep_lean(const PhiloxKeys keys, const SysConsts sc) {
    extern __shared__ float4 s_ntab_lean[];  // [SCMF_NORMAL_SEGS][kLeanCopies]
    for (int i = threadIdx.x; i < SCMF_NORMAL_SEGS * kLeanCopies; i += blockDim.x)
        s_ntab_lean[i] = __ldg(normal_table() + i / kLeanCopies);
    __syncthreads();
    SysDev* S = sc.sys;
    if (S->step >= S->stop_step) return;  // grid-uniform
    const uint32_t step = S->step + 1u;
    const float span = S->omega_span;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gw = blockIdx.x * (blockDim.x >> 5) + warp;  // this warp among all
    const int nw = gridDim.x * (blockDim.x >> 5);
    const float4* tab = s_ntab_lean + (lane & (kLeanCopies - 1));
    MoveConsts c;
    c.k = 0.0f;
    c.k2 = sc.k2;
    c.A = sc.A;
    c.R = sc.R;
    c.inv_dx = sc.inv_dx;
    c.inv_dy = sc.inv_dy;
    c.inv_dz = sc.inv_dz;
    c.nx = sc.nx;
    c.ny = sc.ny;
    c.nz = sc.nz;
    c.pow2 = true;
    c.small = false;
    unsigned nacc = 0;
    for (int a = 0; a < sc.n_arch; ++a) {
        const int L = sc.arch[a].length;
        const int lg = __ffs(L >> 1) - 1;                         // log2(L/2): L/2 divides 32
        const int tpc = 1 << lg;                                  // threads per chain
        const int cs = lane >> lg;                                // chain slot in the warp
        const int tt = lane & (tpc - 1);                          // pair index in the chain
        const int cpw = 32 >> lg;                                 // chains per group
        const int be = 2 * tt, bo = be + 1;
        const bool first = tt == 0, last = tt == tpc - 1;         // chain ends: one bond
        const float cc_e = first ? sc.cdeg[1] : sc.cdeg[2], ac4_e = first ? sc.ac4deg[1] : sc.ac4deg[2];
        const float cc_o = last ? sc.cdeg[1] : sc.cdeg[2], ac4_o = last ? sc.ac4deg[1] : sc.ac4deg[2];
        const int toff_e = (int)__ldg(sc.arch[a].types + be) * (int)sc.n_cells;
        const int toff_o = (int)__ldg(sc.arch[a].types + bo) * (int)sc.n_cells;
        // a chain end's missing bond: the shuffles below return the lane's own
        // bead there, and these zero spring constants make its term +-0
        const float k2_l = first ? 0.0f : sc.k2, k2_r = last ? 0.0f : sc.k2;
        const int nch = sc.arch[a].n_chains;
        const int bead0 = sc.arch[a].bead0;
        const uint32_t rng0 = (uint32_t)sc.arch[a].rng0;
        const int groups = (nch + cpw - 1) >> (5 - lg);
        // the pairs and chain id of the warp's next group are loaded one group
        // ahead, so the DRAM latency overlaps this group's trials
        float2 nvx = make_float2(0.0f, 0.0f), nvy = nvx, nvz = nvx;
        auto fetch = [&](int grp) {
            const int ch = min(grp * cpw + cs, nch - 1);
            const int gn = bead0 + ch * L + be;
            nvx = __ldcs(reinterpret_cast<const float2*>(sc.x + gn));
            nvy = __ldcs(reinterpret_cast<const float2*>(sc.y + gn));
            nvz = __ldcs(reinterpret_cast<const float2*>(sc.z + gn));
        };
        if (gw < groups) fetch(gw);
        for (int grp = gw; grp < groups; grp += nw) {  // warp-uniform bounds
            const int chain = grp * cpw + cs;
            const bool live = chain < nch;
            const int chc = live ? chain : nch - 1;
            const int g = bead0 + chc * L + be;
            const float2 vx = nvx, vy = nvy, vz = nvz;
            const uint32_t gc = rng0 + (uint32_t)chc;  // storage order is the stream order
            if (grp + nw < groups) fetch(grp + nw);
            float xe = vx.x, xo = vx.y, ye = vy.x, yo = vy.y, ze = vz.x, zo = vz.y;
            // even bead 2t: bonds to 2t-1 (lane - 1's odd bead; the bead itself at the chain start) and 2t+1
            const float lx = __shfl_up_sync(0xffffffffu, xo, 1, tpc);
            const float ly = __shfl_up_sync(0xffffffffu, yo, 1, tpc);
            const float lz = __shfl_up_sync(0xffffffffu, zo, 1, tpc);
            const uint4 w = philox4x32_10(make_uint4(gc, (uint32_t)be, step, 0u), keys);
            const uint4 wo = philox4x32_10(make_uint4(gc, (uint32_t)bo, step, 0u), keys);
            float n0, n1, n2;
            normals3<kLeanCopies>(w, tab, n0, n1, n2);
            bool acc_e, mv_e;
            int ce_old, ce_new;
            {
                float fx = __fmaf_rn(__fsub_rn(lx, xe), k2_l, 0.0f);
                float fy = __fmaf_rn(__fsub_rn(ly, ye), k2_l, 0.0f);
                float fz = __fmaf_rn(__fsub_rn(lz, ze), k2_l, 0.0f);
                add_bond(c.k2, xe, ye, ze, xo, yo, zo, fx, fy, fz);
                acc_e = trial_lean(c, xe, ye, ze, fx, fy, fz, cc_e, ac4_e, n0, n1, n2, accept_word(w), span, live,
                                   sc.omega + toff_e, ce_old, ce_new);
                mv_e = acc_e && ce_new != ce_old;
            }
            // odd bead 2t+1: bonds to 2t (moved) and 2t+2 (lane + 1's moved even bead; the bead itself at the end)
            const float rx = __shfl_down_sync(0xffffffffu, xe, 1, tpc);
            const float ry = __shfl_down_sync(0xffffffffu, ye, 1, tpc);
            const float rz = __shfl_down_sync(0xffffffffu, ze, 1, tpc);
            normals3<kLeanCopies>(wo, tab, n0, n1, n2);
            bool acc_o, mv_o;
            int co_old, co_new;
            {
                float fx = __fmaf_rn(__fsub_rn(xe, xo), c.k2, 0.0f);
                float fy = __fmaf_rn(__fsub_rn(ye, yo), c.k2, 0.0f);
                float fz = __fmaf_rn(__fsub_rn(ze, zo), c.k2, 0.0f);
                add_bond(k2_r, xo, yo, zo, rx, ry, rz, fx, fy, fz);
                acc_o = trial_lean(c, xo, yo, zo, fx, fy, fz, cc_o, ac4_o, n0, n1, n2, accept_word(wo), span, live,
                                   sc.omega + toff_o, co_old, co_new);
                mv_o = acc_o && co_new != co_old;
            }
            nacc += (acc_e ? 1u : 0u) + (acc_o ? 1u : 0u);
            if (MODE == kMoveGrid && __any_sync(0xffffffffu, mv_e || mv_o)) {
                uint32_t* cnt = S->counts[S->cur];
                const bool c16 = S->count16 != 0;
                if (mv_e) count_move(cnt, c16, toff_e, ce_old, ce_new);
                if (mv_o) count_move(cnt, c16, toff_o, co_old, co_new);
            }
            if (live) {
                __stcs(reinterpret_cast<float2*>(sc.x + g), make_float2(xe, xo));
                __stcs(reinterpret_cast<float2*>(sc.y + g), make_float2(ye, yo));
                __stcs(reinterpret_cast<float2*>(sc.z + g), make_float2(ze, zo));
            }
        }
    }
    nacc = warp_sum(nacc);
    if (lane == 0 && nacc) atomicAdd(&S->slot_acc[gw % kSlots], (unsigned long long)nacc);
}

// The lean kernel's structure for launches of many systems (batches, served
// rounds) and for single systems that k_sweep_lean does not take: linear chains
// whose ceil(L/2) divides 32 with L even (LaunchShape::warp_even), any grid (FOLD
// 0: every axis a power of two; -1: the fold is chosen per system) and any key
// mode.  Each tile's system constants come from its SysDev into registers; at
// 96 registers (no spill) the 256-system mix ran 7.39e10 bead-moves/s against
// 7.00e10 with k_sweep_reg (80-88 registers spilled and lost).
template <int FOLD>
__device__ __forceinline__ bool trial_leanm(const MoveConsts& c, float& x, float& y, float& z, float fx, float fy,
                                           float fz, float cc, float ac4, float n0, float n1, float n2, uint32_t aw,
                                           float span, bool live, const float* __restrict__ w_t, int& cell_old,
                                           int& cell_new) {
    const float A = c.A, R = c.R;
    const float dx = __fmaf_rn(A, fx, __fmul_rn(R, n0));
    const float dy = __fmaf_rn(A, fy, __fmul_rn(R, n1));
    const float dz = __fmaf_rn(A, fz, __fmul_rn(R, n2));
    const float d2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
    const float fd = __fmaf_rn(fx, dx, __fmaf_rn(fy, dy, __fmul_rn(fz, dz)));
    const float deb = __fmul_rn(ac4, __fmaf_rn(cc, d2, __fmul_rn(-2.0f, fd)));
    const float u = u01(aw);
    bool acc = false;
    cell_old = cell_new = 0;
    // the omega span rejects most trials before the folds and gathers (see trial_lean)
    if (__any_sync(0xffffffffu, maybe_accepted(deb, span, log_lower(u)))) {
        const float px = __fadd_rn(x, dx), py = __fadd_rn(y, dy), pz = __fadd_rn(z, dz);
        cell_old = cell_of<FOLD>(c, x, y, z);
        cell_new = cell_of<FOLD>(c, px, py, pz);
        const float dE = __fadd_rn(__fsub_rn(__ldg(w_t + cell_new), __ldg(w_t + cell_old)), deb);
        acc = dE < 0.0f;
        const bool near = !acc && -dE > log_lower(u);
        if (__any_sync(0xffffffffu, near)) acc = acc || (near && log_f(u) < -dE);
        acc = acc && live;
        if (acc) {
            x = px;
            y = py;
            z = pz;
        }
    }
    return acc;
}

template <int MODE, int FOLD, int KEYS>
__global__ void __maxnreg__(96) k_sweep_leanm(const MoveTile* __restrict__ tiles, const int32_t* __restrict__ list, int n_list,
                                             const PhiloxKeys keys) {
    __shared__ float4 s_ntab[SCMF_NORMAL_SEGS];
    load_normal_table(s_ntab);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int li = blockIdx.x; li < n_list; li += gridDim.x) {
        const int ti = list ? __ldg(list + li) : li;
        const MoveTile t = tiles[ti];
        SysDev* S = t.sys;
        if (S->step >= S->stop_step) continue;  // block-uniform
        const uint32_t step = S->step + 1u;
        MoveConsts c;
        c.k = S->k; c.k2 = S->k2; c.A = S->A; c.R = S->R;
        c.inv_dx = S->inv_dx; c.inv_dy = S->inv_dy; c.inv_dz = S->inv_dz;
        load_fold(c, S);
        const uint32_t k0 = S->seed_lo, k1 = S->seed_hi;
        float* const PX = S->x;
        float* const PY = S->y;
        float* const PZ = S->z;
        const float* const OM = S->omega;
        const float span = S->omega_span;
        const int NCi = (int)S->n_cells;
        const ArchDev* Ap = t.arch;
        const int L = Ap->length;
        const int tpc = L >> 1;                                   // threads per chain, divides 32
        const int cs = (int)div_magic((uint32_t)lane, Ap->tpc_magic, tpc);
        const int tt = lane - cs * tpc;                           // pair index in the chain
        const int cpw = 32 / tpc;                                 // chains per warp iteration
        const int be = 2 * tt, bo = be + 1;
        const bool first = tt == 0, last = tt == tpc - 1;         // chain ends: one bond
        const float cc_e = first ? S->cdeg[1] : S->cdeg[2], ac4_e = first ? S->ac4deg[1] : S->ac4deg[2];
        const float cc_o = last ? S->cdeg[1] : S->cdeg[2], ac4_o = last ? S->ac4deg[1] : S->ac4deg[2];
        const int toff_e = (int)__ldg(Ap->types + be) * NCi;
        const int toff_o = (int)__ldg(Ap->types + bo) * NCi;
        // a chain end's missing bond: the shuffles below return the lane's own
        // bead there, and these zero spring constants make its term +-0
        const float k2_l = first ? 0.0f : c.k2, k2_r = last ? 0.0f : c.k2;
        // random-stream id of the tile's first chain (storage order is the stream order)
        const uint32_t rng0 = (uint32_t)(Ap->rng_base + (t.chain0 - Ap->chain_base));
        const int nch = t.n_chains;
        const int stride = nwarps * cpw;
        unsigned nacc = 0;
        // the pair and chain id of the next iteration are loaded one iteration
        // ahead, so the DRAM latency overlaps this iteration's trials
        float2 nvx = make_float2(0.0f, 0.0f), nvy = nvx, nvz = nvx;
        auto fetch = [&](int cb) {
            const int ch = min(cb + cs, nch - 1);
            const int gn = (int)t.bead0 + ch * L + be;
            nvx = __ldcs(reinterpret_cast<const float2*>(PX + gn));
            nvy = __ldcs(reinterpret_cast<const float2*>(PY + gn));
            nvz = __ldcs(reinterpret_cast<const float2*>(PZ + gn));
        };
        if (warp * cpw < nch) fetch(warp * cpw);
        for (int cbase = warp * cpw; cbase < nch; cbase += stride) {  // warp-uniform bounds
            const int chain = cbase + cs;
            const bool live = chain < nch;
            const int chc = live ? chain : nch - 1;
            const int g = (int)t.bead0 + chc * L + be;
            const float2 vx = nvx, vy = nvy, vz = nvz;
            const uint32_t gc = rng0 + (uint32_t)chc;
            if (cbase + stride < nch) fetch(cbase + stride);
            float xe = vx.x, xo = vx.y, ye = vy.x, yo = vy.y, ze = vz.x, zo = vz.y;
            // even bead 2t: bonds to 2t-1 (lane - 1's odd bead; the bead itself at the chain start) and 2t+1
            const float lx = __shfl_up_sync(0xffffffffu, xo, 1, tpc);
            const float ly = __shfl_up_sync(0xffffffffu, yo, 1, tpc);
            const float lz = __shfl_up_sync(0xffffffffu, zo, 1, tpc);
            const uint4 w = philox_block<KEYS>(make_uint4(gc, (uint32_t)be, step, 0u), k0, k1, keys);
            const uint4 wo = philox_block<KEYS>(make_uint4(gc, (uint32_t)bo, step, 0u), k0, k1, keys);
            float n0, n1, n2;
            normals3(w, s_ntab, n0, n1, n2);
            bool acc_e, mv_e;
            int ce_old, ce_new;
            {
                float fx = __fmaf_rn(__fsub_rn(lx, xe), k2_l, 0.0f);
                float fy = __fmaf_rn(__fsub_rn(ly, ye), k2_l, 0.0f);
                float fz = __fmaf_rn(__fsub_rn(lz, ze), k2_l, 0.0f);
                add_bond(c.k2, xe, ye, ze, xo, yo, zo, fx, fy, fz);
                acc_e = trial_leanm<FOLD>(c, xe, ye, ze, fx, fy, fz, cc_e, ac4_e, n0, n1, n2, accept_word(w), span,
                                          live, OM + toff_e, ce_old, ce_new);
                mv_e = acc_e && ce_new != ce_old;
            }
            // odd bead 2t+1: bonds to 2t (moved) and 2t+2 (lane + 1's moved even bead; the bead itself at the end)
            const float rx = __shfl_down_sync(0xffffffffu, xe, 1, tpc);
            const float ry = __shfl_down_sync(0xffffffffu, ye, 1, tpc);
            const float rz = __shfl_down_sync(0xffffffffu, ze, 1, tpc);
            normals3(wo, s_ntab, n0, n1, n2);
            bool acc_o, mv_o;
            int co_old, co_new;
            {
                float fx = __fmaf_rn(__fsub_rn(xe, xo), c.k2, 0.0f);
                float fy = __fmaf_rn(__fsub_rn(ye, yo), c.k2, 0.0f);
                float fz = __fmaf_rn(__fsub_rn(ze, zo), c.k2, 0.0f);
                add_bond(k2_r, xo, yo, zo, rx, ry, rz, fx, fy, fz);
                acc_o = trial_leanm<FOLD>(c, xo, yo, zo, fx, fy, fz, cc_o, ac4_o, n0, n1, n2, accept_word(wo), span,
                                          live, OM + toff_o, co_old, co_new);
                mv_o = acc_o && co_new != co_old;
            }
            nacc += (acc_e ? 1u : 0u) + (acc_o ? 1u : 0u);
            if (MODE == kMoveGrid && __any_sync(0xffffffffu, mv_e || mv_o)) {
                uint32_t* cnt = S->counts[S->cur];
                const bool c16 = S->count16 != 0;
                if (mv_e) count_move(cnt, c16, toff_e, ce_old, ce_new);
                if (mv_o) count_move(cnt, c16, toff_o, co_old, co_new);
            }
            if (live) {
                __stcs(reinterpret_cast<float2*>(PX + g), make_float2(xe, xo));
                __stcs(reinterpret_cast<float2*>(PY + g), make_float2(ye, yo));
                __stcs(reinterpret_cast<float2*>(PZ + g), make_float2(ze, zo));
            }
        }
        nacc = warp_sum(nacc);
        if (lane == 0 && nacc) atomicAdd(&S->slot_acc[(ti * kMaxWarps + warp) % kSlots], (unsigned long long)nacc);
    }
}

// ------------------------------------------------------------------ field

// omega of one cell from its counts (NT = 0: runtime type count, up to
// kMaxTypes).  Expression order matches the oracle's field_update():
// phi_S = n_S * scale, tot = sum_S phi_S (S ascending), then
// SCMF0: w_T = (tot - 1) cf_TT + sum_{S != T} cf_TS (phi_T - phi_S)
// literal: w_T = (tot - 1) cf_TT + sum_{S != T} cf_TS phi_S.
template <int NT>
__device__ __forceinline__ double omega_of_cell(int nt, const uint32_t* cnt, float scale, bool lit, bool upd, float* w,
                                                const float* cf) {
    constexpr int M = NT > 0 ? NT : kMaxTypes;
    float phi[M];
    float tot = 0.0f;
#pragma unroll
    for (int u = 0; u < M; ++u) {
        if (u < nt) {
            phi[u] = (float)cnt[u] * scale;
            tot = tot + phi[u];
        }
    }
    double ef = 0.0;
#pragma unroll
    for (int t = 0; t < M; ++t) {
        if (t < nt) {
            if (upd) {
                float v = (tot - 1.0f) * cf[t + nt * t];
#pragma unroll
                for (int u = 0; u < M; ++u) {
                    if (u < nt && u != t) {
                        if (!lit)
                            v = v + cf[t + nt * u] * (phi[t] - phi[u]);
                        else
                            v = v + cf[t + nt * u] * phi[u];
                    }
                }
                w[t] = v;
            }
            ef += (double)w[t] * (double)cnt[t];
        }
    }
    return ef;
}

// Scalar path: one cell (any count width, any alignment).
template <int NT, bool FUSED>
__device__ __forceinline__ double field_cell(int n, int64_t cell, int64_t NC, float scale, bool lit, bool upd,
                                             bool c16, const uint32_t* src32, float* W, const float* cf,
                                             unsigned long long* avg, float& wmax, float& wmin) {
    constexpr int M = NT > 0 ? NT : kMaxTypes;
    const int nt = NT > 0 ? NT : n;
    const uint16_t* src16 = reinterpret_cast<const uint16_t*>(src32);
    uint32_t cnt[M];
    float w[M];
#pragma unroll
    for (int u = 0; u < M; ++u) {
        if (u < nt) {
            cnt[u] = c16 ? (uint32_t)src16[u * NC + cell] : src32[u * NC + cell];
            if (!upd) w[u] = W[u * NC + cell];
            if (avg) avg[u * NC + cell] += cnt[u];
        }
    }
    const double ef = omega_of_cell<NT>(nt, cnt, scale, lit, upd, w, cf);
#pragma unroll
    for (int t = 0; t < M; ++t) {
        if (t < nt && upd) W[t * NC + cell] = w[t];
        if (t < nt) {
            wmax = fmaxf(wmax, w[t]);  // fmaxf / fminf skip NaN
            wmin = fminf(wmin, w[t]);
        }
    }
    return ef;
}

// Vector path: four consecutive cells with 16-byte loads and stores (32-bit
// counts, n_cells and the tile start multiples of 4).
template <int NT, bool FUSED>
__device__ __forceinline__ double field_cells4(int64_t cell, int64_t NC, float scale, bool lit, bool upd,
                                               const uint32_t* src32, float* W, const float* cf,
                                               unsigned long long* avg, float& wmax, float& wmin) {
    uint4 cv[NT];
    float4 wv[NT];
#pragma unroll
    for (int u = 0; u < NT; ++u) {
        cv[u] = *reinterpret_cast<const uint4*>(src32 + u * NC + cell);
        if (!upd) wv[u] = *reinterpret_cast<const float4*>(W + u * NC + cell);
    }
    if (avg) {
#pragma unroll
        for (int u = 0; u < NT; ++u) {
            ulonglong2* a = reinterpret_cast<ulonglong2*>(avg + u * NC + cell);
            ulonglong2 lo = a[0], hi = a[1];
            lo.x += cv[u].x; lo.y += cv[u].y;
            hi.x += cv[u].z; hi.y += cv[u].w;
            a[0] = lo;
            a[1] = hi;
        }
    }
    double ef = 0.0;
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        uint32_t cnt[NT];
        float w[NT];
#pragma unroll
        for (int u = 0; u < NT; ++u) {
            cnt[u] = l == 0 ? cv[u].x : l == 1 ? cv[u].y : l == 2 ? cv[u].z : cv[u].w;
            w[u] = l == 0 ? wv[u].x : l == 1 ? wv[u].y : l == 2 ? wv[u].z : wv[u].w;
        }
        ef += omega_of_cell<NT>(NT, cnt, scale, lit, upd, w, cf);
#pragma unroll
        for (int u = 0; u < NT; ++u) {
            wmax = fmaxf(wmax, w[u]);
            wmin = fminf(wmin, w[u]);
            if (l == 0) wv[u].x = w[u];
            else if (l == 1) wv[u].y = w[u];
            else if (l == 2) wv[u].z = w[u];
            else wv[u].w = w[u];
        }
    }
#pragma unroll
    for (int u = 0; u < NT; ++u) {
        if (upd) *reinterpret_cast<float4*>(W + u * NC + cell) = wv[u];
    }
    return ef;
}

// Closes one system after a launch (one block): sums the accept slots and the
// energy partials part[0 .. count) in an order fixed by the block size, and
// thread 0 publishes the statistics and, for a full sweep, advances the step
// and makes the new counts current.  Partials written by other blocks of the
// same launch are read through L2.
__device__ void close_system(SysDev* S, const double* part, int count, int mode, unsigned long long* s_a,
                             double* s_f) {
    const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5;
    unsigned long long a = 0;
    double f = 0.0;
    if ((mode & kCloseMove) && tid < kSlots) {
        a = __ldcg(&S->slot_acc[tid]);
        S->slot_acc[tid] = 0ull;
    }
    if (mode & (kCloseField | kCloseBond))
        for (int i = tid; i < count; i += T) f += __ldcg(part + i);
    a = warp_sum(a);
    f = warp_sum(f);
    if (lane == 0) {
        s_a[warp] = a;
        s_f[warp] = f;
    }
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < (T + 31) / 32; ++w) {
            a += s_a[w];
            f += s_f[w];
        }
        if (mode & kCloseMove) {
            S->last_accepts = a;
            S->total_accepts += a;
            S->total_moves += (unsigned long long)S->n_beads;
        }
        if (mode & kCloseField) S->e_field = f;
        if (mode & kCloseBond) {
            S->e_bond = f;
            S->e_bond_step = S->step + 1u;
        }
        if ((mode & kCloseAverage) && S->avg && S->avg_every && ((S->step + 1u) % S->avg_every) == 0u)
            S->avg_samples += 1ull;
        if (mode & kCloseAdvance) S->step += 1u;
    }
    __syncthreads();
}

// Order-preserving integer key of a non-NaN float (for atomicMax / atomicMin)
// and its inverse.
__device__ __forceinline__ uint32_t ord_key(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord_val(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

template <bool FUSED, int NT>
__global__ void __launch_bounds__(256) k_field(const FieldTile* __restrict__ tiles, int n_tiles, int force_update,
                                                double* __restrict__ ef_part, int close_mode) {
    __shared__ double s_ef[32];
    __shared__ float s_mx[32], s_mn[32];
    __shared__ unsigned long long s_acc[32];
    __shared__ float cf[kMaxTypes * kMaxTypes];
    __shared__ int s_last;
    const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5;
    for (int ti = blockIdx.x; ti < n_tiles; ti += gridDim.x) {
        const FieldTile t = tiles[ti];
        SysDev* S = t.sys;
        if (FUSED && S->step >= S->stop_step) continue;  // block-uniform: the system's sweeps are done
        for (int i = tid; i < kMaxTypes * kMaxTypes; i += T) cf[i] = S->cf[i];
        __syncthreads();
        const uint32_t cur = S->cur;
        const uint32_t sweep = S->step + 1u;
        const bool upd = force_update || S->field_rule == 1 || (sweep % 10u) != 0u;
        const int n = S->n_types;
        const int64_t NC = S->n_cells;
        const float scale = S->scale;
        const bool lit = S->hamiltonian == 1;
        const bool c16 = S->count16 != 0;
        const uint32_t* src32 = S->field_counts ? S->field_counts : S->counts[cur];
        float* W = S->omega;
        // the fused sweep samples the time-averaged density at every avg_every-th sweep
        unsigned long long* avg = FUSED && S->avg && S->avg_every && (sweep % S->avg_every) == 0u ? S->avg : nullptr;
        double ef = 0.0;
        float wmax = -INFINITY, wmin = INFINITY;  // omega of the tile's cells (new or kept)
        const int64_t end = t.cell0 + t.n_cells;
        if (NT > 0 && !c16 && (NC & 3) == 0 && (t.cell0 & 3) == 0 && (t.n_cells & 3) == 0) {
            for (int64_t cell = t.cell0 + 4 * tid; cell < end; cell += 4 * T)
                ef += field_cells4<(NT > 0 ? NT : 1), FUSED>(cell, NC, scale, lit, upd, src32, W, cf, avg, wmax, wmin);
        } else {
            for (int64_t cell = t.cell0 + tid; cell < end; cell += T)
                ef += field_cell<NT, FUSED>(n, cell, NC, scale, lit, upd, c16, src32, W, cf, avg, wmax, wmin);
        }
        ef = warp_sum(ef);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            wmax = fmaxf(wmax, __shfl_xor_sync(0xffffffffu, wmax, o));
            wmin = fminf(wmin, __shfl_xor_sync(0xffffffffu, wmin, o));
        }
        if (lane == 0) {
            s_ef[warp] = ef;
            s_mx[warp] = wmax;
            s_mn[warp] = wmin;
        }
        __syncthreads();
        if (tid == 0) {
            double e = 0.0;
            for (int w = 0; w < (T + 31) / 32; ++w) {
                e += s_ef[w];
                wmax = fmaxf(wmax, s_mx[w]);
                wmin = fminf(wmin, s_mn[w]);
            }
            ef_part[ti] = e;
            if (wmax >= wmin) {  // the tile held a non-NaN omega
                atomicMax(&S->om_max_key, ord_key(wmax));
                atomicMin(&S->om_min_key, ord_key(wmin));
            }
            if (close_mode) {
                // publish the partial, then count the tile; the block that
                // finishes a system's last tile closes it (no waiting)
                __threadfence();
                const unsigned done = atomicAdd(&S->field_done, 1u) + 1u;
                s_last = done == (unsigned)t.n_tiles_sys;
            }
        }
        __syncthreads();
        if (close_mode && s_last) {
            __threadfence();
            if (tid == 0) {
                // every tile of the system has folded its omega in: publish the
                // span (+inf when no bound is known) and reset the keys
                const uint32_t kx = atomicExch(&S->om_max_key, 0u);
                const uint32_t kn = atomicExch(&S->om_min_key, 0xFFFFFFFFu);
                const float span = kx >= kn ? __fsub_rn(ord_val(kx), ord_val(kn)) : INFINITY;
                S->omega_span = span >= 0.0f ? span : INFINITY;  // NaN (inf - inf): no bound
            }
            close_system(S, ef_part + t.first_tile, t.n_tiles_sys, close_mode, s_acc, s_ef);
            if (tid == 0) S->field_done = 0u;
        }
        __syncthreads();
    }
}

// Closes a launch for every system of the plan (one block per system): the
// sums of close_system over each system's tile ranges.
__global__ void __launch_bounds__(256) k_close(const SysClose* __restrict__ list, int n_sys,
                                                const unsigned* __restrict__ acc_part, int warps_per_tile,
                                                const double* __restrict__ ef_part, const double* __restrict__ eb_part,
                                                int mode) {
    __shared__ unsigned long long s_a[32];
    __shared__ double s_f[32];
    for (int si = blockIdx.x; si < n_sys; si += gridDim.x) {
        const SysClose L = list[si];
        if (mode & kCloseBond)
            close_system(L.sys, eb_part + L.move_first, L.move_count, mode, s_a, s_f);
        else
            close_system(L.sys, ef_part + L.field_first, L.field_count, mode, s_a, s_f);
    }
}

// Bond energy sum_bonds k |r_i - r_j|^2 of the current positions, each bond
// once, one partial per tile (closed by k_close with kCloseBond).
__global__ void __launch_bounds__(256) k_bond_energy(const MoveTile* __restrict__ tiles, int n_tiles,
                                                      double* __restrict__ eb_part) {
    __shared__ double s_e[32];
    const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5;
    for (int ti = blockIdx.x; ti < n_tiles; ti += gridDim.x) {
        const MoveTile t = tiles[ti];
        SysDev* S = t.sys;
        const ArchDev* Ap = t.arch;
        const int L = Ap->length;
        const int nb = t.n_chains * L;
        const float* X = S->x + t.bead0;
        const float* Y = S->y + t.bead0;
        const float* Z = S->z + t.bead0;
        const float k = S->k;
        double e = 0.0;
        for (int i = tid; i < nb; i += T) {
            const int cl = (int)div_magic((uint32_t)i, Ap->len_magic, L);
            const int b = i - cl * L;
            const BeadInfo bi = Ap->beads[b];
            for (int d = 0; d < bi.deg; ++d) {
                const int j = bi.nbr[d];
                if (j <= b) continue;
                const int jj = cl * L + j;
                const float ex = X[i] - X[jj], ey = Y[i] - Y[jj], ez = Z[i] - Z[jj];
                e += (double)k * (double)(ex * ex + ey * ey + ez * ez);
            }
        }
        e = warp_sum(e);
        if (lane == 0) s_e[warp] = e;
        __syncthreads();
        if (tid == 0) {
            double a = 0.0;
            for (int w = 0; w < (T + 31) / 32; ++w) a += s_e[w];
            eb_part[ti] = a;
        }
        __syncthreads();
    }
}

// Adds the current counts into the time-averaged density accumulator and
// counts the sample (a sample taken outside the fused sweep).
__global__ void k_average_sample(SysDev* S, int64_t n) {
    const uint32_t* c32 = S->counts[S->cur];
    const uint16_t* c16 = reinterpret_cast<const uint16_t*>(c32);
    const bool half = S->count16 != 0;
    unsigned long long* avg = S->avg;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        avg[i] += half ? (unsigned long long)c16[i] : (unsigned long long)c32[i];
    if (blockIdx.x == 0 && threadIdx.x == 0) S->avg_samples += 1ull;
}

// Chain observables in double, one warp per chain and one partial row of
// kObsSlots sums per move tile (fixed reduction order).  Per chain:
// R_e = last bead - first bead (test.cpp:47-68 takes beads 0 and 31 of every
// chain); R_g^2 = mean |r - r_cm|^2; bonds counted once (j > i); with a
// reference snapshot, bead and centre-of-mass displacements.  Ana_Info
// (struct.h:65-75) names these analyses; the reference computes only R_e.
__global__ void __launch_bounds__(256) k_observables(const MoveTile* __restrict__ tiles, int n_tiles,
                                                      const float* __restrict__ ref, int64_t n_beads_sys,
                                                      double* __restrict__ part) {
    __shared__ double s_w[kMaxWarps][kObsSlots];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
    for (int ti = blockIdx.x; ti < n_tiles; ti += gridDim.x) {
        const MoveTile t = tiles[ti];
        const SysDev* S = t.sys;
        const ArchDev* Ap = t.arch;
        const int L = Ap->length;
        double acc[kObsSlots];
#pragma unroll
        for (int k = 0; k < kObsSlots; ++k) acc[k] = 0.0;
        for (int cl = warp; cl < t.n_chains; cl += nwarps) {
            const int64_t b0 = t.bead0 + (int64_t)cl * L;
            const float* X = S->x + b0;
            const float* Y = S->y + b0;
            const float* Z = S->z + b0;
            double sx = 0.0, sy = 0.0, sz = 0.0, rx = 0.0, ry = 0.0, rz = 0.0;
            double bx = 0.0, by = 0.0, bz = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
            for (int b = lane; b < L; b += 32) {
                const double x = X[b], y = Y[b], z = Z[b];
                sx += x; sy += y; sz += z;
                const BeadInfo bi = Ap->beads[b];
                for (int d = 0; d < bi.deg; ++d) {
                    const int j = bi.nbr[d];
                    if (j <= b) continue;
                    const double ex = (double)X[j] - x, ey = (double)Y[j] - y, ez = (double)Z[j] - z;
                    bx += ex * ex; by += ey * ey; bz += ez * ez;
                }
                if (ref) {
                    const double ux = x - (double)ref[b0 + b], uy = y - (double)ref[n_beads_sys + b0 + b],
                                 uz = z - (double)ref[2 * n_beads_sys + b0 + b];
                    mx += ux * ux; my += uy * uy; mz += uz * uz;
                    rx += (double)ref[b0 + b];
                    ry += (double)ref[n_beads_sys + b0 + b];
                    rz += (double)ref[2 * n_beads_sys + b0 + b];
                }
            }
            sx = warp_sum(sx); sy = warp_sum(sy); sz = warp_sum(sz);
            const double cx = sx / L, cy = sy / L, cz = sz / L;
            double gx = 0.0, gy = 0.0, gz = 0.0;
            for (int b = lane; b < L; b += 32) {
                const double ux = (double)X[b] - cx, uy = (double)Y[b] - cy, uz = (double)Z[b] - cz;
                gx += ux * ux; gy += uy * uy; gz += uz * uz;
            }
            gx = warp_sum(gx); gy = warp_sum(gy); gz = warp_sum(gz);
            bx = warp_sum(bx); by = warp_sum(by); bz = warp_sum(bz);
            if (ref) {
                mx = warp_sum(mx); my = warp_sum(my); mz = warp_sum(mz);
                rx = warp_sum(rx); ry = warp_sum(ry); rz = warp_sum(rz);
            }
            if (lane == 0) {
                const double ex = (double)X[L - 1] - (double)X[0], ey = (double)Y[L - 1] - (double)Y[0],
                             ez = (double)Z[L - 1] - (double)Z[0];
                acc[kObsRe] += ex * ex; acc[kObsRe + 1] += ey * ey; acc[kObsRe + 2] += ez * ez;
                acc[kObsRg] += gx / L; acc[kObsRg + 1] += gy / L; acc[kObsRg + 2] += gz / L;
                acc[kObsBond] += bx; acc[kObsBond + 1] += by; acc[kObsBond + 2] += bz;
                if (ref) {
                    acc[kObsMsd] += mx; acc[kObsMsd + 1] += my; acc[kObsMsd + 2] += mz;
                    const double dx = cx - rx / L, dy = cy - ry / L, dz = cz - rz / L;
                    acc[kObsMsdCom] += dx * dx; acc[kObsMsdCom + 1] += dy * dy; acc[kObsMsdCom + 2] += dz * dz;
                }
            }
        }
        if (lane == 0)
            for (int k = 0; k < kObsSlots; ++k) s_w[warp][k] = acc[k];
        __syncthreads();
        if (tid < kObsSlots) {
            double a = 0.0;
            for (int w = 0; w < nwarps; ++w) a += s_w[w][tid];
            part[(int64_t)ti * kObsSlots + tid] = a;
        }
        __syncthreads();
    }
}

// State checks of scmf_validate (counters in out[], no trap).
__global__ void k_validate_positions(const SysDev* S, int64_t n, unsigned long long* out) {
    unsigned long long bad = 0, far = 0;
    const float lim = 0x1p22f;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float x = S->x[i], y = S->y[i], z = S->z[i];
        if (!isfinite(x) || !isfinite(y) || !isfinite(z)) {
            ++bad;
            continue;
        }
        if (fabsf(x * S->inv_dx) >= lim || fabsf(y * S->inv_dy) >= lim || fabsf(z * S->inv_dz) >= lim) ++far;
    }
    bad = warp_sum(bad);
    far = warp_sum(far);
    if ((threadIdx.x & 31) == 0 && (bad | far)) {
        atomicAdd(out + 0, bad);
        atomicAdd(out + 1, far);
    }
}

__global__ void k_validate_cells(const SysDev* S, const uint32_t* a, const uint32_t* b, int64_t n_words,
                                 int64_t n_values, unsigned long long* out, unsigned long long* sums) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    unsigned long long diff = 0, bad = 0;
    for (int64_t i = i0; i < n_words; i += stride) diff += a[i] != b[i] ? 1ull : 0ull;
    for (int64_t i = i0; i < n_values; i += stride)
        if (!isfinite(S->omega[i])) ++bad;
    const bool c16 = S->count16 != 0;
    const uint16_t* a16 = reinterpret_cast<const uint16_t*>(a);
    const int64_t nc = S->n_cells;
    for (int t = 0; t < S->n_types; ++t) {
        unsigned long long v = 0;
        for (int64_t c = i0; c < nc; c += stride)
            v += c16 ? (unsigned long long)a16[t * nc + c] : (unsigned long long)a[t * nc + c];
        v = warp_sum(v);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(sums + t, v);
    }
    diff = warp_sum(diff);
    bad = warp_sum(bad);
    if ((threadIdx.x & 31) == 0 && (diff | bad)) {
        atomicAdd(out + 2, diff);
        atomicAdd(out + 3, bad);
    }
}

// ------------------------------------------------------------- transposes
__device__ __forceinline__ int64_t aos_bead_of(const SysDev* S, const ArchDev* archs, int n_arch, int64_t i) {
    int a = 0;
    while (a + 1 < n_arch && i >= archs[a + 1].bead_base) ++a;
    const ArchDev& A = archs[a];
    const int64_t r = i - A.bead_base;
    const int64_t slot_local = r / A.length;
    const int64_t b = r - slot_local * A.length;
    const uint32_t gc = S->chain_id[A.chain_base + slot_local];
    return A.bead_base + (int64_t)(gc - (uint32_t)A.rng_base) * A.length + b;
}

__global__ void k_aos_to_soa(const float* __restrict__ aos, SysDev* S, const ArchDev* archs, int n_arch,
                             int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t src = aos_bead_of(S, archs, n_arch, i);
        S->x[i] = aos[3 * src];
        S->y[i] = aos[3 * src + 1];
        S->z[i] = aos[3 * src + 2];
    }
}

__global__ void k_soa_to_aos(float* __restrict__ aos, const SysDev* S, const ArchDev* archs, int n_arch,
                             int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t dst = aos_bead_of(S, archs, n_arch, i);
        aos[3 * dst] = S->x[i];
        aos[3 * dst + 1] = S->y[i];
        aos[3 * dst + 2] = S->z[i];
    }
}

__global__ void k_unpack16(const SysDev* S, uint32_t* out, int64_t n) {
    const uint16_t* src = reinterpret_cast<const uint16_t*>(S->counts[S->cur]);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = src[i];
}

// ------------------------------------------------------------ diagnostics
__global__ void k_debug_math(uint32_t k0, uint32_t k1, int n, uint32_t* words, float* logs, float* normals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4 w = philox4x32_10(make_uint4((uint32_t)i, 0u, 0u, 0u), k0, k1);
    words[4 * i] = w.x;
    words[4 * i + 1] = w.y;
    words[4 * i + 2] = w.z;
    words[4 * i + 3] = w.w;
    logs[i] = log_f(u01(w.w));
    float n0, n1, n2;
    normals3(w, normal_table(), n0, n1, n2);
    normals[3 * i] = n0;
    normals[3 * i + 1] = n1;
    normals[3 * i + 2] = n2;
}

// -------------------------------------------------------------- launchers
int launch_debug_math(uint32_t k0, uint32_t k1, int n, uint32_t* words, float* logs, float* normals, void* stream) {
    k_debug_math<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(k0, k1, n, words, logs, normals);
    return (int)cudaGetLastError();
}

int sm_count() {
    static std::mutex mu;
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    std::lock_guard<std::mutex> g(mu);
    if (cached[dev] == 0) {
        int n = 0;
        cached[dev] = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && n > 0 ? n : 148;
    }
    return cached[dev];
}

static int grid_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    const int64_t cap = (int64_t)sm_count() * 32;
    if (b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

// The statistics of the last sweep in the public layout (scmf_get_sweep_stats).
__global__ void k_stats_out(SysDev* S) {
    scmf_stats o;
    o.step = S->step;
    o.last_accepts = S->last_accepts;
    o.total_accepts = S->total_accepts;
    o.total_moves = S->total_moves;
    o.e_bond = S->e_bond_step == S->step + 1u ? S->e_bond : __longlong_as_double(0x7FF8000000000000ll);
    o.e_field = S->e_field;
    o.error_word = S->error_word;
    o.reserved = 0u;
    S->stats_out = o;
}

__global__ void k_copy_counts(const SysDev* __restrict__ S, uint32_t* __restrict__ dst, int64_t n) {
    const uint32_t* src = S->counts[S->cur];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

int launch_copy_counts(const SysDev* d_sys, uint32_t* dst, int64_t n_words, void* stream) {
    k_copy_counts<<<grid_for(n_words, 256), 256, 0, (cudaStream_t)stream>>>(d_sys, dst, n_words);
    return (int)cudaGetLastError();
}

int launch_stats_out(SysDev* d_sys, void* stream) {
    k_stats_out<<<1, 1, 0, (cudaStream_t)stream>>>(d_sys);
    return (int)cudaGetLastError();
}

int launch_init_coords(SysDev* d_sys, const ArchDev* d_arch, int n_arch, int n_chains, void* stream) {
    if (n_chains <= 0) return 0;
    const int th = 128;
    k_init_coords<<<(n_chains + th - 1) / th, th, 0, (cudaStream_t)stream>>>(d_sys, d_arch, n_arch, n_chains);
    return (int)cudaGetLastError();
}

// Opt the sweep kernels in to the largest dynamic shared memory once, outside
// any stream capture (called when a system is created).
template <int MODE, int KEYS>
static cudaError_t allow_smem(int bytes) {
    cudaError_t e = cudaFuncSetAttribute(k_sweep<MODE, false, KEYS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_sweep_linear<MODE, KEYS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    return e;
}

int configure_kernels() {
    // once per device, with that device current
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    cudaError_t e0 = cudaGetDevice(&dev);
    if (e0 != cudaSuccess) return (int)e0;
    std::lock_guard<std::mutex> g(mu);
    if (dev >= 0 && dev < 64 && done[dev]) return 0;
    int2 fold_tab[257] = {};
    for (uint32_t n = 2; n <= 256; ++n) {
        const uint32_t bias = n * (((1u << 22) + n - 1) / n);  // a multiple of n, at least 2^22
        fold_tab[n] = make_int2((int)(0x4B400000u - bias), (int)(uint32_t)(((1ull << 32) + n - 1) / n));
    }
    cudaError_t ef = cudaMemcpyToSymbol(c_fold, fold_tab, sizeof fold_tab);
    if (ef != cudaSuccess) return (int)ef;
    ef = cudaFuncSetAttribute(k_sweep_lean<kMoveOnly>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLeanSmem);
    if (ef == cudaSuccess)
        ef = cudaFuncSetAttribute(k_sweep_lean<kMoveGrid>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLeanSmem);
    if (ef != cudaSuccess) return (int)ef;
    const int bytes = (int)sweep_smem_bytes(kMaxTileBeads, kMaxLength);
    cudaError_t e = cudaSuccess;
    for (int keys = kKeysNone; keys <= kKeysBoth && e == cudaSuccess; ++keys) {
        if (keys == kKeysNone) {
            e = allow_smem<kGridOnly, kKeysNone>(bytes);
            if (e == cudaSuccess) e = allow_smem<kMoveOnly, kKeysNone>(bytes);
            if (e == cudaSuccess) e = allow_smem<kMoveGrid, kKeysNone>(bytes);
        } else if (keys == kKeysHigh) {
            e = allow_smem<kMoveOnly, kKeysHigh>(bytes);
            if (e == cudaSuccess) e = allow_smem<kMoveGrid, kKeysHigh>(bytes);
        } else {
            e = allow_smem<kMoveOnly, kKeysBoth>(bytes);
            if (e == cudaSuccess) e = allow_smem<kMoveGrid, kKeysBoth>(bytes);
        }
    }
    if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev] = true;
    return (int)e;
}

template <int MODE, bool FLAT>
static void launch_reg(const LaunchShape& sh, int blocks, int threads, cudaStream_t st, const MoveTile* tiles,
                       const int32_t* list, int n, unsigned* acc) {
    const int keys = MODE == kGridOnly ? kKeysNone : sh.keyed;
    if constexpr (MODE != kGridOnly && !FLAT) {
        if (sh.lean && keys == kKeysBoth && sh.fold == 0 && !list) {
            k_sweep_lean<MODE><<<sm_count(), kLeanThreads, kLeanSmem, st>>>(sh.keys, sh.sc);
            return;
        }
        if (sh.warp_even) {
            if (keys == kKeysBoth) {
                if (sh.fold == 0) k_sweep_leanm<MODE, 0, kKeysBoth><<<blocks, threads, 0, st>>>(tiles, list, n, sh.keys);
                else k_sweep_leanm<MODE, -1, kKeysBoth><<<blocks, threads, 0, st>>>(tiles, list, n, sh.keys);
            } else if (keys == kKeysHigh) {
                if (sh.fold == 0) k_sweep_leanm<MODE, 0, kKeysHigh><<<blocks, threads, 0, st>>>(tiles, list, n, sh.keys);
                else k_sweep_leanm<MODE, -1, kKeysHigh><<<blocks, threads, 0, st>>>(tiles, list, n, sh.keys);
            } else {
                if (sh.fold == 0) k_sweep_leanm<MODE, 0, kKeysNone><<<blocks, threads, 0, st>>>(tiles, list, n, sh.keys);
                else k_sweep_leanm<MODE, -1, kKeysNone><<<blocks, threads, 0, st>>>(tiles, list, n, sh.keys);
            }
            return;
        }
    }
    if (keys == kKeysBoth) {
        if (sh.fold == 0)
            k_sweep_reg<MODE, FLAT, 0, kKeysBoth><<<blocks, threads, 0, st>>>(tiles, list, n, acc, sh.keys);
        else
            k_sweep_reg<MODE, FLAT, -1, kKeysBoth><<<blocks, threads, 0, st>>>(tiles, list, n, acc, sh.keys);
    } else if (keys == kKeysHigh) {
        if (sh.fold == 0)
            k_sweep_reg<MODE, FLAT, 0, kKeysHigh><<<blocks, threads, 0, st>>>(tiles, list, n, acc, sh.keys);
        else
            k_sweep_reg<MODE, FLAT, -1, kKeysHigh><<<blocks, threads, 0, st>>>(tiles, list, n, acc, sh.keys);
    } else {
        if (sh.fold == 0)
            k_sweep_reg<MODE, FLAT, 0, kKeysNone><<<blocks, threads, 0, st>>>(tiles, list, n, acc, sh.keys);
        else
            k_sweep_reg<MODE, FLAT, -1, kKeysNone><<<blocks, threads, 0, st>>>(tiles, list, n, acc, sh.keys);
    }
}

template <int MODE>
static int launch_sweep_t(const MoveTile* tiles, int n_tiles, int mtb, int ml, LaunchShape sh, unsigned* acc,
                          cudaStream_t st) {
    if (mtb > kMaxTileBeads || ml > kMaxLength || sh.threads > 256 || sh.threads < 32) return (int)cudaErrorInvalidValue;
    const int blocks = sh.blocks > 0 ? sh.blocks : n_tiles;
    const int keys = MODE == kGridOnly ? kKeysNone : sh.keyed;
    if (sh.linear && ml <= 64) {
        // tiles whose chains fill warps exactly run the barrier-free kernel,
        // the others (sh.flat_list) the block-wide one: one launch each
        const int n_warp = sh.n_flat > 0 ? sh.n_warp : n_tiles;
        const int32_t* warp_list = sh.n_flat > 0 ? sh.warp_list : nullptr;
        if (n_warp > 0 && sh.part != 2)
            launch_reg<MODE, false>(sh, sh.blocks > 0 ? min(sh.blocks, n_warp) : n_warp, sh.threads, st, tiles,
                                    warp_list, n_warp, acc);
        if (sh.n_flat > 0 && sh.part != 1)
            launch_reg<MODE, true>(sh, sh.blocks > 0 ? min(sh.blocks, sh.n_flat) : sh.n_flat,
                                   sh.flat_threads > 0 ? sh.flat_threads : sh.threads, st, tiles, sh.flat_list,
                                   sh.n_flat, acc);
    } else if (sh.linear) {
        // per-warp slice: ceil(chains per tile / warps) chains of the longest length
        const int nw = sh.threads / 32;
        const int wb = ((sh.max_chains + nw - 1) / nw) * ml;
        const size_t smem = (size_t)nw * 3 * wb * sizeof(float);
        if (smem > sweep_smem_bytes(kMaxTileBeads, kMaxLength)) return (int)cudaErrorInvalidValue;
        if (keys == kKeysBoth)
            k_sweep_linear<MODE, kKeysBoth><<<blocks, sh.threads, smem, st>>>(tiles, nullptr, n_tiles, wb, acc, sh.keys);
        else if (keys == kKeysHigh)
            k_sweep_linear<MODE, kKeysHigh><<<blocks, sh.threads, smem, st>>>(tiles, nullptr, n_tiles, wb, acc, sh.keys);
        else
            k_sweep_linear<MODE, kKeysNone><<<blocks, sh.threads, smem, st>>>(tiles, nullptr, n_tiles, wb, acc, sh.keys);
    } else {
        const size_t smem = sweep_smem_bytes(mtb, ml);
        if (keys == kKeysBoth)
            k_sweep<MODE, false, kKeysBoth><<<blocks, sh.threads, smem, st>>>(tiles, n_tiles, mtb, ml, acc, sh.keys);
        else if (keys == kKeysHigh)
            k_sweep<MODE, false, kKeysHigh><<<blocks, sh.threads, smem, st>>>(tiles, n_tiles, mtb, ml, acc, sh.keys);
        else
            k_sweep<MODE, false, kKeysNone><<<blocks, sh.threads, smem, st>>>(tiles, n_tiles, mtb, ml, acc, sh.keys);
    }
    return (int)cudaGetLastError();
}

int launch_sweep(int mode, const MoveTile* tiles, int n_tiles, int mtb, int ml, LaunchShape sh, unsigned* acc_part,
                 void* stream) {
    if (n_tiles <= 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    if (mode == kMoveOnly) return launch_sweep_t<kMoveOnly>(tiles, n_tiles, mtb, ml, sh, acc_part, st);
    if (mode == kMoveGrid) return launch_sweep_t<kMoveGrid>(tiles, n_tiles, mtb, ml, sh, acc_part, st);
    return launch_sweep_t<kGridOnly>(tiles, n_tiles, mtb, ml, sh, acc_part, st);
}

template <bool FUSED>
static void launch_field_t(int nt, const FieldTile* tiles, int n_tiles, int force_update, int blocks, int threads,
                           double* ef, int close_mode, cudaStream_t st) {
    if (nt == 2)
        k_field<FUSED, 2><<<blocks, threads, 0, st>>>(tiles, n_tiles, force_update, ef, close_mode);
    else if (nt == 3)
        k_field<FUSED, 3><<<blocks, threads, 0, st>>>(tiles, n_tiles, force_update, ef, close_mode);
    else if (nt == 1)
        k_field<FUSED, 1><<<blocks, threads, 0, st>>>(tiles, n_tiles, force_update, ef, close_mode);
    else
        k_field<FUSED, 0><<<blocks, threads, 0, st>>>(tiles, n_tiles, force_update, ef, close_mode);
}

int launch_field(bool fused, int force_update, const FieldTile* tiles, int n_tiles, LaunchShape sh, double* ef_part,
                 int close_mode, void* stream) {
    if (n_tiles <= 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    const int blocks = sh.blocks > 0 ? sh.blocks : n_tiles;
    const int threads = sh.threads > 256 ? 256 : sh.threads;
    if (fused)
        launch_field_t<true>(sh.n_types, tiles, n_tiles, force_update, blocks, threads, ef_part, close_mode, st);
    else
        launch_field_t<false>(sh.n_types, tiles, n_tiles, force_update, blocks, threads, ef_part, close_mode, st);
    return (int)cudaGetLastError();
}

int launch_bond_energy(const MoveTile* tiles, int n_tiles, LaunchShape sh, double* eb_part, void* stream) {
    if (n_tiles <= 0) return 0;
    k_bond_energy<<<n_tiles, sh.threads > 256 ? 256 : sh.threads, 0, (cudaStream_t)stream>>>(tiles, n_tiles, eb_part);
    return (int)cudaGetLastError();
}

int launch_close(const SysClose* list, int n_sys, const unsigned* acc_part, int warps_per_tile, const double* ef_part,
                 const double* eb_part, int mode, void* stream) {
    if (n_sys <= 0) return 0;
    k_close<<<n_sys < 1024 ? n_sys : 1024, 256, 0, (cudaStream_t)stream>>>(list, n_sys, acc_part, warps_per_tile,
                                                                             ef_part, eb_part, mode);
    return (int)cudaGetLastError();
}

// One chunk of a chunked upload: positions of storage beads [i0, i1) (the
// AoS bead of storage bead i is bead i: chain ids are the identity plus each
// architecture's random-stream base) and their counts into counts[0].
__global__ void k_aos_chunk(const float* __restrict__ aos, SysDev* S, const ArchDev* archs, int n_arch, int64_t i0,
                            int64_t i1) {
    MoveConsts c;
    c.k = S->k; c.k2 = S->k2; c.A = S->A; c.R = S->R;
    c.inv_dx = S->inv_dx; c.inv_dy = S->inv_dy; c.inv_dz = S->inv_dz;
    load_fold(c, S);
    const int64_t NC = S->n_cells;
    uint32_t* cnt = S->counts[0];
    const bool c16 = S->count16 != 0;
    for (int64_t i = i0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < i1; i += (int64_t)gridDim.x * blockDim.x) {
        const float x = aos[3 * i], y = aos[3 * i + 1], z = aos[3 * i + 2];
        S->x[i] = x;
        S->y[i] = y;
        S->z[i] = z;
        int a = 0;
        while (a + 1 < n_arch && i >= archs[a + 1].bead_base) ++a;
        const ArchDev& A = archs[a];
        const int r = (int)(i - A.bead_base);  // systems hold fewer than 2^31 beads
        const int b = r % A.length;
        const int64_t idx = (int64_t)A.types[b] * NC + cell_of(c, x, y, z);
        if (c16)
            atomicAdd(cnt + (idx >> 1), 1u << ((idx & 1) * 16));
        else
            atomicAdd(cnt + idx, 1u);
    }
}

int launch_aos_chunk(const float* aos, SysDev* sys, const ArchDev* arch, int n_arch, int64_t i0, int64_t i1,
                     void* stream) {
    if (i1 <= i0) return 0;
    k_aos_chunk<<<grid_for(i1 - i0, 256), 256, 0, (cudaStream_t)stream>>>(aos, sys, arch, n_arch, i0, i1);
    return (int)cudaGetLastError();
}

int launch_aos_to_soa(const float* aos, SysDev* sys, const ArchDev* arch, int n_arch, int64_t n, void* stream) {
    if (n <= 0) return 0;
    k_aos_to_soa<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(aos, sys, arch, n_arch, n);
    return (int)cudaGetLastError();
}

int launch_soa_to_aos(float* aos, const SysDev* sys, const ArchDev* arch, int n_arch, int64_t n, void* stream) {
    if (n <= 0) return 0;
    k_soa_to_aos<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(aos, sys, arch, n_arch, n);
    return (int)cudaGetLastError();
}

int launch_unpack_counts16(const SysDev* sys, uint32_t* out, int64_t n, void* stream) {
    if (n <= 0) return 0;
    k_unpack16<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(sys, out, n);
    return (int)cudaGetLastError();
}
int launch_validate_positions(const SysDev* sys, int64_t n, unsigned long long* out, void* stream) {
    if (n <= 0) return 0;
    k_validate_positions<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(sys, n, out);
    return (int)cudaGetLastError();
}
int launch_validate_cells(const SysDev* sys, const uint32_t* a, const uint32_t* b, int64_t n_words, int64_t n_values,
                          unsigned long long* out, unsigned long long* sums, void* stream) {
    const int64_t n = n_words > n_values ? n_words : n_values;
    if (n <= 0) return 0;
    k_validate_cells<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(sys, a, b, n_words, n_values, out, sums);
    return (int)cudaGetLastError();
}
int launch_average_sample(SysDev* sys, int64_t n, void* stream) {
    if (n <= 0) return 0;
    k_average_sample<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(sys, n);
    return (int)cudaGetLastError();
}
int launch_observables(const MoveTile* tiles, int n_tiles, const float* ref_xyz, int64_t n_beads_sys, double* part,
                       void* stream) {
    if (n_tiles <= 0) return 0;
    k_observables<<<n_tiles, 256, 0, (cudaStream_t)stream>>>(tiles, n_tiles, ref_xyz, n_beads_sys, part);
    return (int)cudaGetLastError();
}

}  // namespace scmf

// ---------------------------------------------------------------------------
// Field update without allocation.
//
// For callers that cannot call cudaMalloc (code that runs where allocation is
// forbidden or must not stall, such as a step that is replayed inside someone
// else's captured stream work, or an embedding application that owns all
// device memory and hands out only pointers to its own buffers), the omega
// update of caller-owned counts into caller-owned omega is offered with its
// only scratch, the per-tile partial sums of the field energy, held in a fixed
// array in this library's device memory.  Every GPU that loads the library
// holds that array (kNoAllocMaxTiles doubles, 16 KiB) until the process exits.
namespace scmf {

constexpr int kNoAllocTileCells = 4096;
constexpr int kNoAllocMaxTiles = 2048;  // n_cells <= 2048 * 4096 = 8,388,608

static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxTiles];

struct FieldParams {
    int64_t n_cells;
    float scale;
    int n_types;
    int lit;
    float cf[kMaxTypes * kMaxTypes];
};

// One tile of kNoAllocTileCells cells per block: omega of every cell and the
// tile's field energy sum_T omega_T n_T into partials[tile] (no atomics).
__global__ void __launch_bounds__(256) k_field_noalloc(const uint32_t* __restrict__ counts, float* __restrict__ omega,
                                                        FieldParams p, double* __restrict__ partials) {
    __shared__ double s_ef[32];
    __shared__ float cf[kMaxTypes * kMaxTypes];
    const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < kMaxTypes * kMaxTypes; i += T) cf[i] = p.cf[i];
    __syncthreads();
    const int64_t c0 = (int64_t)blockIdx.x * kNoAllocTileCells;
    const int64_t c1 = min(c0 + (int64_t)kNoAllocTileCells, p.n_cells);
    double ef = 0.0;
    float wmax = -INFINITY, wmin = INFINITY;  // not used: the caller's omega has no span slot
    for (int64_t cell = c0 + tid; cell < c1; cell += T)
        ef += field_cell<0, false>(p.n_types, cell, p.n_cells, p.scale, p.lit != 0, true, false, counts, omega, cf,
                                   nullptr, wmax, wmin);
    ef = warp_sum(ef);
    if (lane == 0) s_ef[warp] = ef;
    __syncthreads();
    if (tid == 0) {
        double e = 0.0;
        for (int w = 0; w < (T + 31) / 32; ++w) e += s_ef[w];
        partials[blockIdx.x] = e;
    }
}

// Sum of the tile partials in a fixed order (one block).
__global__ void __launch_bounds__(256) k_sum_partials(const double* __restrict__ partials, int n,
                                                       double* __restrict__ out) {
    __shared__ double s[256];
    double e = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) e += partials[i];
    s[threadIdx.x] = e;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

// The id of the calling thread's current CUDA context (0 when none is current
// or the driver cannot tell).  Taken through the driver entry points, so the
// library needs no link against libcuda.
static unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, nullptr) == cudaSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, nullptr) == cudaSuccess)
            get_id = reinterpret_cast<GetId>(f);
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of the scratch array for the current device.  The host-side
// name of a __device__ variable is only a stand-in for it and must never be
// passed to a kernel.  The address is looked up (with the device current) on
// the first call in a context and cached with that context's id; a context
// created later on the device (after cudaDeviceReset, or when the primary
// context was released and retained again) loads the module anew, so its id
// differs and the address is looked up again.  Without a context id from the
// driver it is looked up on every call.
static double* noalloc_scratch(int device, cudaError_t* err) {
    struct Entry {
        unsigned long long ctx;
        double* addr;
    };
    static std::mutex mu;
    static Entry cache[64] = {};
    if (device < 0 || device >= 64) {
        *err = cudaErrorInvalidDevice;
        return nullptr;
    }
    std::lock_guard<std::mutex> g(mu);
    const unsigned long long ctx = current_context_id();
    if (ctx != 0 && cache[device].ctx == ctx && cache[device].addr) {
        *err = cudaSuccess;
        return cache[device].addr;
    }
    void* p = nullptr;
    *err = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (*err != cudaSuccess) return nullptr;
    // the lookup makes the device's context current if none was: take its id now
    cache[device] = Entry{current_context_id(), static_cast<double*>(p)};
    return cache[device].addr;
}

}  // namespace scmf

// The entry point (declared in include/scmf.h).
extern "C" scmf_status scmf_update_omega_noalloc(const uint32_t* d_counts, float* d_omega, int32_t n_types,
                                                 int64_t n_cells, double field_scaling, const double* xn,
                                                 int32_t reference_nbeads, int32_t hamiltonian, double* d_energy,
                                                 void* stream) {
    using namespace scmf;
    if (!d_counts || !d_omega || !xn || !d_energy) return fail(SCMF_E_INVALID, "NULL argument");
    if (n_types < 1 || n_types > kMaxTypes) return fail(SCMF_E_INVALID, "n_types %d not in [1,%d]", n_types, kMaxTypes);
    if (n_cells < 1) return fail(SCMF_E_INVALID, "n_cells must be positive");
    if (n_cells > (int64_t)kNoAllocMaxTiles * kNoAllocTileCells)
        return fail(SCMF_E_INVALID,
                    "n_cells %lld exceeds the %lld cells the fixed scratch of the allocation-free field update covers",
                    (long long)n_cells, (long long)kNoAllocMaxTiles * kNoAllocTileCells);
    if (reference_nbeads < 1) return fail(SCMF_E_INVALID, "reference_nbeads must be >= 1");
    if (hamiltonian != SCMF_HAM_SCMF0 && hamiltonian != SCMF_HAM_LITERAL) return fail(SCMF_E_INVALID, "unknown hamiltonian");
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return fail(SCMF_E_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    double* scratch = noalloc_scratch(device, &e);
    if (!scratch) return fail(SCMF_E_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    FieldParams p{};
    p.n_cells = n_cells;
    p.scale = (float)field_scaling;
    p.n_types = n_types;
    p.lit = hamiltonian == SCMF_HAM_LITERAL;
    field_coefficients(n_types, xn, reference_nbeads, hamiltonian, p.cf);
    const int tiles = (int)((n_cells + kNoAllocTileCells - 1) / kNoAllocTileCells);
    cudaStream_t st = (cudaStream_t)stream;
    k_field_noalloc<<<tiles, 256, 0, st>>>(d_counts, d_omega, p, scratch);
    k_sum_partials<<<1, 256, 0, st>>>(scratch, tiles, d_energy);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(SCMF_E_CUDA, "launch: %s", cudaGetErrorString(e));
    return SCMF_OK;
}
