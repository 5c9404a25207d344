// sm_100a kernels of the SCMF engine.
//
//   k_init_coords   random-walk chains (device_function.cu:140-207)
//   k_sweep<mode>   one MC sweep over tiles of whole chains, staged in shared
//                   memory: odd/even (graph-colour) half-sweeps of smart-MC
//                   trials (device_function.cu:444-454, 509-799), then the
//                   per-type cell counts of the final positions
//                   (device_function.cu:471-508) and the bond energy
//   k_field<fused>  counts -> omega (SCMF0, device_function.cu:373-412) with the
//                   field-energy reduction; in the fused step it also clears the
//                   other counts buffer and closes the sweep (step, statistics)
//
// Built with --fmad=false -prec-div=true -prec-sqrt=true: positions and counts
// are bit-identical to the CPU oracle, whatever the tiling or launch shape.
#include <cuda_runtime.h>
#include <stdint.h>

#include "scmf_internal.h"
#include "scmf_math.cuh"

namespace scmf {

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
    uint4 w = philox4x32_10(make_uint4((uint32_t)g, 0u, kInitStep, 0u), k0, k1);
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
            normals3(philox4x32_10(make_uint4((uint32_t)g, (uint32_t)j, kInitStep, 1u), k0, k1), n0, n1, n2);
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
    int nx, ny, nz;
};

__device__ __forceinline__ int cell_of(const MoveConsts& c, float x, float y, float z) {
    const int ix = fold(x, c.inv_dx, c.nx);
    const int iy = fold(y, c.inv_dy, c.ny);
    const int iz = fold(z, c.inv_dz, c.nz);
    return ix + c.nx * (iy + c.ny * iz);
}

// One smart-MC trial (device_function.cu:637-717, 562-588, 444-454) of a bead
// at (x,y,z) with deg bonded neighbours q[0..deg) in ascending bead order.
// Same expression order as the oracle's move_bead().  On return (px,py,pz) is
// the bead's final position; eb gains k |r - q_d|^2 of the final position for
// every neighbour d flagged in lower_mask (neighbours of a lower colour, which
// have already made their final move this sweep).
template <int MAXDEG>
__device__ __forceinline__ bool trial(const MoveConsts& c, float x, float y, float z, const float* qx,
                                      const float* qy, const float* qz, int deg, unsigned lower_mask, uint4 w,
                                      const float* __restrict__ w_t, float& px, float& py, float& pz, float& eb) {
    const float k = c.k, k2 = c.k2, A = c.A, R = c.R;
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
#pragma unroll
    for (int d = 0; d < MAXDEG; ++d) {
        if (d < deg) {
            fx = fx + (qx[d] - x) * k2;
            fy = fy + (qy[d] - y) * k2;
            fz = fz + (qz[d] - z) * k2;
        }
    }
    float n0, n1, n2;
    normals3(w, n0, n1, n2);
    const float dx = A * fx + R * n0;
    const float dy = A * fy + R * n1;
    const float dz = A * fz + R * n2;
    px = x + dx;
    py = y + dy;
    pz = z + dz;
    float nfx = 0.0f, nfy = 0.0f, nfz = 0.0f;
    float deb = 0.0f;
    float o2s[MAXDEG], e2s[MAXDEG];
#pragma unroll
    for (int d = 0; d < MAXDEG; ++d) {
        if (d < deg) {
            nfx = nfx + (qx[d] - px) * k2;
            nfy = nfy + (qy[d] - py) * k2;
            nfz = nfz + (qz[d] - pz) * k2;
            const float ox = x - qx[d], oy = y - qy[d], oz = z - qz[d];
            const float ex = ox + dx, ey = oy + dy, ez = oz + dz;
            const float o2 = ox * ox + oy * oy + oz * oz;
            const float e2 = ex * ex + ey * ey + ez * ez;
            o2s[d] = o2;
            e2s[d] = e2;
            deb = deb + k * (e2 - o2);
        }
    }
    const float smc = 0.5f * ((nfx + fx) * dx + (nfy + fy) * dy + (nfz + fz) * dz) +
                      0.25f * A * (nfx * nfx + nfy * nfy + nfz * nfz - fx * fx - fy * fy - fz * fz);
    const float w_old = __ldg(w_t + cell_of(c, x, y, z));
    const float w_new = __ldg(w_t + cell_of(c, px, py, pz));
    float dE = (w_new - w_old) + deb;
    dE = dE + smc;
    // log(u) >= -24 ln2 > -17 for every u the generator yields: dE >= 17 rejects
    bool acc;
    if (dE < 0.0f)
        acc = true;
    else if (dE < 17.0f)
        acc = log_f(u01(accept_word(w))) < -dE;
    else
        acc = false;
    if (!acc) {
        px = x;
        py = y;
        pz = z;
    }
#pragma unroll
    for (int d = 0; d < MAXDEG; ++d)
        if (d < deg && (lower_mask >> d) & 1u) eb += k * (acc ? e2s[d] : o2s[d]);
    return acc;
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
//   MODE kMoveOnly / kMoveGrid / kGridOnly: moves, moves + counts of the final
//   positions into counts[cur^1], counts of the current positions into counts[cur].
//   LINEAR: every architecture of the launch is a linear chain (bonds i-i+1,
//   even beads colour 0, odd beads colour 1); neighbours are computed, not looked up.
template <int MODE, bool LINEAR>
__global__ void __launch_bounds__(256, 4) k_sweep(const MoveTile* __restrict__ tiles, int n_tiles,
                                                   int max_tile_beads, int max_length) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* sx = reinterpret_cast<float*>(smem_raw);
    float* sy = sx + max_tile_beads;
    float* sz = sy + max_tile_beads;
    size_t off = ((size_t)max_tile_beads * 3 * sizeof(float) + 15) & ~(size_t)15;
    BeadInfo* sinfo = reinterpret_cast<BeadInfo*>(smem_raw + off);
    off = (off + (size_t)max_length * sizeof(BeadInfo) + 15) & ~(size_t)15;
    uint16_t* scol = reinterpret_cast<uint16_t*>(smem_raw + off);
    uint8_t* stype = reinterpret_cast<uint8_t*>(sinfo);  // LINEAR: types only
    __shared__ float s_eb[32];
    __shared__ unsigned s_acc[32];

    const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5;
    for (int ti = blockIdx.x; ti < n_tiles; ti += gridDim.x) {
        const MoveTile t = tiles[ti];
        SysDev* S = t.sys;
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
        c.nx = S->nx; c.ny = S->ny; c.nz = S->nz;
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
            unsigned nacc = 0;
            float eb = 0.0f;
            for (int col = 0; col < Ap->n_colors; ++col) {
                const int ncol = Ap->color_off[col + 1] - Ap->color_off[col];
                const uint32_t mg = Ap->color_magic[col];
                const int items = t.n_chains * ncol;
                for (int j = tid; j < items; j += T) {
                    const int cl = (int)div_magic((uint32_t)j, mg, ncol);
                    const int base = cl * L;
                    float qx[LINEAR ? 2 : kMaxDeg], qy[LINEAR ? 2 : kMaxDeg], qz[LINEAR ? 2 : kMaxDeg];
                    int b, deg, type;
                    unsigned lower = 0;
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
                        lower = col == 1 ? 3u : 0u;
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
                                if (sinfo[bi.nbr[d]].color < col) lower |= 1u << d;
                            }
                        }
                    }
                    const uint4 w = philox4x32_10(make_uint4(__ldg(cid + cl), (uint32_t)b, step, 0u), k0, k1);
                    float px, py, pz;
                    const bool acc = trial<LINEAR ? 2 : kMaxDeg>(c, sx[base + b], sy[base + b], sz[base + b], qx, qy,
                                                                 qz, deg, lower, w, omega + (int64_t)type * NC, px,
                                                                 py, pz, eb);
                    if (acc) {
                        sx[base + b] = px;
                        sy[base + b] = py;
                        sz[base + b] = pz;
                    }
                    nacc += acc ? 1u : 0u;
                }
                __syncthreads();
            }
            eb = warp_sum(eb);
            nacc = warp_sum(nacc);
            if (lane == 0) {
                s_eb[warp] = eb;
                s_acc[warp] = nacc;
            }
            __syncthreads();
            if (tid == 0) {
                double e = 0.0;
                unsigned long long a = 0;
                for (int w = 0; w < (T + 31) / 32; ++w) {
                    e += (double)s_eb[w];
                    a += s_acc[w];
                }
                const int slot = ti % kSlots;
                atomicAdd(&S->slot_eb[slot], e);
                atomicAdd(&S->slot_acc[slot], a);
            }
        }

        if (MODE != kMoveOnly) {
            const uint32_t buf = (MODE == kMoveGrid) ? (S->cur ^ 1u) : S->cur;
            uint32_t* cnt = S->counts[buf];
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

// ------------------------------------------------------------------ field
__device__ __forceinline__ double read_clear(double* p) {
    return __longlong_as_double((long long)atomicExch(reinterpret_cast<unsigned long long*>(p), 0ull));
}

// Field of one cell for NT monomer types (NT = 0: runtime count, up to kMaxTypes).
// Expression order matches the oracle's field_update().
template <int NT, bool FUSED>
__device__ __forceinline__ double field_cell(int n, int64_t cell, int64_t NC, float scale, bool lit, bool upd,
                                             bool c16, const uint32_t* src32, uint32_t* clr32, float* W,
                                             const float* cf) {
    constexpr int M = NT > 0 ? NT : kMaxTypes;
    const int nt = NT > 0 ? NT : n;
    const uint16_t* src16 = reinterpret_cast<const uint16_t*>(src32);
    uint16_t* clr16 = reinterpret_cast<uint16_t*>(clr32);
    float phi[M];
    uint32_t cnt[M];
    float tot = 0.0f;
#pragma unroll
    for (int u = 0; u < M; ++u) {
        if (u < nt) {
            cnt[u] = c16 ? (uint32_t)src16[u * NC + cell] : src32[u * NC + cell];
            phi[u] = (float)cnt[u] * scale;
            tot = tot + phi[u];
        }
    }
    double ef = 0.0;
#pragma unroll
    for (int tt = 0; tt < M; ++tt) {
        if (tt < nt) {
            float w;
            if (upd) {
                w = (tot - 1.0f) * cf[tt + nt * tt];
#pragma unroll
                for (int u = 0; u < M; ++u) {
                    if (u < nt && u != tt) {
                        if (!lit)
                            w = w + cf[tt + nt * u] * (phi[tt] - phi[u]);
                        else
                            w = w + cf[tt + nt * u] * phi[u];
                    }
                }
                W[tt * NC + cell] = w;
            } else {
                w = W[tt * NC + cell];
            }
            ef += (double)w * (double)cnt[tt];
            if (FUSED) {
                if (c16)
                    clr16[tt * NC + cell] = 0;
                else
                    clr32[tt * NC + cell] = 0u;
            }
        }
    }
    return ef;
}

template <bool FUSED, int NT>
__global__ void __launch_bounds__(256) k_field(const FieldTile* __restrict__ tiles, int n_tiles, int force_update) {
    __shared__ double s_ef[32];
    __shared__ float cf[kMaxTypes * kMaxTypes];
    __shared__ int s_last;
    const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5;
    for (int ti = blockIdx.x; ti < n_tiles; ti += gridDim.x) {
        const FieldTile t = tiles[ti];
        SysDev* S = t.sys;
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
        const uint32_t* src32 = S->counts[FUSED ? (cur ^ 1u) : cur];
        uint32_t* clr32 = FUSED ? S->counts[cur] : nullptr;
        float* W = S->omega;
        double ef = 0.0;
        const int64_t end = t.cell0 + t.n_cells;
        for (int64_t cell = t.cell0 + tid; cell < end; cell += T)
            ef += field_cell<NT, FUSED>(n, cell, NC, scale, lit, upd, c16, src32, clr32, W, cf);
        ef = warp_sum(ef);
        if (lane == 0) s_ef[warp] = ef;
        __syncthreads();
        if (tid == 0) {
            double e = 0.0;
            for (int w = 0; w < (T + 31) / 32; ++w) e += s_ef[w];
            atomicAdd(&S->slot_ef[ti % kSlots], e);
            __threadfence();
            const unsigned prev = atomicAdd(&S->field_done, 1u);
            s_last = (prev == (unsigned)t.n_tiles_sys - 1u);
        }
        __syncthreads();
        if (s_last && tid == 0) {
            __threadfence();
            double e_f = 0.0;
            for (int s = 0; s < kSlots; ++s) e_f += read_clear(&S->slot_ef[s]);
            S->e_field = e_f;
            if (FUSED) {
                unsigned long long a = 0;
                double e_b = 0.0;
                for (int s = 0; s < kSlots; ++s) {
                    a += atomicExch(&S->slot_acc[s], 0ull);
                    e_b += read_clear(&S->slot_eb[s]);
                }
                S->last_accepts = a;
                S->total_accepts += a;
                S->total_moves += (unsigned long long)S->n_beads;
                S->e_bond = e_b;
                S->cur = cur ^ 1u;
                S->step = sweep;
            }
            S->field_done = 0u;
            __threadfence();
        }
        __syncthreads();
    }
}

__global__ void k_finalize_move(SysDev* S) {
    if (threadIdx.x != 0) return;
    unsigned long long a = 0;
    double e_b = 0.0;
    for (int s = 0; s < kSlots; ++s) {
        a += atomicExch(&S->slot_acc[s], 0ull);
        e_b += read_clear(&S->slot_eb[s]);
    }
    S->last_accepts = a;
    S->total_accepts += a;
    S->total_moves += (unsigned long long)S->n_beads;
    S->e_bond = e_b;
    S->step = S->step + 1u;
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
    return A.bead_base + (int64_t)(gc - (uint32_t)A.chain_base) * A.length + b;
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
__global__ void k_debug_math(uint32_t k0, uint32_t k1, int n, uint32_t* words, float* logs, float* sines,
                             float* cosines, float* normals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint4 w = philox4x32_10(make_uint4((uint32_t)i, 0u, 0u, 0u), k0, k1);
    words[4 * i] = w.x;
    words[4 * i + 1] = w.y;
    words[4 * i + 2] = w.z;
    words[4 * i + 3] = w.w;
    logs[i] = log_f(u01(w.x));
    float s, c;
    sincos_turn(w.y, s, c);
    sines[i] = s;
    cosines[i] = c;
    float n0, n1, n2;
    normals3(w, n0, n1, n2);
    normals[3 * i] = n0;
    normals[3 * i + 1] = n1;
    normals[3 * i + 2] = n2;
}

// -------------------------------------------------------------- launchers
int launch_debug_math(uint32_t k0, uint32_t k1, int n, uint32_t* words, float* logs, float* sines, float* cosines,
                      float* normals, void* stream) {
    k_debug_math<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(k0, k1, n, words, logs, sines, cosines, normals);
    return (int)cudaGetLastError();
}

static int grid_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b > 148 * 32) b = 148 * 32;
    return (int)(b < 1 ? 1 : b);
}

int launch_init_coords(SysDev* d_sys, const ArchDev* d_arch, int n_arch, int n_chains, void* stream) {
    if (n_chains <= 0) return 0;
    const int th = 128;
    k_init_coords<<<(n_chains + th - 1) / th, th, 0, (cudaStream_t)stream>>>(d_sys, d_arch, n_arch, n_chains);
    return (int)cudaGetLastError();
}

// Opt the sweep kernels in to the largest dynamic shared memory once, outside
// any stream capture (called when a system is created).
template <int MODE, bool LINEAR>
static cudaError_t allow_smem(int bytes) {
    return cudaFuncSetAttribute(k_sweep<MODE, LINEAR>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

int configure_kernels() {
    static int done = 0;
    if (done) return 0;
    const int bytes = (int)sweep_smem_bytes(kMaxTileBeads, kMaxLength);
    cudaError_t e = allow_smem<kMoveOnly, false>(bytes);
    if (e == cudaSuccess) e = allow_smem<kMoveGrid, false>(bytes);
    if (e == cudaSuccess) e = allow_smem<kGridOnly, false>(bytes);
    if (e == cudaSuccess) e = allow_smem<kMoveOnly, true>(bytes);
    if (e == cudaSuccess) e = allow_smem<kMoveGrid, true>(bytes);
    if (e == cudaSuccess) e = allow_smem<kGridOnly, true>(bytes);
    if (e == cudaSuccess) done = 1;
    return (int)e;
}

template <int MODE>
static int launch_sweep_t(const MoveTile* tiles, int n_tiles, int mtb, int ml, LaunchShape sh, cudaStream_t st) {
    const size_t smem = sweep_smem_bytes(mtb, ml);
    if (mtb > kMaxTileBeads || ml > kMaxLength || sh.threads > 256) return (int)cudaErrorInvalidValue;
    const int blocks = sh.blocks > 0 ? sh.blocks : n_tiles;
    if (sh.linear)
        k_sweep<MODE, true><<<blocks, sh.threads, smem, st>>>(tiles, n_tiles, mtb, ml);
    else
        k_sweep<MODE, false><<<blocks, sh.threads, smem, st>>>(tiles, n_tiles, mtb, ml);
    return (int)cudaGetLastError();
}

int launch_sweep(int mode, const MoveTile* tiles, int n_tiles, int mtb, int ml, LaunchShape sh, void* stream) {
    if (n_tiles <= 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    if (mode == kMoveOnly) return launch_sweep_t<kMoveOnly>(tiles, n_tiles, mtb, ml, sh, st);
    if (mode == kMoveGrid) return launch_sweep_t<kMoveGrid>(tiles, n_tiles, mtb, ml, sh, st);
    return launch_sweep_t<kGridOnly>(tiles, n_tiles, mtb, ml, sh, st);
}

template <bool FUSED>
static void launch_field_t(int nt, const FieldTile* tiles, int n_tiles, int force_update, int blocks, int threads,
                           cudaStream_t st) {
    if (nt == 2)
        k_field<FUSED, 2><<<blocks, threads, 0, st>>>(tiles, n_tiles, force_update);
    else if (nt == 3)
        k_field<FUSED, 3><<<blocks, threads, 0, st>>>(tiles, n_tiles, force_update);
    else if (nt == 1)
        k_field<FUSED, 1><<<blocks, threads, 0, st>>>(tiles, n_tiles, force_update);
    else
        k_field<FUSED, 0><<<blocks, threads, 0, st>>>(tiles, n_tiles, force_update);
}

int launch_field(bool fused, int force_update, const FieldTile* tiles, int n_tiles, LaunchShape sh, void* stream) {
    if (n_tiles <= 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    const int blocks = sh.blocks > 0 ? sh.blocks : n_tiles;
    const int threads = sh.threads > 256 ? 256 : sh.threads;
    if (fused)
        launch_field_t<true>(sh.n_types, tiles, n_tiles, force_update, blocks, threads, st);
    else
        launch_field_t<false>(sh.n_types, tiles, n_tiles, force_update, blocks, threads, st);
    return (int)cudaGetLastError();
}

int launch_finalize_move(SysDev* sys, void* stream) {
    k_finalize_move<<<1, 32, 0, (cudaStream_t)stream>>>(sys);
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

}  // namespace scmf
