// Fused B200 pipeline of one coupled step (solvers/coupled_step.py:73-464)
// plus the column and streaming kernels shared with the
// operator API.
//
// Per step (no droplet):  surface height -> arc weight sum -> inject + cap
// -> thermal (advect/diffuse, losses, phase, T_max, cooling rate)
// -> VOF advect+reinit -> column pass (contact angle, flags, sync, time above,
//    active-cell list) -> forces + collide + Mach clamp over the active list
// -> stream -> [remelt / solidify].
//
// Cell kernels use 32x8 (k, j) tiles with one grid z-slice per i, so the cell
// coordinates come from the launch geometry without integer division, and
// consecutive lanes touch consecutive k (coalesced, k is the fastest axis).
#include <cmath>
#include <mutex>

#include "../../include/waam_b200.h"
#include "waam_common.cuh"
#include "waam_internal.cuh"

using namespace waam;

namespace waam {

#define STREAM(s) reinterpret_cast<cudaStream_t>(s)
constexpr int kMainEvents = 7;
constexpr int kMaxDevices = 64;
constexpr int kTileRedBlocks = 592;   // <= kWsMaxPartials; a fixed grid keeps the sum order fixed
constexpr int kListThreads = 128;
constexpr int kArcTableMax = 1024;    // nz up to which the arc depth weights come from a table
constexpr int kArcAxisMax = 3072;     // nx + ny + nz up to which the arc shape uses axis tables
// the collision's persistent grid: 4 blocks of 128 threads (96 registers) per
// SM, 75,776 threads, one pass over the ~66 k active cells of the standard
// workload (measured with the population copy: 0.2132 against 0.2154 ms per
// droplet period for 2 per SM, 0.2150 for 3; no change on the 512x256x160
// and 64x32x32 workloads; without the copy 2 per SM had been best)
constexpr int kListBlocks = 148 * 4;


// ---------------------------------------------------------------------------
// Contact-angle ghost-phi BC (kernels.py:933-991), one warp per (i, j)
// column, lanes over k.  The reference updates phi in place; its serial
// order makes cell k see the final value of cell k-1 (rule "gas above pool")
// and the ghost write of cell k-1 (rule "fluid on substrate"), while other
// columns are read before the kernel (snapshot `snap`).  The ghost write of
// cell k-1 depends only on snapshot data, so it is computed in parallel; the
// k-1 -> k dependence through the final value is resolved by a warp-wide
// fixed-point iteration, whose fixed point is the unique serial result.
// ---------------------------------------------------------------------------
struct ContactConst {
    float cos_t, sin_t, film, spread;
};

// cos/sin of the contact angle are evaluated once on the host in double and
// rounded to float (the same values the oracle uses).
__device__ __forceinline__ ContactConst contact_const(float cos_t, float sin_t) {
    ContactConst cc;
    cc.cos_t = cos_t;
    cc.sin_t = sin_t;
    cc.film = 0.5f * (1.0f - cc.cos_t);
    cc.spread = cc.film * (0.85f + 0.15f * cc.sin_t);
    return cc;
}

// Value of one non-solid cell after all rules, given the final value of the
// cell below (prev, valid only if has_prev) -- kernels.py:957-990.
__device__ __forceinline__ float contact_rules(const ContactConst& cc, float start, int flag,
                                               bool below_solid, bool any_nb, bool has_prev,
                                               float prev) {
    float v = start;
    if (below_solid && flag == GAS) {
        if (v < cc.film) v = cc.film;
    }
    if (has_prev && prev > 0.55f && flag == GAS) {
        float t = prev - cc.sin_t;
        t = fmax_(cc.film, fmin_(t, 0.95f));
        if (v < t) v = t;
    }
    if (v < 0.45f && any_nb) {
        if (v < cc.spread) v = cc.spread;
    }
    if (below_solid && v > 0.2f) {
        if (v < 0.65f) v = 0.65f;
    }
    return v;
}

// Runs the column pass for one warp; `emit(k, c, value, flag_old, valid)` is
// called by every lane of every chunk (convergent), value = final phi (snap
// for solid cells).
// skip(k0): the chunk at k0 is a quiet all-GAS chunk (warp-uniform); it is
// left alone and the next chunk starts from a GAS cell below with phi < 0.55
// and no ghost value, which is what its cells would see.
template <class Emit, class Skip>
__device__ __forceinline__ void contact_column(const Dims d, const float* __restrict__ snap,
                                               const int32_t* __restrict__ flags, int i, int j,
                                               bool wetting, const ContactConst& cc, Emit emit,
                                               Skip skip) {
    const int lane = threadIdx.x & 31;
    int carry_flag = SOLID;      // old flag of the cell below the chunk
    float carry_final = 0.0f;    // final phi of the cell below the chunk
    float carry_ghost = -1.0f;   // ghost value written into the chunk's first cell (<0: none)
    const int sx = d.ny * d.nz;
    for (int k0 = 0; k0 < d.nz; k0 += 32) {
        if (skip(k0)) {
            carry_flag = GAS;
            carry_final = 0.0f;
            carry_ghost = -1.0f;
            continue;
        }
        int k = k0 + lane;
        bool valid = k < d.nz;
        int c = d.idx(i, j, valid ? k : d.nz - 1);
        float s = valid ? snap[c] : 0.0f;
        int flag = valid ? flags[c] : SOLID;
        if (!wetting) {
            emit(k, c, s, flag, valid);
            continue;
        }
        int flag_up = (valid && k + 1 < d.nz) ? flags[c + 1] : SOLID;
        int flag_dn = __shfl_up_sync(0xffffffffu, flag, 1);
        if (lane == 0) flag_dn = carry_flag;
        bool below_solid = k > 0 && flag_dn == SOLID;
        // neighbour columns, pre-kernel values
        bool any_nb = false;
        if (valid && flag != SOLID) {
            if (j - 1 >= 0 && snap[c - d.nz] > 0.55f) any_nb = true;
            if (j + 1 < d.ny && snap[c + d.nz] > 0.55f) any_nb = true;
            if (i - 1 >= 0 && snap[c - sx] > 0.55f) any_nb = true;
            if (i + 1 < d.nx && snap[c + sx] > 0.55f) any_nb = true;
        }
        // ghost value this cell writes into k+1 ("fluid on substrate")
        float ghost_out = -1.0f;
        if (valid && flag != SOLID && below_solid) {
            float r1 = s;
            if (flag == GAS && r1 < cc.film) r1 = cc.film;
            if (r1 > 0.55f && k + 1 < d.nz && flag_up == GAS) {
                float g = r1 - cc.sin_t;
                ghost_out = fmax_(cc.film, fmin_(g, 0.98f));
            }
        }
        float ghost_in = __shfl_up_sync(0xffffffffu, ghost_out, 1);
        if (lane == 0) ghost_in = carry_ghost;
        float start = s;
        if (ghost_in >= 0.0f && start < ghost_in) start = ghost_in;
        bool active = valid && flag != SOLID;
        // fixed point over the chunk
        float cur = active ? contact_rules(cc, start, flag, below_solid, any_nb, false, 0.0f) : s;
        for (int it = 0; it < 34; ++it) {
            float prev = __shfl_up_sync(0xffffffffu, cur, 1);
            bool has_prev = k > 0;
            if (lane == 0) prev = carry_final;
            float nv = active ? contact_rules(cc, start, flag, below_solid, any_nb, has_prev, prev)
                              : (valid ? start : s);
            bool changed = nv != cur;
            cur = nv;
            if (!__any_sync(0xffffffffu, changed)) break;
        }
        emit(k, c, cur, flag, valid);
        carry_flag = __shfl_sync(0xffffffffu, flag, 31);
        carry_final = __shfl_sync(0xffffffffu, cur, 31);
        carry_ghost = __shfl_sync(0xffffffffu, ghost_out, 31);
    }
}

__global__ void k_contact_op(Dims d, const float* __restrict__ snap, float* __restrict__ phi,
                             const int32_t* __restrict__ flags, float cos_t, float sin_t) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (warp >= d.nx * d.ny) return;
    int i = warp / d.ny, j = warp % d.ny;
    ContactConst cc = contact_const(cos_t, sin_t);
    contact_column(d, snap, flags, i, j, true, cc, [&](int k, int c, float v, int flag, bool valid) {
        if (valid && flag != SOLID) phi[c] = v;
    }, [](int) { return false; });
}

int launch_contact_columns(Dims d, const float* snap, float* phi, const int32_t* flags,
                           float theta, void* stream) {
    int64_t threads = (int64_t)d.nx * d.ny * 32;
    int blocks = (int)((threads + kThreads - 1) / kThreads);
    k_contact_op<<<blocks, kThreads, 0, STREAM(stream)>>>(d, snap, phi, flags,
                                                         (float)cos((double)theta),
                                                         (float)sin((double)theta));
    return check_launch("k_contact_op");
}

// ---------------------------------------------------------------------------
// Pull streaming (kernels.py:2971-3010): x periodic, y/z clamped, bounce-back
// from SOLID sources for non-gas cells.  Every thread first issues its 19
// source loads back to back (independent addresses, so all are in flight at
// once), then, for the few non-gas cells, replaces the populations whose
// source is SOLID by the cell's own opposite population, then stores.
// The per-population base pointers come precomputed in the launch
// parameters -- for interior cells (no wrap or clamp on any axis) already
// shifted by the pull offset -- so an address costs one multiply-add.
// ---------------------------------------------------------------------------
template <typename T>
struct StreamPtrs {
    const T* src[19];    // population q shifted by the interior pull offset
    const T* base[19];   // population q of the input
    T* dst[19];          // population q of the output
};

template <typename T>
static StreamPtrs<T> stream_ptrs(const Dims& d, const void* f_src, void* f_dst) {
    StreamPtrs<T> P;
    const int64_t n = d.n(), sx = (int64_t)d.ny * d.nz, sy = d.nz;
    const uintptr_t a = reinterpret_cast<uintptr_t>(f_src), b = reinterpret_cast<uintptr_t>(f_dst);
    for (int q = 0; q < 19; ++q) {
        const int64_t off = ex(q) * sx + ey(q) * sy + ez(q);   // < n for every q >= 1, 0 for q = 0
        P.src[q] = reinterpret_cast<const T*>(a + (uintptr_t)((q * n - off) * (int64_t)sizeof(T)));
        P.base[q] = reinterpret_cast<const T*>(a + (uintptr_t)(q * n * (int64_t)sizeof(T)));
        P.dst[q] = reinterpret_cast<T*>(b + (uintptr_t)(q * n * (int64_t)sizeof(T)));
    }
    return P;
}

__device__ __forceinline__ int stream_source(const Dims& d, bool interior, int i, int j, int k,
                                             int c, int q) {
    if (interior) return c - (ex(q) * d.ny * d.nz + ey(q) * d.nz + ez(q));
    int ni = i - ex(q);
    ni = ni < 0 ? ni + d.nx : (ni >= d.nx ? ni - d.nx : ni);
    const int nj = imax(0, imin(j - ey(q), d.ny - 1));
    const int nk = imax(0, imin(k - ez(q), d.nz - 1));
    return (ni * d.ny + nj) * d.nz + nk;
}

// T is the stored element: streaming moves stored values unchanged, whatever
// the population storage.
template <typename T>
__device__ __forceinline__ void stream_cell(const Dims& d, const StreamPtrs<T>& P,
                                            const int32_t* __restrict__ flags, int i, int j,
                                            int k, int c) {
    const int flag = flags[c];
    if (flag == SOLID) return;
    const bool interior = i > 0 && i < d.nx - 1 && j > 0 && j < d.ny - 1 && k > 0 && k < d.nz - 1;
    T v[19];
    if (interior) {
#pragma unroll
        for (int q = 0; q < 19; ++q) v[q] = P.src[q][c];
    } else {
#pragma unroll
        for (int q = 0; q < 19; ++q) v[q] = P.base[q][stream_source(d, false, i, j, k, c, q)];
    }
    if (flag != GAS) {
#pragma unroll
        for (int q = 1; q < 19; ++q)
            if (flags[stream_source(d, interior, i, j, k, c, q)] == SOLID) v[q] = P.base[opp(q)][c];
    }
#pragma unroll
    for (int q = 0; q < 19; ++q) P.dst[q][c] = v[q];
}

__device__ __forceinline__ bool is_active(int flag) { return flag == FLUID || flag == IFACE; }

// next_flags (null: none): the flags of the step after the streamed one.
// Cells active there (FLUID / IFACE) are left alone: that step's collision
// writes all 19 populations of each of them into the buffer the stream
// writes, and nothing reads that buffer between the two (the lagged stream
// of WaamStepParams.hold_stream).
template <typename T>
__global__ void __launch_bounds__(256) k_stream(Dims d, const __grid_constant__ StreamPtrs<T> P,
                                                const int32_t* __restrict__ flags,
                                                const int32_t* __restrict__ next_flags) {
    int i, j, k, c;
    if (!tile_cell(d, i, j, k, c)) return;
    if (next_flags != nullptr && is_active(next_flags[c])) return;
    stream_cell(d, P, flags, i, j, k, c);
}


template <typename T>
static void launch_stream_t(const Dims& d, const void* f_src, void* f_dst, const int32_t* flags,
                            const int32_t* next_flags, cudaStream_t s) {
    k_stream<T><<<tile_grid(d), tile_block(), 0, s>>>(d, stream_ptrs<T>(d, f_src, f_dst), flags,
                                                       next_flags);
}

int launch_stream(Dims d, const float* f_src, float* f_dst, const int32_t* flags, void* stream) {
    launch_stream_t<float>(d, f_src, f_dst, flags, nullptr, STREAM(stream));
    return check_launch("k_stream");
}

// The fused step's stream: 4-byte or 2-byte stored populations.
static int launch_stream_stored(Dims d, const void* f_src, void* f_dst, const int32_t* flags,
                                int storage, cudaStream_t s,
                                const int32_t* next_flags = nullptr) {
    if (storage == kStoreF32)
        launch_stream_t<float>(d, f_src, f_dst, flags, next_flags, s);
    else
        launch_stream_t<uint16_t>(d, f_src, f_dst, flags, next_flags, s);
    return check_launch("k_stream");
}

// ---------------------------------------------------------------------------
// Fused step kernels
// ---------------------------------------------------------------------------

// Top metal cell of the torch column and the arc-k fallback of
// solvers/coupled_step.py:34-59, computed by one warp (every lane returns it).
__device__ __forceinline__ float surface_arc_k(const Dims& d, const float* phi,
                                               const int32_t* flags, const float* scalars,
                                               int nz_solid) {
    const int lane = threadIdx.x & 31;
    float arc_i = scalars[kScalarArcI], arc_j = scalars[kScalarArcJ];
    int i0 = imax(0, imin((int)arc_i, d.nx - 1));
    int j0 = imax(0, imin((int)arc_j, d.ny - 1));
    int best = -1;
    for (int k = lane; k < d.nz; k += 32) {
        int c = d.idx(i0, j0, k);
        if (flags[c] != GAS && phi[c] > 0.05f) best = k;
    }
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
    int ks = best >= 0 ? best : imax(1, nz_solid - 1);
    float kf = (float)ks;
    if (kf < 1.0f) kf = (float)imax(1, nz_solid - 1);
    return kf;
}

__global__ void k_surface_arc(Dims d, const float* phi, const int32_t* flags, float* scalars,
                              int nz_solid) {
    const float kf = surface_arc_k(d, phi, flags, scalars, nz_solid);
    if (threadIdx.x == 0) scalars[kScalarArcK] = kf;
}

__device__ double tile_block_sum(double v) {
    __shared__ double sh[(kTileK * kTileJ) / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int t = threadIdx.y * kTileK + threadIdx.x;
    if ((t & 31) == 0) sh[t >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (t == 0)
        for (int w = 0; w < (kTileK * kTileJ) / 32; ++w) s += sh[w];
    __syncthreads();
    return s;
}

// Arc weight sum over 32x8 tiles (pass 1 of kernels.py:443-510 / 548-622),
// deterministic: fixed tile-to-block assignment, double partials, the last
// block sums them in order.  Writes the weight sum and the energy per weight.
// The depth weight of a cell that is not liquid depends on k alone: it comes
// from a per-block table of the nz values (kArcTableMax at most; larger nz
// computes it per cell).  The spatial factor of every weighted cell is left
// in `shape` for the injection pass, which then needs no exponential.
__global__ void __launch_bounds__(256) k_arc_norm_tiles(Dims d, const int32_t* __restrict__ flags,
                                                        const float* __restrict__ f_l,
                                                        const float* __restrict__ phi, int nz_solid,
                                                        ArcParams p, float* scalars,
                                                        float arc_k_offset, float Qe_dt, float dx3,
                                                        Workspace ws, float* __restrict__ shape) {
    // every block finds the arc k itself (one warp scans the torch column), so
    // the surface query needs no launch of its own; block 0 publishes it
    __shared__ float s_arc_k;
    __shared__ float s_wd[kArcTableMax];
    if (threadIdx.y == 0) {
        const float kf = surface_arc_k(d, phi, flags, scalars, nz_solid);
        if (threadIdx.x == 0) {
            s_arc_k = kf;
            if (blockIdx.x == 0) scalars[kScalarArcK] = kf;
        }
    }
    __syncthreads();
    p.arc_k = s_arc_k + arc_k_offset;
    p.arc_i = scalars[kScalarArcI];
    p.arc_j = scalars[kScalarArcJ];
    const bool table = d.nz <= kArcTableMax;
    if (table)
        for (int k = threadIdx.y * kTileK + threadIdx.x; k < d.nz; k += kTileK * kTileJ)
            s_wd[k] = arc_weight(k, p.arc_k, 0.0f, p.pen, p.enable);
    __syncthreads();
    const int kt = (d.nz + kTileK - 1) / kTileK, jt = (d.ny + kTileJ - 1) / kTileJ;
    const int tiles = kt * jt * d.nx;
    // four tiles per pass: their flags and liquid fractions are all requested
    // before any weight is computed (f_l of gas cells is read and ignored)
    constexpr int kU = 4;
    double part = 0.0;
    for (int t0 = blockIdx.x; t0 < tiles; t0 += kU * gridDim.x) {
        int fg[kU], ci[kU], cj[kU], ck[kU];
        float fl[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int t = t0 + u * gridDim.x;
            const int a = t % kt, r = t / kt;
            const int b = r % jt, i = r / jt;
            const int k = a * kTileK + threadIdx.x, j = b * kTileJ + threadIdx.y;
            const bool ok = t < tiles && k < d.nz && j < d.ny;
            const int c = ok ? (i * d.ny + j) * d.nz + k : 0;
            fg[u] = ok ? flags[c] : GAS;
            fl[u] = ok ? f_l[c] : 0.0f;
            ci[u] = i;
            cj[u] = j;
            ck[u] = k;
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            if (fg[u] == GAS) continue;
            // arc_cell_weight (waam_common.cuh) with the depth weight from the table
            const float wd = !table ? arc_weight(ck[u], p.arc_k, fl[u], p.pen, p.enable)
                                    : (fl[u] > 0.55f ? 1.0f : s_wd[ck[u]]);
            if (wd < 1e-6f) continue;
            const float sh = arc_cell_shape(p, ci[u], cj[u], ck[u]);
            shape[(ci[u] * d.ny + cj[u]) * d.nz + ck[u]] = sh;
            part += (double)(sh * wd);
        }
    }
    part = tile_block_sum(part);
    __shared__ bool last;
    int t0 = threadIdx.y * kTileK + threadIdx.x;
    if (t0 == 0) {
        ws.partials[blockIdx.x] = part;
        __threadfence();
        unsigned prev = atomicAdd(ws.counter, 1u);
        last = prev == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    // the last block sums the partials: fixed strided assignment + fixed tree
    __threadfence();
    double acc = 0.0;
    for (unsigned bb = t0; bb < gridDim.x; bb += kTileK * kTileJ)
        acc += ((volatile double*)ws.partials)[bb];
    double tot = tile_block_sum(acc);
    if (t0 == 0) {
        *ws.counter = 0u;
        float w_total = (float)tot;
        float epw = 0.0f;
        if (w_total > 1e-9f) epw = Qe_dt / (w_total * dx3);
        scalars[kScalarWsum] = w_total;
        scalars[kScalarEpw] = epw;
    }
}

// Quiet-tile classification (WaamFields.tile_bits).  A tile is quiet when its
// columns were all GAS in the last two column passes (chunk bits 0 and 1) and
// every cell within two lattice steps of it is GAS: the chunks of the
// 5 x (8 + 4) columns around it at the same k are all GAS (bit 0), the top
// two cells of the chunks below (bit 2) and the bottom two of the chunks
// above (bit 3) too -- x periodic, y and z out of range count as GAS.  Writes
// one work byte per tile and appends the work tiles to the list (count in
// list[0], zeroed before the launch).
// One warp per (i, j-tile) band of tiles: lane q < 60 owns the neighbour
// column (di, dj) = (q / 12 - 2, q % 12 - 2) and loads its three chunk bytes
// per k-tile; the warp votes.  A tile costs one round of independent loads.
// A quiet tile's arc weight slot (tile_part) is set to 0.  The grid's last
// block runs the surface query of the step (scalars[kScalarArcK]).
constexpr int kClassifyWarps = 8;
__global__ void __launch_bounds__(32 * kClassifyWarps)
    k_classify_tiles(Dims d, const uint8_t* __restrict__ chunk, uint8_t* __restrict__ work,
                     int32_t* __restrict__ list, int skip, double* __restrict__ tile_part,
                     const float* __restrict__ phi, const int32_t* __restrict__ flags,
                     float* __restrict__ scalars, int nz_solid) {
    if (blockIdx.x == gridDim.x - 1) {
        if (threadIdx.x < 32) {
            const float kf = surface_arc_k(d, phi, flags, scalars, nz_solid);
            if (threadIdx.x == 0) scalars[kScalarArcK] = kf;
        }
        return;
    }
    const int KT = tiles_k(d), JT = tiles_j(d);
    const int band = blockIdx.x * kClassifyWarps + (threadIdx.x >> 5);
    if (band >= d.nx * JT) return;   // warp-uniform
    const int lane = threadIdx.x & 31;
    const int i = band / JT, jt = band % JT;
    const int j0 = jt * kTileJ, j1 = imin(j0 + kTileJ, d.ny);
    // the lane's two neighbour columns (second: q = lane + 32 < 60); -1: none
    int64_t col[2];
    bool is_core[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int q = lane + 32 * h;
        const int di = q / (kTileJ + 4) - 2, dj = q % (kTileJ + 4) - 2;
        const int jj = j0 + dj;
        const bool ok = q < 5 * (kTileJ + 4) && jj >= 0 && jj < imin(d.ny, j1 + 2);
        const int ii = ((i + di) % d.nx + d.nx) % d.nx;
        col[h] = ok ? ((int64_t)ii * d.ny + jj) * KT : -1;
        is_core[h] = ok && di == 0 && dj >= 0 && jj < j1;
    }
    uint64_t wmask = 0;   // work k-tiles of the band (KT <= 64 with tiles on)
    for (int kt = 0; kt < KT; ++kt) {
        bool w = true;
        if (skip) {
            // every load is issued before any is tested
            unsigned b[2], c[2], lo[2], hi[2];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const bool ok = col[h] >= 0;
                c[h] = ok ? chunk[col[h] + kt] : 3u;
                lo[h] = ok && kt > 0 ? chunk[col[h] + kt - 1] : 0xffu;
                hi[h] = ok && kt + 1 < KT ? chunk[col[h] + kt + 1] : 0xffu;
            }
            bool quiet = true;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                b[h] = c[h] & (lo[h] >> 2) & (hi[h] >> 3);
                if (col[h] >= 0 && !(b[h] & 1u)) quiet = false;
                if (is_core[h] && (c[h] & 3u) != 3u) quiet = false;
            }
            w = !__all_sync(0xffffffffu, quiet);
        }
        if (lane == 0) {
            work[(int64_t)band * KT + kt] = w ? 1 : 0;
            if (!w) tile_part[(int64_t)band * KT + kt] = 0.0;
        }
        if (w) wmask |= 1ull << kt;
    }
    if (wmask == 0) return;
    int base = 0;
    if (lane == 0) base = atomicAdd(&list[0], __popcll(wmask));
    base = __shfl_sync(0xffffffffu, base, 0);
    // the band's work tiles in k-tile order, one lane per k-tile (a count
    // left non-zero by a step that stopped after this kernel cannot write
    // past the list)
    const int64_t cap = tile_total(d);
    for (int kt = lane; kt < KT; kt += 32) {
        const int64_t slot = (int64_t)base + __popcll(wmask & ((1ull << kt) - 1ull));
        if (((wmask >> kt) & 1ull) && slot < cap) list[1 + slot] = pack_tile(i, jt, kt);
    }
}

// The arc weight sum over the tiles of the work list (quiet tiles are all GAS
// and weigh nothing).  Each listed tile's sum goes to its own slot of
// tile_part (k_classify_tiles zeroes the quiet tiles' slots); the last block
// adds all slots in tile order, so the total does not depend on the list's
// order.  The surface query's arc k comes from k_classify_tiles.  A block
// takes kArcBatch listed tiles at a time: their loads are all issued first and
// their block sums share one barrier.  Otherwise as k_arc_norm_tiles.
constexpr int kArcBatch = 8;
__global__ void __launch_bounds__(256) k_arc_norm_list(Dims d, const int32_t* __restrict__ flags,
                                                       const float* __restrict__ f_l,
                                                       ArcParams p, float* scalars,
                                                       float arc_k_offset, float Qe_dt, float dx3,
                                                       Workspace ws, float* __restrict__ shape,
                                                       const int32_t* __restrict__ list,
                                                       double* __restrict__ tile_part, int tiles) {
    __shared__ float s_wd[kArcTableMax];
    p.arc_k = scalars[kScalarArcK] + arc_k_offset;
    p.arc_i = scalars[kScalarArcI];
    p.arc_j = scalars[kScalarArcJ];
    const bool table = d.nz <= kArcTableMax;
    if (table)
        for (int k = threadIdx.y * kTileK + threadIdx.x; k < d.nz; k += kTileK * kTileJ)
            s_wd[k] = arc_weight(k, p.arc_k, 0.0f, p.pen, p.enable);
    // The spatial factor's exponent is a sum of an i, a j and a k term
    // (Gaussian: di^2 + dj^2 + dk^2 / 4; Goldak: xt^2 / a^2 + dj^2 / b^2 +
    // dk^2 / c^2, waam_common.cuh arc_cell_shape); each term is tabulated once
    // per block with the per-cell expression and added in the same order, so
    // a cell costs one exponential and no division.
    __shared__ float s_axis[kArcAxisMax];
    const bool axes = d.nx + d.ny + d.nz <= kArcAxisMax;
    if (axes) {
        const float eps = 1e-6f;
        for (int t = threadIdx.y * kTileK + threadIdx.x; t < d.nx + d.ny + d.nz;
             t += kTileK * kTileJ) {
            float v;
            if (t < d.nx) {
                const float di = (float)t - p.arc_i;
                if (p.kind == 0) {
                    v = di * di;
                } else {
                    const float xt = di * p.sign;
                    const float a = xt >= 0.0f ? p.a_f : p.a_r;
                    v = (xt * xt) / (a * a + eps);
                }
            } else if (t < d.nx + d.ny) {
                const float dj = (float)(t - d.nx) - p.arc_j;
                v = p.kind == 0 ? dj * dj : (dj * dj) / (p.b * p.b + eps);
            } else {
                const float dk = (float)(t - d.nx - d.ny) - p.arc_k;
                v = p.kind == 0 ? dk * dk * 0.25f : (dk * dk) / (p.c * p.c + eps);
            }
            s_axis[t] = v;
        }
    }
    __syncthreads();
    auto shape_of = [&](int i, int j, int k) -> float {
        if (!axes) return arc_cell_shape(p, i, j, k);
        const float sum = (s_axis[i] + s_axis[d.nx + j]) + s_axis[d.nx + d.ny + k];
        if (p.kind == 0) return waam_expf(-sum * p.inv2s2);
        const float xt = ((float)i - p.arc_i) * p.sign;
        return (xt >= 0.0f ? p.ff : p.fr) * waam_expf(-3.0f * sum);
    };
    const int tid = threadIdx.y * kTileK + threadIdx.x;
    const int cnt = imin(list[0], tiles);
    constexpr int kU = kArcBatch, kWarps = (kTileK * kTileJ) / 32;
    __shared__ double s_part[kU][kWarps];
    for (int e0 = blockIdx.x * kU; e0 < cnt; e0 += kU * gridDim.x) {
        int ent[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) ent[u] = e0 + u < cnt ? list[1 + e0 + u] : -1;
        int fg[kU], ci[kU], cj[kU], ck[kU];
        float fl[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            int i = 0, j = 0, k = 0, c = 0;
            const bool ok = ent[u] >= 0 && list_tile_cell(d, ent[u], i, j, k, c);
            fg[u] = ok ? flags[c] : GAS;
            fl[u] = ok ? f_l[c] : 0.0f;
            ci[u] = i;
            cj[u] = j;
            ck[u] = k;
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            double v = 0.0;
            if (fg[u] != GAS) {
                const float wd = !table ? arc_weight(ck[u], p.arc_k, fl[u], p.pen, p.enable)
                                        : (fl[u] > 0.55f ? 1.0f : s_wd[ck[u]]);
                if (!(wd < 1e-6f)) {
                    const float sh = shape_of(ci[u], cj[u], ck[u]);
                    shape[(ci[u] * d.ny + cj[u]) * d.nz + ck[u]] = sh;
                    v = (double)(sh * wd);
                }
            }
            // the block sum of tile_block_sum: warp tree, then the warps in order
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
            if ((tid & 31) == 0) s_part[u][tid >> 5] = v;
        }
        __syncthreads();
        int mine = -1;   // thread u < kU writes tile u's slot
#pragma unroll
        for (int u = 0; u < kU; ++u)
            if (tid == u) mine = ent[u];
        if (mine >= 0) {
            double sum = 0.0;
            for (int w = 0; w < kWarps; ++w) sum += s_part[tid][w];
            tile_part[tile_index(d, mine)] = sum;
        }
        __syncthreads();
    }
    __shared__ bool last;
    if (tid == 0) {
        __threadfence();
        const unsigned prev = atomicAdd(ws.counter, 1u);
        last = prev == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the slots come from other blocks (fenced before their arrival count):
    // read them from L2 (__ldcg), independent loads that can all be in flight;
    // a quiet tile's slot is 0 and adds nothing
    double acc = 0.0;
    for (int t = tid; t < tiles; t += kTileK * kTileJ) acc += __ldcg(tile_part + t);
    const double tot = tile_block_sum(acc);
    if (tid == 0) {
        *ws.counter = 0u;
        const float w_total = (float)tot;
        float epw = 0.0f;
        if (w_total > 1e-9f) epw = Qe_dt / (w_total * dx3);
        scalars[kScalarWsum] = w_total;
        scalars[kScalarEpw] = epw;
    }
}

// Pass 2 for one cell: H += epw * weight (non-gas cells), then the enthalpy
// ceiling (solvers/coupled_step.py:107-108); wd_dry is the depth weight of
// the cell's k for a cell that is not liquid.
__device__ __forceinline__ void inject_cell(float* __restrict__ H, const int32_t* __restrict__ flags,
                                            const float* __restrict__ f_l, float epw, int cap,
                                            const PhaseParams& ph, const float* __restrict__ cp_f,
                                            const VarPhase& vp, const float* __restrict__ shape,
                                            float wd_dry, int c) {
    const int flag = flags[c];
    const float fl = f_l[c];           // requested with the flag (ignored for gas cells)
    float h = cap ? H[c] : 0.0f;
    if (flag == GAS) return;
    // arc_cell_heat (waam_common.cuh) with the spatial factor the weight-sum
    // pass left in `shape` and the depth weight from the table
    float dh = 0.0f;
    bool hit = false;
    if (epw > 0.0f) {
        const float wd = fl > 0.55f ? 1.0f : wd_dry;
        if (!(wd < 1e-6f)) {
            dh = epw * shape[c] * wd;
            hit = true;
        }
    }
    if (!hit && !cap) return;
    if (!cap) h = H[c];
    if (hit) h = h + dh;
    // table path: the ceiling with the rho*cp fields of the previous step
    // (kernels.py:1988-2010)
    if (cap) h = cp_f ? cap_h_var(vp, cp_f[c], h) : cap_h(ph, h);
    H[c] = h;
}

__global__ void __launch_bounds__(256) k_arc_inject_tiles(Dims d, float* __restrict__ H,
                                                          const int32_t* __restrict__ flags,
                                                          const float* __restrict__ f_l,
                                                          ArcParams p, const float* scalars,
                                                          float arc_k_offset, int cap,
                                                          PhaseParams ph,
                                                          const float* __restrict__ cp_f,
                                                          VarPhase vp,
                                                          const float* __restrict__ shape) {
    int i, j, k, c;
    const bool ok = tile_cell(d, i, j, k, c);
    p.arc_k = scalars[kScalarArcK] + arc_k_offset;
    // depth weights of the block's 32 k values (non-liquid cells)
    __shared__ float s_wd[kTileK];
    if (threadIdx.y == 0)
        s_wd[threadIdx.x] = arc_weight(blockIdx.x * kTileK + threadIdx.x, p.arc_k, 0.0f, p.pen,
                                       p.enable);
    __syncthreads();
    if (!ok) return;
    inject_cell(H, flags, f_l, scalars[kScalarEpw], cap, ph, cp_f, vp, shape, s_wd[threadIdx.x], c);
}

// The injection over the tiles of the work list (quiet tiles are all GAS, so
// the injection and the ceiling leave them unchanged).
__global__ void __launch_bounds__(256) k_arc_inject_list(Dims d, float* __restrict__ H,
                                                         const int32_t* __restrict__ flags,
                                                         const float* __restrict__ f_l,
                                                         ArcParams p, const float* scalars,
                                                         float arc_k_offset, int cap,
                                                         PhaseParams ph,
                                                         const float* __restrict__ cp_f,
                                                         VarPhase vp,
                                                         const float* __restrict__ shape,
                                                         const int32_t* __restrict__ list,
                                                         int tiles) {
    p.arc_k = scalars[kScalarArcK] + arc_k_offset;
    __shared__ float s_wd[kArcTableMax];
    const bool table = d.nz <= kArcTableMax;
    if (table)
        for (int k = threadIdx.y * kTileK + threadIdx.x; k < d.nz; k += kTileK * kTileJ)
            s_wd[k] = arc_weight(k, p.arc_k, 0.0f, p.pen, p.enable);
    __syncthreads();
    const float epw = scalars[kScalarEpw];
    for_list_tiles(list, imin(list[0], tiles), [&](int ent) {
        int i, j, k, c;
        if (!list_tile_cell(d, ent, i, j, k, c)) return;
        const float wd = table ? s_wd[k] : arc_weight(k, p.arc_k, 0.0f, p.pen, p.enable);
        inject_cell(H, flags, f_l, epw, cap, ph, cp_f, vp, shape, wd, c);
    });
}

struct ThermalArgs {
    PhaseParams ph;
    float cpa, dt_lu, inv_dt;
    int heat_loss, conv, rad;
    float T_amb, h_conv, eps_rad, dt_phys, dx, sigma_sb, h_floor;
    uint32_t* cache_stamp;  // counted up once per step (null: no population cache)
};

// Table path of the thermal stage: the property refresh (kernels.py:1710-1772)
// is computed per cell from T before the cell's own enthalpy update and
// written to the property fields; the update uses the cell's rho*cp and alpha.
struct TableArgs {
    VarPhase vp;
    TableConsts tc;
    WaamMaterialTables tb;
    float* cp_f;
    float* alpha_f;
    float* dg_f;
    float* tau_f;
};

// Thermal stage for every cell: kernels.py:1611-1682 (advect/diffuse),
// 2030-2082 + 1937-1950 (losses, floor), 1519-1556 twice around the ceiling
// 1953-1984 (only the second update_phase is observable), 3016-3032 (T_max),
// 2013-2027 (cooling rate).  H and T are double-buffered so neighbour reads
// see the pre-stage values.  Also resets the active-cell shard counters of the step and
// counts up the population copy's stamp (one thermal stage between two collisions).
// TABLES: refresh_thermal_properties, advect_diffuse_temperature_variable,
// clamp_enthalpy_floor and update_phase_variable_cp / the variable ceiling
// (kernels.py:1710-1863, 1922-1935, 1988-2010) instead of the scalar forms.
template <bool TABLES>
__device__ __forceinline__ void thermal_cell(
    const Dims& d, const float* __restrict__ H, float* __restrict__ H_next,
    const float* __restrict__ T, float* __restrict__ T_next, float* __restrict__ f_l,
    const float* __restrict__ ux, const float* __restrict__ uy, const float* __restrict__ uz,
    const int32_t* __restrict__ flags, float* __restrict__ T_max, float* __restrict__ T_prev,
    float* __restrict__ dT_dt, const ThermalArgs& a, const TableArgs& tba, uint32_t* status,
    int i, int j, int k, int c) {
    const int flag = flags[c];
    float h = H[c];
    CellProps pr{};
    if (TABLES) {
        pr = refresh_cell(tba.tb, tba.tc, flag, T[c]);
        tba.cp_f[c] = pr.cp_rho;
        tba.alpha_f[c] = pr.alpha;
        tba.dg_f[c] = pr.dgamma;
        tba.tau_f[c] = pr.tau;
    }
    if (flag != GAS) {
        float u = 0.0f, v = 0.0f, w = 0.0f;
        if (flag != SOLID) {
            u = ux[c];
            v = uy[c];
            w = uz[c];
        }
        const float cpa = TABLES ? pr.cp_rho * pr.alpha : a.cpa;
        h = h + thermal_dh_offsets(d, H, T, flags, u, v, w, i, j, k, c, flag, h, T[c], cpa,
                                   a.dt_lu);
        if (a.heat_loss) {
            int ne = 0;
            const int sx = d.ny * d.nz;
            if (k + 1 < d.nz && flags[c + 1] == GAS) ne++;
            if (j + 1 < d.ny && flags[c + d.nz] == GAS) ne++;
            if (j - 1 >= 0 && flags[c - d.nz] == GAS) ne++;
            if (i + 1 < d.nx && flags[c + sx] == GAS) ne++;
            if (i - 1 >= 0 && flags[c - sx] == GAS) ne++;
            if (ne != 0) {
                float Te = fmin_(T[c], 2500.0f);
                float q = 0.0f;
                if (a.conv == 1) q += a.h_conv * (Te - a.T_amb);
                if (a.rad == 1) {
                    float t4 = Te * Te * Te * Te;
                    float a4 = a.T_amb * a.T_amb * a.T_amb * a.T_amb;
                    q += a.eps_rad * a.sigma_sb * (t4 - a4);
                }
                h -= q * (float)ne * a.dt_phys / a.dx;
            }
            const float h_floor = TABLES ? pr.cp_rho * a.T_amb : a.h_floor;
            if (h < h_floor) h = h_floor;
        }
        if (a.ph.cap_enabled) h = TABLES ? cap_h_var(tba.vp, pr.cp_rho, h) : cap_h(a.ph, h);
        if (status != nullptr && !isfinite(h)) atomicOr(status, WAAM_HEALTH_NONFINITE_H);
    }
    float t, fl;
    if (TABLES)
        phase_var(tba.vp, pr.cp_rho, h, t, fl);
    else
        phase(a.ph, h, t, fl);
    H_next[c] = h;
    T_next[c] = t;
    f_l[c] = fl;
    if (flag != GAS) {
        if (t > T_max[c]) T_max[c] = t;
        float tp = T_prev[c];
        dT_dt[c] = (t - tp) * a.inv_dt;
        T_prev[c] = t;
    }
}

template <bool TABLES>
__global__ void __launch_bounds__(256) k_thermal_fused(
    Dims d, const float* __restrict__ H, float* __restrict__ H_next, const float* __restrict__ T,
    float* __restrict__ T_next, float* __restrict__ f_l, const float* __restrict__ ux,
    const float* __restrict__ uy, const float* __restrict__ uz, const int32_t* __restrict__ flags,
    float* __restrict__ T_max, float* __restrict__ T_prev, float* __restrict__ dT_dt,
    unsigned* active_count, ThermalArgs a, TableArgs tba, uint32_t* status) {
    if (blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0) {
        const int t = threadIdx.y * kTileK + threadIdx.x;
        if (t < kActiveShards) active_count[t] = 0u;
        if (t == 0 && a.cache_stamp) *a.cache_stamp += 1u;
    }
    int i, j, k, c;
    if (!tile_cell(d, i, j, k, c)) return;
    thermal_cell<TABLES>(d, H, H_next, T, T_next, f_l, ux, uy, uz, flags, T_max, T_prev, dT_dt, a,
                         tba, status, i, j, k, c);
}

// The thermal stage over the tiles of the work list.  A quiet tile was all
// GAS in the flags of this step and of the step before, so the previous
// step already left both enthalpy / temperature buffers equal there and its
// column pass left f_l = 0 (GAS): the stage would rewrite the same values.
// Six blocks per SM without tables (at most 42 registers; measured: the stage
// 22 % faster); the table form keeps its registers.
template <bool TABLES>
__global__ void __launch_bounds__(256, TABLES ? 1 : 6) k_thermal_list(
    Dims d, const float* __restrict__ H, float* __restrict__ H_next, const float* __restrict__ T,
    float* __restrict__ T_next, float* __restrict__ f_l, const float* __restrict__ ux,
    const float* __restrict__ uy, const float* __restrict__ uz, const int32_t* __restrict__ flags,
    float* __restrict__ T_max, float* __restrict__ T_prev, float* __restrict__ dT_dt,
    unsigned* active_count, ThermalArgs a, TableArgs tba, uint32_t* status,
    const int32_t* __restrict__ list, int tiles) {
    if (blockIdx.x == 0) {
        const int t = threadIdx.y * kTileK + threadIdx.x;
        if (t < kActiveShards) active_count[t] = 0u;
        if (t == 0 && a.cache_stamp) *a.cache_stamp += 1u;
    }
    for_list_tiles(list, imin(list[0], tiles), [&](int ent) {
        int i, j, k, c;
        if (!list_tile_cell(d, ent, i, j, k, c)) return;
        thermal_cell<TABLES>(d, H, H_next, T, T_next, f_l, ux, uy, uz, flags, T_max, T_prev, dT_dt,
                             a, tba, status, i, j, k, c);
    });
}

// VOF advection + reinitialisation (kernels.py:2320-2391) -> phi_tmp.  A gas
// cell whose six face neighbours are gas (or outside y/z) has zero velocity on
// every face, so all fluxes vanish and phi_tmp = reinit(phi) exactly.
__device__ __forceinline__ void vof_cell(const Dims& d, const float* __restrict__ phi,
                                         float* __restrict__ phi_tmp,
                                         const float* __restrict__ ux,
                                         const float* __restrict__ uy,
                                         const float* __restrict__ uz,
                                         const int32_t* __restrict__ flags, int i, int j, int k,
                                         int c) {
    const int flag = flags[c];
    const float p0 = phi[c];
    float p = p0;
    if (flag != SOLID) {
        // kernels.py:2320-2361 for one non-solid cell: donor-cell fluxes through
        // the six faces (x periodic, no flux through y / z domain faces or into
        // SOLID cells, GAS cells at rest).  The six neighbour flags are loaded
        // once for the quiet-gas test and the fluxes.
        const int sx = d.ny * d.nz, sy = d.nz;
        const int cw = i > 0 ? c - sx : c + (d.nx - 1) * sx;
        const int ce = i < d.nx - 1 ? c + sx : c - (d.nx - 1) * sx;
        const bool hs = j > 0, hn = j < d.ny - 1, hb = k > 0, ht = k < d.nz - 1;
        const int fw = flags[cw], fe = flags[ce];
        const int fs = hs ? flags[c - sy] : GAS, fn = hn ? flags[c + sy] : GAS;
        const int fb = hb ? flags[c - 1] : GAS, ft = ht ? flags[c + 1] : GAS;
        // a GAS cell whose six face neighbours are GAS (or outside y / z) has zero
        // velocity on every face: phi_tmp = reinit(phi) exactly
        const bool quiet = flag == GAS && ((fw == GAS) & (fe == GAS) & (fs == GAS) & (fn == GAS) &
                                           (fb == GAS) & (ft == GAS));
        if (!quiet) {
            const bool moving = flag != GAS;
            const float vx = moving ? ux[c] : 0.0f, vy = moving ? uy[c] : 0.0f;
            const float vz = moving ? uz[c] : 0.0f;
            // flux through the face between this cell and neighbour cn (flag fn_):
            // face velocity = mean of the lower and upper cell, upwind phi
            auto flux = [&](bool exists, int fn_, int cn, const float* vel, float v_own,
                            bool own_lower) -> float {
                if (!exists || fn_ == SOLID) return 0.0f;
                const float vn = fn_ != GAS ? vel[cn] : 0.0f;
                const float uf = own_lower ? 0.5f * (v_own + vn) : 0.5f * (vn + v_own);
                if (uf > 0.0f) return uf * (own_lower ? p0 : phi[cn]);
                return uf * (own_lower ? phi[cn] : p0);
            };
            const float Fe = flux(true, fe, ce, ux, vx, true);
            const float Fw = flux(true, fw, cw, ux, vx, false);
            const float Fn = flux(hn, fn, c + sy, uy, vy, true);
            const float Fs = flux(hs, fs, c - sy, uy, vy, false);
            const float Ft = flux(ht, ft, c + 1, uz, vz, true);
            const float Fb = flux(hb, fb, c - 1, uz, vz, false);
            p = p0 - (Fe - Fw) - (Fn - Fs) - (Ft - Fb);
        }
    }
    phi_tmp[c] = reinit_phi(p, flag);
}

__global__ void __launch_bounds__(256) k_vof_advect(Dims d, const float* __restrict__ phi,
                                                    float* __restrict__ phi_tmp,
                                                    const float* __restrict__ ux,
                                                    const float* __restrict__ uy,
                                                    const float* __restrict__ uz,
                                                    const int32_t* __restrict__ flags) {
    int i, j, k, c;
    if (!tile_cell(d, i, j, k, c)) return;
    vof_cell(d, phi, phi_tmp, ux, uy, uz, flags, i, j, k, c);
}

// VOF advection over the tiles of the work list.  In a quiet tile every cell
// within two lattice steps is GAS: all face velocities vanish and phi is
// already reinitialised, so phi_tmp would equal phi; the column pass skips
// those tiles, and a worked cell next to one only compares its phi_tmp (<=
// phi < 0.05 there) against 0.55.
__global__ void __launch_bounds__(256) k_vof_list(Dims d, const float* __restrict__ phi,
                                                  float* __restrict__ phi_tmp,
                                                  const float* __restrict__ ux,
                                                  const float* __restrict__ uy,
                                                  const float* __restrict__ uz,
                                                  const int32_t* __restrict__ flags,
                                                  const int32_t* __restrict__ list, int tiles) {
    for_list_tiles(list, imin(list[0], tiles), [&](int ent) {
        int i, j, k, c;
        if (!list_tile_cell(d, ent, i, j, k, c)) return;
        vof_cell(d, phi, phi_tmp, ux, uy, uz, flags, i, j, k, c);
    });
}

struct ColumnArgs {
    int vof, wetting, nz_solid;
    float cos_t, sin_t;
    float dt_phys, T800, T1100, Ts;
    int zero_forces;  // keep F == 0 outside the active cells (see k_collide_list)
    int clear_all;    // the previous step left forces outside the active set
    int shard_cap;    // list slots per shard: ceil(nx*ny / kActiveShards) * nz
    // quiet tiles (null: none): work byte per tile, chunk bits per column chunk
    const uint8_t* tile_work;
    uint8_t* chunk_bits;
    int tile_history;  // 1: chunk bit 1 takes the previous bit 0; 0: history restarts
    int32_t* tile_list;  // non-null: its count is zeroed for the next step's classification
};

// Column pass: contact-angle BC (kernels.py:933-991) on phi_tmp, flags from
// phi (2394-2419), phi/f_l sync (3484-3504) and time-above-T (3261-3283,
// which runs after collide/stream in the reference but only reads T and the
// post-VOF flags).  Appends every FLUID/IFACE cell to the active list
// (column c goes to shard c % 64, in k order within a warp) and zeroes the
// force of cells leaving the active set.  Eight blocks per SM (at most 32
// registers; measured: the step 1.3-1.8 % faster).
__global__ void __launch_bounds__(256, 8) k_column(Dims d, const float* __restrict__ phi_tmp,
                                                float* __restrict__ phi,
                                                int32_t* __restrict__ flags,
                                                float* __restrict__ f_l,
                                                const float* __restrict__ T,
                                                float* __restrict__ t800,
                                                float* __restrict__ t1100,
                                                float* __restrict__ tsol, float* __restrict__ Fx,
                                                float* __restrict__ Fy, float* __restrict__ Fz,
                                                int* __restrict__ active_list,
                                                unsigned* __restrict__ active_count,
                                                int32_t* __restrict__ flags_copy,
                                                float* __restrict__ scalars,
                                                ColumnArgs a) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        scalars[kScalarCollideArcK] = scalars[kScalarArcK];
        scalars[kScalarCollideArcI] = scalars[kScalarArcI];
        scalars[kScalarCollideArcJ] = scalars[kScalarArcJ];
        // this step's work list was read by the thermal and VOF stages
        if (a.tile_list != nullptr) a.tile_list[0] = 0;
    }
    if (warp >= d.nx * d.ny) return;
    const int lane = threadIdx.x & 31;
    int i = warp / d.ny, j = warp % d.ny;
    ContactConst cc = contact_const(a.cos_t, a.sin_t);
    const float* src = a.vof ? phi_tmp : phi;
    const int KT = tiles_k(d), JT = tiles_j(d);
    // The column's work bytes and chunk bits, all requested at once (lane kt
    // holds chunk kt and kt + 32; KT <= 64 with tiles on), so that no chunk
    // waits for a load of its own before its cells are requested.
    uint64_t quiet_mask = 0;
    unsigned cb_lo = 0u, cb_hi = 0u;
    if (a.tile_work != nullptr) {
        const int64_t tw0 = ((int64_t)i * JT + j / kTileJ) * KT;
        const int64_t cb0 = ((int64_t)i * d.ny + j) * KT;
        const bool in0 = lane < KT, in1 = lane + 32 < KT;
        const unsigned w0 = in0 ? a.tile_work[tw0 + lane] : 1u;
        const unsigned w1 = in1 ? a.tile_work[tw0 + lane + 32] : 1u;
        cb_lo = in0 ? a.chunk_bits[cb0 + lane] : 0u;
        cb_hi = in1 ? a.chunk_bits[cb0 + lane + 32] : 0u;
        quiet_mask = (uint64_t)__ballot_sync(0xffffffffu, w0 == 0u) |
                     ((uint64_t)__ballot_sync(0xffffffffu, w1 == 0u) << 32);
    }
    // chunk kc's bits as they were before this pass (warp-uniform kc)
    auto old_bits = [&](int kc) -> unsigned {
        return __shfl_sync(0xffffffffu, kc < 32 ? cb_lo : cb_hi, kc & 31);
    };
    // A quiet chunk keeps its (GAS) flags.  Its flag copy is still written
    // until the last three passes have all written GAS copies of it (chunk
    // bits 4-5 count them), so that each of the three rotating copies holds
    // the whole step's flags however old its last worked pass is.
    auto skip = [&](int k0) -> bool {
        const bool quiet = (quiet_mask >> (k0 >> 5)) & 1ull;
        if (quiet && flags_copy != nullptr) {
            uint8_t* cbp = a.chunk_bits + ((int64_t)i * d.ny + j) * KT + (k0 >> 5);
            const unsigned old = old_bits(k0 >> 5);
            const unsigned cnt = (old >> 4) & 3u;
            if (cnt < 3u) {
                if (k0 + lane < d.nz) flags_copy[d.idx(i, j, k0 + lane)] = GAS;
                __syncwarp();
                if (lane == 0) *cbp = (uint8_t)((old & 0xcfu) | ((cnt + 1u) << 4));
            }
        }
        return quiet;
    };
    contact_column(d, src, flags, i, j, a.vof && a.wetting, cc,
                   [&](int k, int c, float v, int flag_old, bool valid) {
                       int flag = flag_old;
                       if (valid) {
                           if (a.vof) {
                               float fl = f_l[c];
                               flag = flag_from(v, fl, k, a.nz_solid);
                               phi[c] = v;
                               flags[c] = flag;
                               if (flag == GAS || v < 0.05f || flag == SOLID) {
                                   if (fl != 0.0f) f_l[c] = 0.0f;
                               }
                           }
                           if (flag != GAS) {
                               float t = T[c];
                               if (t >= a.T800) t800[c] += a.dt_phys;
                               if (t >= a.T1100) t1100[c] += a.dt_phys;
                               if (t >= a.Ts) tsol[c] += a.dt_phys;
                           }
                           if (a.zero_forces && !is_active(flag) &&
                               (a.clear_all || is_active(flag_old))) {
                               Fx[c] = 0.0f;
                               Fy[c] = 0.0f;
                               Fz[c] = 0.0f;
                           }
                       }
                       if (valid && flags_copy) flags_copy[c] = flag;
                       if (a.chunk_bits != nullptr) {
                           // chunk bits: all GAS, that of the previous pass, top and
                           // bottom two cells GAS (cells beyond nz count as GAS)
                           const unsigned gm = __ballot_sync(0xffffffffu, !valid || flag == GAS);
                           const unsigned old = old_bits(k >> 5);
                           if (lane == 0) {
                               uint8_t* cbp = a.chunk_bits + ((int64_t)i * d.ny + j) * KT + (k >> 5);
                               unsigned nb = gm == 0xffffffffu ? 1u : 0u;
                               if (a.tile_history && (old & 1u)) nb |= 2u;
                               if ((gm >> 30) == 3u) nb |= 4u;
                               if ((gm & 3u) == 3u) nb |= 8u;
                               // bits 4-5: consecutive passes (at most 3) whose
                               // flag copies of the chunk were all GAS
                               unsigned cnt = a.tile_history ? (old >> 4) & 3u : 0u;
                               cnt = (nb & 1u) && flags_copy ? (cnt < 3u ? cnt + 1u : 3u) : 0u;
                               *cbp = (uint8_t)(nb | (cnt << 4));
                           }
                       }
                       bool act = valid && is_active(flag);
                       unsigned m = __ballot_sync(0xffffffffu, act);
                       if (m) {
                           // one counter per shard of columns keeps the atomics spread out
                           const int shard = warp & (kActiveShards - 1);
                           unsigned base = 0;
                           if (lane == 0)
                               base = atomicAdd(active_count + shard, (unsigned)__popc(m));
                           base = __shfl_sync(0xffffffffu, base, 0);
                           if (act)
                               active_list[(int64_t)shard * a.shard_cap + base +
                                           __popc(m & ((1u << lane) - 1u))] = c;
                       }
                   }, skip);
}

struct CollideArgs {
    ForceParams P;
    int kind, from_buffer;  // kind 0 MRT, 1 SRT, 2 SRT with the per-cell tau_f
    float omega, omega_b, C_darcy, u_cap;
    const float* dgamma_f;  // non-null: Marangoni with the per-cell dgamma (table path)
    const float* tau_f;
    float* tape_f;          // non-null: adjoint tape of the pre-collision populations
    int32_t* tape_cells;
    int32_t* tape_count;
    int64_t tape_cap;
    // non-null: the Lorentz force J x B of the welding current is added after
    // the other body forces and before their clamp
    const float* J[3];
    const float* B[3];
    float lz_dt, lz_dx, lz_rho;
    uint32_t* status;       // health word (null: off)
    float rho_lo, rho_hi;   // density band of WAAM_HEALTH_RHO_RANGE (off when hi <= lo)
    // population cache (cache_out null: off; cache_in null: not read this step)
    const void* cache_in;
    void* cache_out;
    const uint32_t* stamp;
};

// Compact copy of the collision's output (WaamFields.pop_cache_*).  Slot
// (column * ceil(nz/32) + k/32) * kCacheDepth + rank, rank = the cell's place
// among the active cells of its 32-cell column chunk (the column pass lists
// them one after another in k order, so the rank comes from the list entries
// just before the cell's); cells of rank kCacheDepth and above go without.
// A slot holds the cell's 19 stored populations (4-byte storage: one word
// each; 2-byte storage: two per word, the last half-word zero), then the
// cell index and the stamp of the step that wrote it: 24 or 12 words, read
// and written as 16-byte vectors.
constexpr int kCacheDepth = 2;

__device__ __forceinline__ uint32_t pop_bits(float v) { return __float_as_uint(v); }
__device__ __forceinline__ uint32_t pop_bits(__half v) { return __half_as_ushort(v); }
__device__ __forceinline__ uint32_t pop_bits(__nv_bfloat16 v) { return __bfloat16_as_ushort(v); }
template <typename T>
__device__ __forceinline__ T pop_of_bits(uint32_t b);
template <>
__device__ __forceinline__ float pop_of_bits<float>(uint32_t b) { return __uint_as_float(b); }
template <>
__device__ __forceinline__ __half pop_of_bits<__half>(uint32_t b) {
    return __ushort_as_half((unsigned short)b);
}
template <>
__device__ __forceinline__ __nv_bfloat16 pop_of_bits<__nv_bfloat16>(uint32_t b) {
    return __ushort_as_bfloat16((unsigned short)b);
}

template <int S>
struct PopCache {
    typedef typename Pop<S>::T T;
    static constexpr int kWords = S == kStoreF32 ? 24 : 12;
    static constexpr int kTag = S == kStoreF32 ? 19 : 10;   // cell index, then stamp

    // f = the slot's populations if it holds cell c with this stamp
    __device__ static __forceinline__ bool load(const void* cache, int slot, int c,
                                                uint32_t stamp, float* f) {
        const uint4* v = reinterpret_cast<const uint4*>(cache) + (int64_t)slot * (kWords / 4);
        uint32_t w[kWords];
#pragma unroll
        for (int u = 0; u < kWords / 4; ++u) {
            const uint4 x = v[u];
            w[4 * u] = x.x;
            w[4 * u + 1] = x.y;
            w[4 * u + 2] = x.z;
            w[4 * u + 3] = x.w;
        }
        if (w[kTag] != (uint32_t)c || w[kTag + 1] != stamp) return false;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            const uint32_t b = S == kStoreF32 ? w[q] : (w[q >> 1] >> (16 * (q & 1))) & 0xffffu;
            f[q] = Pop<S>::get(pop_of_bits<T>(b), q);
        }
        return true;
    }

    __device__ static __forceinline__ void store(void* cache, int slot, int c, uint32_t stamp,
                                                 const T* o) {
        uint32_t w[kWords];
#pragma unroll
        for (int u = 0; u < kWords; ++u) w[u] = 0u;
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            if (S == kStoreF32)
                w[q] = pop_bits(o[q]);
            else
                w[q >> 1] |= pop_bits(o[q]) << (16 * (q & 1));
        }
        w[kTag] = (uint32_t)c;
        w[kTag + 1] = stamp;
        uint4* v = reinterpret_cast<uint4*>(cache) + (int64_t)slot * (kWords / 4);
#pragma unroll
        for (int u = 0; u < kWords / 4; ++u)
            v[u] = make_uint4(w[4 * u], w[4 * u + 1], w[4 * u + 2], w[4 * u + 3]);
    }
};

// kernels.py:1479-1513 apply_lorentz_JxB for one cell (f_l >= 0.05)
__device__ __forceinline__ void lorentz_add(const float* const* J, const float* const* B, int64_t c,
                                            float fl, float dt, float dx, float rho_ref,
                                            float& fx, float& fy, float& fz) {
    const float jx = J[0][c], jy = J[1][c], jz = J[2][c];
    const float bx = B[0][c], by = B[1][c], bz = B[2][c];
    const float fxp = jy * bz - jz * by, fyp = jz * bx - jx * bz, fzp = jx * by - jy * bx;
    const float flw = fmin_(1.0f, fl);
    const float scale = flw * dt * dt / (rho_ref * dx);
    fx += fxp * scale;
    fy += fyp * scale;
    fz += fzp * scale;
}

// Body forces + collision + Mach clamp over the active (FLUID/IFACE) cells
// listed by k_column, shard after shard (solvers/coupled_step.py:298-402).  Forces stay in
// registers and are written once as the step's force field (== the
// reference's F_snap); every other cell keeps F == 0.
template <int S>
__global__ void __launch_bounds__(kListThreads) k_collide_list(
    Dims d, const typename Pop<S>::T* __restrict__ f_src, typename Pop<S>::T* __restrict__ f_dst,
    float* __restrict__ rho,
    float* __restrict__ ux, float* __restrict__ uy, float* __restrict__ uz,
    float* __restrict__ Fx, float* __restrict__ Fy, float* __restrict__ Fz,
    const float* __restrict__ phi, const float* __restrict__ T, const float* __restrict__ f_l,
    const int32_t* __restrict__ flags, const float* __restrict__ scalars,
    const int* __restrict__ active_list, const unsigned* __restrict__ active_count,
    int shard_cap, CollideArgs a) {
    const size_t n = (size_t)d.n();
    __shared__ unsigned start[kActiveShards + 1];
    if (threadIdx.x < 32) {
        // exclusive prefix of the 64 shard counts (two per lane)
        unsigned c0 = active_count[2 * threadIdx.x], c1 = active_count[2 * threadIdx.x + 1];
        unsigned v = c0 + c1, incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
            if (threadIdx.x >= o) incl += y;
        }
        unsigned excl = incl - v;
        start[2 * threadIdx.x] = excl;
        start[2 * threadIdx.x + 1] = excl + c0;
        if (threadIdx.x == 31) start[kActiveShards] = incl;
    }
    __syncthreads();
    const unsigned cnt = start[kActiveShards];
    const bool tape = a.tape_f != nullptr && (int64_t)cnt <= a.tape_cap;
    if (a.tape_f != nullptr && blockIdx.x == 0 && threadIdx.x == 0)
        *a.tape_count = tape ? (int32_t)cnt : -1;
    ForceParams P = a.P;
    P.arc_k = scalars[kScalarCollideArcK];
    P.arc_i = scalars[kScalarCollideArcI];
    P.arc_j = scalars[kScalarCollideArcJ];
    const bool lorentz = a.J[0] != nullptr;
    const float F_cap = P.F_cap;
    if (lorentz) P.F_cap = 0.0f;   // clamped below, after J x B
    // the stamp of this step (slots of the previous step carry stamp - 1)
    const uint32_t stamp = a.cache_out != nullptr ? *a.stamp : 0u;
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt;
         t += gridDim.x * blockDim.x) {
        int lo = 0, hi = kActiveShards;  // last shard with start <= t
        while (hi - lo > 1) {
            int mid = (lo + hi) >> 1;
            if (start[mid] <= t) lo = mid; else hi = mid;
        }
        const int64_t at = (int64_t)lo * shard_cap + (t - start[lo]);
        const int c = active_list[at];
        const int k = c % d.nz;
        const int r = c / d.nz;
        const int j = r % d.ny;
        const int i = r / d.ny;
        int slot = -1;
        if (a.cache_out != nullptr) {
            // rank in the chunk: the entries before it in this shard that lie
            // in the same chunk below it (cells c - (k % 32) .. c - 1)
            const int chunk_lo = c - (k & 31);
            const unsigned pos = t - start[lo];
            int rk = 0;
            while (rk < kCacheDepth && (unsigned)rk < pos) {
                const int e = active_list[at - 1 - rk];
                if (e < chunk_lo || e >= c) break;
                ++rk;
            }
            if (rk < kCacheDepth) slot = (r * ((d.nz + 31) >> 5) + (k >> 5)) * kCacheDepth + rk;
        }
        // the populations (DRAM) are requested first so that their latency
        // overlaps the force stencil (cache-resident phi, T, flags): from the
        // cache slot when it holds this cell from the previous step, else
        // from the 19 population planes
        float f[19], o[19];
        const bool hit = a.cache_in != nullptr && slot >= 0 &&
                         PopCache<S>::load(a.cache_in, slot, c, stamp - 1u, f);
        if (!hit) {
#pragma unroll
            for (int q = 0; q < 19; ++q) f[q] = Pop<S>::get(f_src[q * n + c], q);
        }
        if (tape) {
            a.tape_cells[t] = c;
#pragma unroll
            for (int q = 0; q < 19; ++q) a.tape_f[(int64_t)q * a.tape_cap + t] = f[q];
        }
        const float tau_c = a.kind == 2 ? a.tau_f[c] : 0.0f;
        if (a.dgamma_f) P.dgamma = a.dgamma_f[c];
        float fx = 0.0f, fy = 0.0f, fz = 0.0f;
        if (a.from_buffer) {
            fx = Fx[c];
            fy = Fy[c];
            fz = Fz[c];
        }
        float fl = f_l[c];
        cell_forces_preloaded(d, P, phi, T, flags, i, j, k, c, fl, fx, fy, fz);
        if (lorentz) {
            // the reference order: the other forces, J x B, then the clamp
            // (solvers/coupled_step.py:298-362; kernels.py:3286-3309)
            if (!(fl < 0.05f)) lorentz_add(a.J, a.B, c, fl, a.lz_dt, a.lz_dx, a.lz_rho, fx, fy, fz);
            if (F_cap > 0.0f) {
                const float mag = sqrtf(fx * fx + fy * fy + fz * fz);
                if (mag > F_cap) {
                    const float sc = F_cap / (mag + 1e-12f);
                    fx = fx * sc;
                    fy = fy * sc;
                    fz = fz * sc;
                }
            }
        }
        float rr, u, v, w;
        if (a.kind == 0)
            collide_mrt_cell(f, fl, fx, fy, fz, a.omega, a.omega_b, a.C_darcy, o, rr, u, v, w);
        else  // kernels.py:2889-2965: omega = 1 / (tau + 1e-6) per cell
            collide_srt_cell(f, fl, fx, fy, fz, a.kind == 2 ? 1.0f / (tau_c + 1e-6f) : a.omega,
                             a.C_darcy, o, rr, u, v, w);
        typename Pop<S>::T so[19];
#pragma unroll
        for (int q = 0; q < 19; ++q) {
            so[q] = Pop<S>::put(o[q], q);
            f_dst[q * n + c] = so[q];
        }
        if (slot >= 0) PopCache<S>::store(a.cache_out, slot, c, stamp, so);
        if (a.u_cap > 0.0f) clamp_mach(u, v, w, a.u_cap);
        if (a.status != nullptr) {
            if (!(isfinite(rr) && isfinite(u) && isfinite(v) && isfinite(w)))
                atomicOr(a.status, WAAM_HEALTH_NONFINITE_LBM);
            else if (a.rho_hi > a.rho_lo && !(rr >= a.rho_lo && rr <= a.rho_hi))
                atomicOr(a.status, WAAM_HEALTH_RHO_RANGE);
        }
        rho[c] = rr;
        ux[c] = u;
        uy[c] = v;
        uz[c] = w;
        Fx[c] = fx;
        Fy[c] = fy;
        Fz[c] = fz;
    }
}

// The J x B force the reference adds to SOLID cells with f_l >= 0.05 (it is
// part of the force field the step leaves; the collision never reads it).
__global__ void k_lorentz_solid(int64_t n, const int32_t* __restrict__ flags,
                                const float* __restrict__ f_l, float* Fx, float* Fy, float* Fz,
                                const float* Jx, const float* Jy, const float* Jz,
                                const float* Bx, const float* By, const float* Bz, float dt,
                                float dx, float rho_ref) {
    const float* J[3] = {Jx, Jy, Jz};
    const float* B[3] = {Bx, By, Bz};
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        if (flags[c] != SOLID) continue;
        const float fl = f_l[c];
        if (fl < 0.05f) continue;
        float fx = Fx[c], fy = Fy[c], fz = Fz[c];
        lorentz_add(J, B, c, fl, dt, dx, rho_ref, fx, fy, fz);
        Fx[c] = fx;
        Fy[c] = fy;
        Fz[c] = fz;
    }
}

struct TailArgs {
    float cp_rho, Ts, Tl, L_rho;
    int remelt, trailing, cooled;
    float dir_x, dir_y, dir_z, lookback, T_freeze;
    const float* cp_f;  // non-null: the per-cell rho*cp (kernels.py:2454-2570)
};

// solvers/coupled_step.py:426-458: remelt_hot_solid_scalar (kernels.py:2489),
// solidify_trailing_pool_scalar (2573), solidify_cooled_metal (2422); all
// per cell, applied in the reference order.
__global__ void __launch_bounds__(256) k_tail(Dims d, float* T, float* H, float* f_l, float* phi,
                                              int32_t* flags, float* ux, float* uy, float* uz,
                                              const float* scalars, TailArgs a) {
    int i, j, k, c;
    if (!tile_cell(d, i, j, k, c)) return;
    int flag = flags[c];
    if (a.remelt && flag == SOLID) {
        float Tc = T[c];
        if (!(Tc <= a.Ts + 5.0f)) {
            const float cp_rho = a.cp_f ? a.cp_f[c] : a.cp_rho;
            float H_sol = cp_rho * a.Ts;
            float fl;
            if (Tc >= a.Tl) {
                fl = 1.0f;
                H[c] = cp_rho * a.Tl + a.L_rho + cp_rho * (Tc - a.Tl);
            } else {
                fl = (Tc - a.Ts) / (a.Tl - a.Ts + 1e-6f);
                H[c] = H_sol + fl * a.L_rho;
            }
            f_l[c] = fl;
            phi[c] = 1.0f;
            flags[c] = FLUID;
            flag = FLUID;
        }
    }
    if (a.trailing && flag != GAS && !(phi[c] < 0.85f || f_l[c] < 0.05f)) {
        float arc_k = scalars[kScalarArcK];
        float di = (float)i - scalars[kScalarArcI], dj = (float)j - scalars[kScalarArcJ];
        float dk = (float)k - arc_k;
        float proj = di * a.dir_x + dj * a.dir_y + dk * a.dir_z;
        if (!(proj > -a.lookback) && !(T[c] >= a.T_freeze)) {
            H[c] = (a.cp_f ? a.cp_f[c] : a.cp_rho) * (a.Ts - 1.0f);
            T[c] = a.Ts - 1.0f;
            f_l[c] = 0.0f;
            phi[c] = 1.0f;
            flags[c] = SOLID;
            ux[c] = uy[c] = uz[c] = 0.0f;
            flag = SOLID;
        }
    }
    if (a.cooled && flag != GAS && !(phi[c] < 0.85f)) {
        if (f_l[c] < 0.02f && T[c] < a.Ts) {
            flags[c] = SOLID;
            phi[c] = 1.0f;
            f_l[c] = 0.0f;
            ux[c] = uy[c] = uz[c] = 0.0f;
        }
    }
}

static ArcParams arc_params(const WaamStepParams* p) {
    ArcParams a{};
    a.kind = p->arc_kind;
    a.inv2s2 = 1.0f / (2.0f * p->sigma_heat * p->sigma_heat);
    a.sign = p->sign;
    a.ff = p->ff;
    a.fr = p->fr;
    a.a_f = p->a_f;
    a.a_r = p->a_r;
    a.b = p->gb;
    a.c = p->gc;
    a.pen = p->pen;
    a.enable = p->surface_weighting;
    return a;
}

// Second stream and fork/join events of the fused step, one set per device
// (created on the first step on that device, which should not be inside a
// stream capture).  Calls on different host threads share them; every fork is
// ordered by its own event record, so sharing only serialises.
// hi: the stages of the step (highest priority); s2: VOF advection beside the
// thermal stage (highest priority); s3: the pending stream of the previous
// step (lowest priority), so that its blocks fill what the latency-bound arc,
// thermal and VOF kernels leave free instead of being placed before them.
struct AuxStream {
    cudaStream_t hi = nullptr;
    cudaStream_t s2 = nullptr;
    cudaStream_t s3 = nullptr;
    cudaEvent_t ev[10] = {};
};

static int aux_stream(AuxStream** out) {
    static std::mutex mu;
    static AuxStream table[kMaxDevices];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(WAAM_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(WAAM_ERR_INVALID, "step_main: device index");
    std::lock_guard<std::mutex> lock(mu);
    AuxStream& a = table[dev];
    if (!a.s2) {
        int least = 0, greatest = 0;
        e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
        if (e == cudaSuccess)
            e = cudaStreamCreateWithPriority(&a.hi, cudaStreamNonBlocking, greatest);
        if (e == cudaSuccess)
            e = cudaStreamCreateWithPriority(&a.s2, cudaStreamNonBlocking, greatest);
        if (e == cudaSuccess)
            e = cudaStreamCreateWithPriority(&a.s3, cudaStreamNonBlocking, least);
        for (int q = 0; q < 10 && e == cudaSuccess; ++q)
            e = cudaEventCreateWithFlags(&a.ev[q], cudaEventDisableTiming);
        if (e != cudaSuccess) {
            a.s2 = nullptr;
            return fail(WAAM_ERR_CUDA, cudaGetErrorString(e));
        }
    }
    *out = &a;
    return WAAM_OK;
}

// The stages of a call run on the library's high-priority stream, forked from
// and joined back into the caller's stream (events ev[fork], ev[fork + 1]).
struct WorkStream {
    cudaStream_t caller = nullptr, s = nullptr;
    AuxStream* aux = nullptr;
    int slot = 0;
    int err = WAAM_OK;
    WorkStream(cudaStream_t c, bool use_hi, int fork_slot) : caller(c), s(c), slot(fork_slot) {
        if (!use_hi) return;
        err = aux_stream(&aux);
        if (err) return;
        cudaEventRecord(aux->ev[slot], caller);
        cudaStreamWaitEvent(aux->hi, aux->ev[slot], 0);
        s = aux->hi;
    }
    ~WorkStream() {
        if (aux && s != caller) {
            cudaEventRecord(aux->ev[slot + 1], s);
            cudaStreamWaitEvent(caller, aux->ev[slot + 1], 0);
        }
    }
};

static bool fields_ok(const WaamFields* f) {
    return f && f->f_src && f->f_dst && f->rho && f->ux && f->uy && f->uz && f->T && f->T_next &&
           f->H && f->H_next && f->f_l && f->phi && f->phi_tmp && f->flags && f->T_max &&
           f->T_prev && f->dT_dt && f->t800 && f->t1100 && f->tsol && f->Fx && f->Fy && f->Fz &&
           f->step_scalars && dims_ok(f->nx, f->ny, f->nz) && f->f_src != f->f_dst &&
           f->H != f->H_next && f->T != f->T_next;
}

static bool tables_fields_ok(const WaamFields* f, const WaamStepParams* p) {
    if (!p->use_tables) return true;
    const int32_t cnt[4] = {p->tables.n_cp, p->tables.n_k, p->tables.n_mu, p->tables.n_dgamma};
    for (int q = 0; q < 4; ++q)
        if (cnt[q] < 0 || cnt[q] > WAAM_TABLE_KNOTS) return false;
    return f->cp_rho_f && f->alpha_f && f->dgamma_f && f->tau_f;
}

// waam_step_pre starts a pending stream on the library's low-priority stream
static bool stream_work(const WaamStepParams* p) {
    return p->stream_lag || (p->stream_prev && !p->hold_stream);
}

// The lagged stream leaves to the pending collision the cells that collision
// writes, and reads the flags of two steps from their copies.
static const char* lag_error(const WaamFields* f, const WaamStepParams* p) {
    if (p->stream_lag && (!p->collide_prev || !f->flags_copy_r || !f->flags_copy_rr ||
                          f->flags_copy_rr == f->flags_copy_r))
        return "stream_lag needs collide_prev and two distinct flag copies";
    if (p->hold_stream && (!p->stream_prev || !p->defer_collide || !f->flags_copy_r ||
                           !f->flags_copy_w || !f->flags_copy_rr))
        return "hold_stream needs stream_prev, defer_collide and three flag copies";
    const bool any = f->pop_cache_src || f->pop_cache_dst || f->pop_cache_stamp;
    const bool all = f->pop_cache_src && f->pop_cache_dst && f->pop_cache_stamp;
    if (any && (!all || f->pop_cache_src == f->pop_cache_dst ||
                (reinterpret_cast<uintptr_t>(f->pop_cache_src) |
                 reinterpret_cast<uintptr_t>(f->pop_cache_dst)) % 16 != 0))
        return "population cache needs two distinct 16-byte aligned buffers and the stamp";
    if ((p->cache_read || p->collide_prev_cache_read) && !all)
        return "cache_read needs the population cache";
    return nullptr;
}

static bool tiles_on(const WaamFields* f) {
    return f->tile_bits != nullptr && f->tile_list != nullptr && f->tile_part != nullptr &&
           tiles_packable(Dims{f->nx, f->ny, f->nz});
}
constexpr int kTileListBlocks = 148 * 6;   // persistent grid of the work-list kernels

static VarPhase var_phase(const WaamStepParams* p) {
    return VarPhase{p->H_sol_t, p->H_liq_t, p->L_rho, p->Ts, p->Tl, p->T_cap};
}

}  // namespace waam

namespace waam {
static int launch_collide_tracers(const WaamFields* f, const WaamStepParams* p, const Dims& d,
                                  Workspace ws, const void* pop_in, void* pop_out,
                                  const float* T_cur, int welding, cudaStream_t s);
}  // namespace waam

extern "C" {

int waam_step_launch_count(const WaamFields* f, const WaamStepParams* p, int stage) {
    if (!p) return 0;
    // the pending stream of the previous step is launched by waam_step_pre;
    // with tiles the classification also runs the surface query
    if (stage == 0) {
        const bool tl = f != nullptr && tiles_on(f);
        return (tl ? (p->welding ? 3 : 1) : (p->welding ? 2 : 1)) + (p->stream_lag ? 1 : 0) +
               (p->stream_prev && !p->hold_stream ? 1 : 0) + (p->collide_prev ? 1 : 0);
    }
    // thermal, [vof], column, [collide], [stream] (tracers counted by the caller)
    int n = 1 + (p->vof ? 1 : 0) + 1 + (p->defer_collide ? 0 : 1) + (p->defer_stream ? 0 : 1);
    if (p->substrate_growth || p->bead_freeze) n += 1;
    return n;
}

int waam_step_pre(const WaamFields* f, const WaamStepParams* p, void* workspace,
                  size_t workspace_bytes, void* stream) {
    if (!fields_ok(f) || !p) return fail(WAAM_ERR_INVALID, "step_pre: bad fields or params");
    if (!tables_fields_ok(f, p)) return fail(WAAM_ERR_INVALID, "step_pre: bad material tables");
    if (const char* le = lag_error(f, p)) return fail(WAAM_ERR_INVALID, le);
    Dims d{f->nx, f->ny, f->nz};
    if (!workspace_ok(workspace, workspace_bytes, d.n()))
        return fail(WAAM_ERR_INVALID, "step_pre: workspace too small or misaligned");
    Workspace ws = Workspace::at(workspace);
    WorkStream W(STREAM(stream), true, 4);
    if (W.err) return W.err;
    const cudaStream_t s = W.s;
    const bool tl = tiles_on(f);
    const int64_t n_tiles = tile_total(d);
    const uint8_t* tile_work = tl ? f->tile_bits + (int64_t)tiles_k(d) * d.nx * d.ny : nullptr;
    const bool s3_work = stream_work(p);
    AuxStream* aux = nullptr;
    if (p->collide_prev || s3_work) {
        int ea = aux_stream(&aux);
        if (ea) return ea;
        // the fork points of the pending collision (ev[8]) and streams (ev[2]):
        // the start of the step, before the work-tile classification is
        // launched (so that its blocks are placed first)
        if (p->collide_prev) cudaEventRecord(aux->ev[8], s);
        if (s3_work) cudaEventRecord(aux->ev[2], s);
    }
    if (tl) {
        // the step's work tiles, from the chunk bits the previous column pass
        // left; the list count was zeroed by that column pass (or here, when
        // the tile history restarts)
        if (!p->tile_skip) cudaMemsetAsync(f->tile_list, 0, sizeof(int32_t), s);
        // one block more than the bands need: the surface query
        const int bands = d.nx * tiles_j(d);
        k_classify_tiles<<<(bands + kClassifyWarps - 1) / kClassifyWarps + 1,
                           32 * kClassifyWarps, 0, s>>>(
            d, f->tile_bits, const_cast<uint8_t*>(tile_work), f->tile_list, p->tile_skip,
            f->tile_part, f->phi, f->flags, f->step_scalars, p->nz_solid);
        int e = check_launch("k_classify_tiles");
        if (e) return e;
    }
    if (p->collide_prev) {
        // the previous step's collision and tracers, beside this step's arc
        // stage (waam_step_main waits for them before its thermal stage)
        int ea = WAAM_OK;
        cudaStreamWaitEvent(aux->s2, aux->ev[8], 0);
        ea = launch_collide_tracers(f, p, d, ws, f->f_dst, f->f_src, f->T, p->collide_prev_welding,
                                    aux->s2);
        if (ea) return ea;
        cudaEventRecord(aux->ev[9], aux->s2);
    }
    if (s3_work) {
        int ea = WAAM_OK;
        cudaStreamWaitEvent(aux->s3, aux->ev[2], 0);
        if (p->stream_lag) {
            // the stream of the step before the previous one, held back by
            // the previous step: beside the previous step's collision, from
            // the buffer that collision reads into the one it writes, leaving
            // alone the cells that collision writes (active in the previous
            // step's flags); its own flags are the older copy
            ea = launch_stream_stored(d, f->f_dst, f->f_src, f->flags_copy_rr, p->f_storage,
                                      aux->s3, f->flags_copy_r);
            if (ea) return ea;
        }
        if (p->stream_prev && !p->hold_stream) {
            // the previous step's stream, after its collision
            if (p->collide_prev) cudaStreamWaitEvent(aux->s3, aux->ev[9], 0);
            // the flags it streams with: the previous step's copy if there is
            // one (then the column pass may rewrite the flags meanwhile)
            const int32_t* sf = f->flags_copy_r ? f->flags_copy_r : f->flags;
            ea = launch_stream_stored(d, f->f_src, f->f_dst, sf, p->f_storage, aux->s3);
            if (ea) return ea;
        }
        // waam_step_main joins them before the column pass (without flag
        // copies) or after it
        cudaEventRecord(aux->ev[3], aux->s3);
    }
    if (!p->welding) {
        if (tl) return WAAM_OK;
        k_surface_arc<<<1, 32, 0, s>>>(d, f->phi, f->flags, f->step_scalars,
                                                    p->nz_solid);
        return check_launch("k_surface_arc");
    }
    ArcParams a = arc_params(p);
    float Qe_dt = p->Q_w * p->eta * p->dt;
    float* shape = reinterpret_cast<float*>(static_cast<char*>(workspace) + ws_shape_offset(d.n()));
    const int tiles = (int)tile_grid(d).x * (int)tile_grid(d).y * d.nx;
    const int blocks = tiles < kTileRedBlocks ? tiles : kTileRedBlocks;
    PhaseParams ph = make_phase(p->cp_rho, p->L_rho, p->Ts, p->Tl, p->T_cap, p->cap_enabled);
    if (tl) {
        k_arc_norm_list<<<blocks, tile_block(), 0, s>>>(
            d, f->flags, f->f_l, a, f->step_scalars, p->arc_k_offset, Qe_dt, p->dx3, ws, shape,
            f->tile_list, f->tile_part, (int)n_tiles);
        int e = check_launch("k_arc_norm_list");
        if (e) return e;
        const int lb = (int)(n_tiles < kTileListBlocks ? n_tiles : kTileListBlocks);
        k_arc_inject_list<<<lb, tile_block(), 0, s>>>(
            d, f->H, f->flags, f->f_l, a, f->step_scalars, p->arc_k_offset, p->cap_enabled, ph,
            p->use_tables ? f->cp_rho_f : nullptr, var_phase(p), shape, f->tile_list,
            (int)n_tiles);
        return check_launch("k_arc_inject_list");
    }
    k_arc_norm_tiles<<<blocks, tile_block(), 0, s>>>(
        d, f->flags, f->f_l, f->phi, p->nz_solid, a, f->step_scalars, p->arc_k_offset, Qe_dt,
        p->dx3, ws, shape);
    int e = check_launch("k_arc_norm_tiles");
    if (e) return e;
    k_arc_inject_tiles<<<tile_grid(d), tile_block(), 0, s>>>(
        d, f->H, f->flags, f->f_l, a, f->step_scalars, p->arc_k_offset, p->cap_enabled, ph,
        p->use_tables ? f->cp_rho_f : nullptr, var_phase(p), shape);
    return check_launch("k_arc_inject_tiles");
}

int waam_step_stream(const WaamFields* f, const WaamStepParams* p, void* stream) {
    if (!fields_ok(f) || !p) return fail(WAAM_ERR_INVALID, "step_stream: bad fields or params");
    if (p->f_storage < kStoreF32 || p->f_storage > kStoreBF16)
        return fail(WAAM_ERR_INVALID, "step_stream: bad f_storage");
    Dims d{f->nx, f->ny, f->nz};
    return launch_stream_stored(d, f->f_src, f->f_dst, f->flags, p->f_storage, STREAM(stream));
}

int waam_step_finish(const WaamFields* f, const WaamStepParams* p, void* workspace,
                     size_t workspace_bytes, void* stream) {
    if (!fields_ok(f) || !p) return fail(WAAM_ERR_INVALID, "step_finish: bad fields or params");
    if (p->f_storage < kStoreF32 || p->f_storage > kStoreBF16)
        return fail(WAAM_ERR_INVALID, "step_finish: bad f_storage");
    Dims d{f->nx, f->ny, f->nz};
    if (!workspace_ok(workspace, workspace_bytes, d.n()))
        return fail(WAAM_ERR_INVALID, "step_finish: workspace too small or misaligned");
    if (const char* le = lag_error(f, p)) return fail(WAAM_ERR_INVALID, le);
    Workspace ws = Workspace::at(workspace);
    cudaStream_t s = STREAM(stream);
    int e = WAAM_OK;
    if (p->stream_lag) {
        // the stream held back by the previous step, then its collision
        e = launch_stream_stored(d, f->f_dst, f->f_src, f->flags_copy_rr, p->f_storage, s,
                                 f->flags_copy_r);
        if (e) return e;
    }
    e = launch_collide_tracers(f, p, d, ws, f->f_dst, f->f_src, f->T, p->collide_prev_welding, s);
    if (e) return e;
    return launch_stream_stored(d, f->f_src, f->f_dst, f->flags, p->f_storage, s);
}

int waam_step_main(const WaamFields* f, const WaamStepParams* p, void* workspace,
                   size_t workspace_bytes, void* stream) {
    return waam_step_main_events(f, p, workspace, workspace_bytes, nullptr, 0, stream);
}

}  // extern "C"

namespace waam {
// Collision (forces in registers, Lorentz J x B when the fields carry J and B),
// J x B on solid cells without VOF, then the tracers, over the active list of
// the workspace: populations pop_in -> pop_out, temperature T_cur.
static int launch_collide_tracers(const WaamFields* f, const WaamStepParams* p, const Dims& d,
                                  Workspace ws, const void* pop_in, void* pop_out,
                                  const float* T_cur, int welding, cudaStream_t s) {
    unsigned* active_count = ws.counter + kActiveShardSlot;
    int* active_list = reinterpret_cast<int*>(ws.field);
    const int64_t shard_cap =
        ((int64_t)d.nx * d.ny + kActiveShards - 1) / kActiveShards * (int64_t)d.nz;
    int e = WAAM_OK;
    CollideArgs cl;
    ForceParams& P = cl.P;
    P.W = weld_force_params(p->gas_shear, p->gs_tau_pa, p->recoil, p->recoil_pa, p->recoil_T_ref,
                            p->P_ref, p->T_boil, p->L_vap, p->R_spec, p->C_acc, p->weld_sigma,
                            p->dt, p->dx, p->rho_phys);
    P.csf = p->csf;
    P.wetting = p->wetting;
    P.welding = welding;
    P.hydro = p->hydro;
    P.gamma_lu = p->gamma_lu;
    P.cos_t = (float)cos((double)p->theta);
    P.sin_t = (float)sin((double)p->theta);
    P.dgamma = p->dgamma_lu;
    P.arc_i = P.arc_j = P.arc_k = 0.0f;  // from the device scalars
    P.p_inv2s2 = 1.0f / (2.0f * p->p_sigma * p->p_sigma + 1e-6f);
    float Fphys = p->pressure / (p->rho_phys * p->dx);
    P.p_Flu = Fphys * (p->dt * p->dt) / p->dx;
    P.g_lu = p->g_lu;
    P.beta = p->beta;
    P.T_ref = p->T_ref;
    P.rho_ref = 1.0f;
    P.F_cap = p->F_cap;
    cl.kind = p->use_tables && p->variable_tau ? 2 : p->collision;
    cl.dgamma_f = p->use_tables ? f->dgamma_f : nullptr;
    cl.tau_f = f->tau_f;
    cl.tape_f = f->tape_f;
    cl.tape_cells = f->tape_cells;
    cl.tape_count = f->tape_count;
    cl.tape_cap = f->tape_cap;
    if (f->tape_f && (!f->tape_cells || !f->tape_count || f->tape_cap <= 0))
        return fail(WAAM_ERR_INVALID, "collide: incomplete collision tape");
    cl.from_buffer = p->forces_from_buffer;
    cl.omega = p->omega;
    cl.omega_b = p->omega_b;
    cl.C_darcy = p->C_darcy;
    cl.u_cap = p->u_cap;
    const bool lorentz = f->lorentz_J[0] != nullptr;
    for (int q = 0; q < 3; ++q) {
        cl.J[q] = f->lorentz_J[q];
        cl.B[q] = f->lorentz_B[q];
        if (lorentz && (!f->lorentz_J[q] || !f->lorentz_B[q]))
            return fail(WAAM_ERR_INVALID, "collide: incomplete Lorentz fields");
    }
    cl.lz_dt = p->dt;
    cl.lz_dx = p->dx;
    cl.lz_rho = p->rho_phys;
    cl.status = f->status;
    cl.rho_lo = p->rho_lo;
    cl.rho_hi = p->rho_hi;
    // the population cache: pop_in is f_src (this step's collision) or f_dst
    // (the previous step's, after the buffer swap); each cache buffer goes
    // with its population buffer
    cl.cache_in = nullptr;
    cl.cache_out = nullptr;
    cl.stamp = nullptr;
    if (f->pop_cache_dst) {
        const bool fwd = pop_in == f->f_src;
        cl.cache_out = fwd ? f->pop_cache_dst : f->pop_cache_src;
        if (fwd ? p->cache_read : p->collide_prev_cache_read)
            cl.cache_in = fwd ? f->pop_cache_src : f->pop_cache_dst;
        cl.stamp = f->pop_cache_stamp;
    }
#define WAAM_COLLIDE(S)                                                                    \
    k_collide_list<S><<<kListBlocks, kListThreads, 0, s>>>(                                \
        d, static_cast<const Pop<S>::T*>(pop_in), static_cast<Pop<S>::T*>(pop_out),              \
        f->rho, f->ux, f->uy, f->uz, f->Fx, f->Fy, f->Fz, f->phi, T_cur, f->f_l, f->flags,        \
        f->step_scalars, active_list, active_count, (int)shard_cap, cl)
    if (p->f_storage == kStoreF16)
        WAAM_COLLIDE(kStoreF16);
    else if (p->f_storage == kStoreBF16)
        WAAM_COLLIDE(kStoreBF16);
    else
        WAAM_COLLIDE(kStoreF32);
#undef WAAM_COLLIDE
    e = check_launch("k_collide_list");
    if (e) return e;
    // With VOF the column pass has set f_l = 0 on every SOLID cell, below the
    // 0.05 the force needs: the pass is only run without VOF.
    if (lorentz && !p->vof) {
        k_lorentz_solid<<<elem_blocks(d.n()), kThreads, 0, s>>>(
            d.n(), f->flags, f->f_l, f->Fx, f->Fy, f->Fz, f->lorentz_J[0],
            f->lorentz_J[1], f->lorentz_J[2], f->lorentz_B[0], f->lorentz_B[1], f->lorentz_B[2],
            p->dt, p->dx, p->rho_phys);
        e = check_launch("k_lorentz_solid");
        if (e) return e;
    }
    // tracers read u, f_l and flags only (they follow the stream in the
    // reference order; nothing of theirs depends on it)
    if (f->tracer_pos && f->tracer_active && f->max_tracers > 0) {
        e = launch_advect_tracers(d, f->tracer_pos, f->tracer_active, f->ux, f->uy, f->uz,
                                  f->f_l, f->flags, p->dx, f->max_tracers, s);
        if (e) return e;
    }
    return WAAM_OK;
}

// stages: bit 0 thermal .. column, bit 1 collide .. tail
static int step_main_impl(const WaamFields* f, const WaamStepParams* p, void* workspace,
                          size_t workspace_bytes, void* const* events, int n_events,
                          void* stream, int stages) {
    if (!fields_ok(f) || !p) return fail(WAAM_ERR_INVALID, "step_main: bad fields or params");
    if (!tables_fields_ok(f, p)) return fail(WAAM_ERR_INVALID, "step_main: bad material tables");
    if (const char* le = lag_error(f, p)) return fail(WAAM_ERR_INVALID, le);
    if (p->f_storage < kStoreF32 || p->f_storage > kStoreBF16)
        return fail(WAAM_ERR_INVALID, "step_main: f_storage must be 0 (f32), 1 (f16) or 2 (bf16)");
    if (events && n_events < kMainEvents)
        return fail(WAAM_ERR_INVALID, "step_main: need 7 events");
    if (p->defer_stream && (p->substrate_growth || p->bead_freeze))
        return fail(WAAM_ERR_INVALID, "step_main: defer_stream needs the remelt/solidify tail off");
    if (p->defer_collide && (!p->defer_stream || p->forces_from_buffer || f->tape_f ||
                             f->lorentz_J[0]))
        return fail(WAAM_ERR_INVALID,
                    "step_main: defer_collide needs defer_stream and no force buffer, tape or "
                    "Lorentz fields");
    for (int q = 0; events && q < kMainEvents; ++q)
        if (!events[q]) return fail(WAAM_ERR_INVALID, "step_main: null event handle");
    auto mark = [&](int i) {
        if (events) cudaEventRecord(reinterpret_cast<cudaEvent_t>(events[i]), STREAM(stream));
    };
    Dims d{f->nx, f->ny, f->nz};
    if (!workspace_ok(workspace, workspace_bytes, d.n()))
        return fail(WAAM_ERR_INVALID, "step_main: workspace too small or misaligned");
    Workspace ws = Workspace::at(workspace);
    unsigned* active_count = ws.counter + kActiveShardSlot;
    int* active_list = reinterpret_cast<int*>(ws.field);
    const int64_t shard_cap =
        ((int64_t)d.nx * d.ny + kActiveShards - 1) / kActiveShards * (int64_t)d.nz;
    if (shard_cap * kActiveShards > d.n() + kFieldSlack || shard_cap > INT32_MAX)
        return fail(WAAM_ERR_INVALID, "step_main: nz too large for the active-cell list");
    const int col_blocks = (int)(((int64_t)d.nx * d.ny * 32 + kThreads - 1) / kThreads);
    // without stage events the stages run on the library's high-priority stream
    WorkStream W(STREAM(stream), events == nullptr, 6);
    if (W.err) return W.err;
    cudaStream_t s = W.s;
    int e = WAAM_OK;

    if (stages & 1) {
        if (p->collide_prev) {
            // the previous step's collision (started by waam_step_pre) writes
            // the velocities the thermal and VOF stages read
            AuxStream* sa = nullptr;
            int ea = aux_stream(&sa);
            if (ea) return ea;
            cudaStreamWaitEvent(s, sa->ev[9], 0);
        }
        ThermalArgs ta;
        ta.ph = make_phase(p->cp_rho, p->L_rho, p->Ts, p->Tl, p->T_cap, p->cap_enabled);
        ta.cpa = p->cp_rho * p->alpha_lu;
        ta.dt_lu = 1.0f;
        ta.inv_dt = 1.0f / (p->dt + 1e-12f);
        ta.heat_loss = p->heat_loss;
        ta.conv = p->conv;
        ta.rad = p->rad;
        ta.T_amb = p->T_amb;
        ta.h_conv = p->h_conv;
        ta.eps_rad = p->eps_rad;
        ta.dt_phys = p->dt;
        ta.dx = p->dx;
        ta.sigma_sb = p->sigma_sb;
        ta.h_floor = p->cp_rho * p->T_amb;
        ta.cache_stamp = f->pop_cache_dst ? f->pop_cache_stamp : nullptr;
        TableArgs tba{};
        if (p->use_tables) {
            tba.vp = var_phase(p);
            tba.tc = TableConsts{p->rho_mat, p->dt, p->dx, p->force_scale_lu, p->marangoni_scale,
                                 p->cp_rho, p->alpha_lu, p->dgamma_lu, p->tau_ref, 1};
            tba.tb = p->tables;
            tba.cp_f = f->cp_rho_f;
            tba.alpha_f = f->alpha_f;
            tba.dg_f = f->dgamma_f;
            tba.tau_f = f->tau_f;
        }
        // Without stage events, VOF advection (reads phi, u, flags; writes phi_tmp)
        // runs on a second stream beside the thermal stage (reads H, T, u, flags;
        // writes the thermal fields and f_l).
        AuxStream* aux = nullptr;
        const bool overlap = events == nullptr;
        if (overlap) {
            int ea = aux_stream(&aux);
            if (ea) return ea;
        }
        auto fork = [&](int q) {
            cudaEventRecord(aux->ev[q], s);
            cudaStreamWaitEvent(aux->s2, aux->ev[q], 0);
        };
        auto join = [&](int q) {
            cudaEventRecord(aux->ev[q], aux->s2);
            cudaStreamWaitEvent(s, aux->ev[q], 0);
        };
        // the work tiles waam_step_pre listed (quiet tiles skipped), or every tile
        const bool tl = tiles_on(f);
        const int n_tiles = (int)tile_total(d);
        const int lb = n_tiles < kTileListBlocks ? n_tiles : kTileListBlocks;
        auto launch_vof = [&](cudaStream_t st) {
            if (tl)
                k_vof_list<<<lb, tile_block(), 0, st>>>(d, f->phi, f->phi_tmp, f->ux, f->uy, f->uz,
                                                        f->flags, f->tile_list, n_tiles);
            else
                k_vof_advect<<<tile_grid(d), tile_block(), 0, st>>>(d, f->phi, f->phi_tmp, f->ux,
                                                                     f->uy, f->uz, f->flags);
            return check_launch("k_vof_advect");
        };
        if (overlap && p->vof) {
            fork(0);
            e = launch_vof(aux->s2);
            if (e) return e;
        }
        mark(0);
        if (tl && p->use_tables)
            k_thermal_list<true><<<lb, tile_block(), 0, s>>>(
                d, f->H, f->H_next, f->T, f->T_next, f->f_l, f->ux, f->uy, f->uz, f->flags, f->T_max,
                f->T_prev, f->dT_dt, active_count, ta, tba, f->status, f->tile_list, n_tiles);
        else if (tl)
            k_thermal_list<false><<<lb, tile_block(), 0, s>>>(
                d, f->H, f->H_next, f->T, f->T_next, f->f_l, f->ux, f->uy, f->uz, f->flags, f->T_max,
                f->T_prev, f->dT_dt, active_count, ta, tba, f->status, f->tile_list, n_tiles);
        else if (p->use_tables)
            k_thermal_fused<true><<<tile_grid(d), tile_block(), 0, s>>>(
                d, f->H, f->H_next, f->T, f->T_next, f->f_l, f->ux, f->uy, f->uz, f->flags, f->T_max,
                f->T_prev, f->dT_dt, active_count, ta, tba, f->status);
        else
            k_thermal_fused<false><<<tile_grid(d), tile_block(), 0, s>>>(
                d, f->H, f->H_next, f->T, f->T_next, f->f_l, f->ux, f->uy, f->uz, f->flags, f->T_max,
                f->T_prev, f->dT_dt, active_count, ta, tba, f->status);
        e = check_launch("k_thermal_fused");
        if (e) return e;
        mark(1);

        if (p->vof) {
            if (overlap) {
                join(1);
            } else {
                e = launch_vof(s);
                if (e) return e;
            }
        }
        mark(2);
        if (stream_work(p) && !f->flags_copy_r) {
            // the previous step's stream (started by waam_step_pre) ends here:
            // the column pass writes the flags it reads
            AuxStream* sa = nullptr;
            int ea = aux_stream(&sa);
            if (ea) return ea;
            cudaStreamWaitEvent(s, sa->ev[3], 0);
        }
        ColumnArgs ca;
        ca.vof = p->vof;
        ca.wetting = p->wetting;
        ca.nz_solid = p->nz_solid;
        ca.cos_t = (float)cos((double)p->theta);
        ca.sin_t = (float)sin((double)p->theta);
        ca.dt_phys = p->dt;
        ca.T800 = p->T800;
        ca.T1100 = p->T1100;
        ca.Ts = p->Ts;
        ca.zero_forces = p->forces_from_buffer ? 0 : 1;
        ca.clear_all = p->clear_forces;
        ca.shard_cap = (int)shard_cap;
        ca.tile_work = tl ? f->tile_bits + (int64_t)tiles_k(d) * d.nx * d.ny : nullptr;
        ca.chunk_bits = tl ? f->tile_bits : nullptr;
        ca.tile_history = p->tile_skip ? 1 : 0;
        ca.tile_list = tl ? f->tile_list : nullptr;
        k_column<<<col_blocks, kThreads, 0, s>>>(d, f->phi_tmp, f->phi, f->flags, f->f_l, f->T_next,
                                                 f->t800, f->t1100, f->tsol, f->Fx, f->Fy, f->Fz,
                                                 active_list, active_count, f->flags_copy_w,
                                                 f->step_scalars, ca);
        e = check_launch("k_column");
        if (e) return e;
        mark(3);
    }

    if (stages & 2) {
        if (stream_work(p) && f->flags_copy_r) {
            // the streams waam_step_pre started end here: the collision writes
            // the populations of the active cells into the buffer they write
            AuxStream* sa = nullptr;
            int ea = aux_stream(&sa);
            if (ea) return ea;
            cudaStreamWaitEvent(s, sa->ev[3], 0);
        }
        if (!p->defer_collide) {
            e = launch_collide_tracers(f, p, d, ws, f->f_src, f->f_dst, f->T_next, p->welding, s);
            if (e) return e;
            mark(4);
            if (!p->defer_stream) {
                e = launch_stream_stored(d, f->f_dst, f->f_src, f->flags, p->f_storage, s);
                if (e) return e;
            }
        }
        mark(5);

        if (p->substrate_growth || p->bead_freeze) {
            TailArgs t;
            t.cp_rho = p->cp_rho;
            t.Ts = p->Ts;
            t.Tl = p->Tl;
            t.L_rho = p->L_rho;
            t.remelt = 1;
            t.trailing = p->welding && p->bead_freeze;
            t.cooled = 1;
            t.dir_x = p->dir_x;
            t.dir_y = p->dir_y;
            t.dir_z = p->dir_z;
            t.lookback = p->lookback;
            t.T_freeze = p->T_freeze;
            t.cp_f = p->use_tables ? f->cp_rho_f : nullptr;
            k_tail<<<tile_grid(d), tile_block(), 0, s>>>(d, f->T_next, f->H_next, f->f_l, f->phi,
                                                          f->flags, f->ux, f->uy, f->uz,
                                                          f->step_scalars, t);
            e = check_launch("k_tail");
        }
        mark(6);
    }
    return e;
}
}  // namespace waam

extern "C" {

int waam_step_main_events(const WaamFields* f, const WaamStepParams* p, void* workspace,
                          size_t workspace_bytes, void* const* events, int n_events,
                          void* stream) {
    return step_main_impl(f, p, workspace, workspace_bytes, events, n_events, stream, 3);
}

int waam_step_main_stage(const WaamFields* f, const WaamStepParams* p, int stage, void* workspace,
                         size_t workspace_bytes, void* const* events, int n_events,
                         void* stream) {
    if (stage != 0 && stage != 1) return fail(WAAM_ERR_INVALID, "step_main_stage: stage 0 or 1");
    return step_main_impl(f, p, workspace, workspace_bytes, events, n_events, stream,
                          1 << stage);
}

}  // extern "C"
