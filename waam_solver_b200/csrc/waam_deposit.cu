// Droplet deposition: kernels.py:278-400 feed_wire_surface and the footprint
// retry loop of solvers/coupled_step.py:126-151.
//
// The reference converts gas cells to metal under a shared reserve-then-commit
// volume budget, so its result depends on the order in which cells are
// visited; this library fixes that order to the serial lexicographic (i, j, k)
// one.  Serially, a gas cell of pass 1 converts when it lies in the footprint,
// budget is left and it has a metal neighbour at its visit: a neighbour that
// was metal before the pass, or one of its predecessors (i-1, j, k),
// (i, j-1, k), (i, j, k-1) that converted earlier in the same pass (the other
// three neighbours have not been visited yet).  Without the budget the set S
// of converted cells is the least solution of
//
//   conv(i,j,k) = E(i,j,k) && (M(i,j,k) || conv(i-1,j,k) || conv(i,j-1,k)
//                                        || conv(i,j,k-1))
//
// (E: gas cell in the footprint, M: metal neighbour before the pass), and the
// budget converts exactly the first m cells of S in visiting order, m being
// the number of float32 additions of cell_vol made while the running volume
// is below the target.  Pass 2 is the same recursion with the wider footprint,
// the cells pass 1 converted as extra seeds (they are metal now, whichever
// side of the cell they sit on) and the remaining budget.  Pass 3 refreshes
// the liquid cells of the wide footprint.
//
// k_deposit_wavefront evaluates this in one CTA: each column (i, j) of the
// search box is a bitmask over k in shared memory, the k recursion is a
// Kogge-Stone prefix inside each 64-bit word, the (i, j) recursion a
// wavefront over the anti-diagonals i + j, and the budget cut an exclusive
// scan of the column popcounts.  Boxes whose bitmasks exceed the shared memory
// of one CTA (search radii beyond ~45 cells) run k_deposit_serial, the same
// semantics cell by cell on one thread.  Both loop over the retry radii on the
// device, so a droplet costs one launch.
#include <cmath>

#include "../../include/waam_b200.h"
#include "waam_common.cuh"
#include "waam_internal.cuh"

namespace waam {

#define STREAM(s) reinterpret_cast<cudaStream_t>(s)

namespace {

typedef unsigned long long u64;

constexpr int kDepThreads = 1024;
// per column word: conv/eligible bitmasks of pass 1 and 2, seed bitmask, prefix
constexpr int kDepWordBytes = 3 * 8 + 4;
constexpr int kDepMaxSmem = 224 * 1024;

struct DepositTries {
    float r[WAAM_DEPOSIT_MAX_TRIES];
    int n;
    double accept;   // stop once the converted volume reaches this (m^3)
};

// Search box and footprint of one attempt (kernels.py:322-333).
struct DepBox {
    int i0, i1, j0, j1, k0, k1;
    float foot2, rd2, drop_cz;
};

__host__ __device__ inline DepBox deposit_box(const Dims& d, float arc_i, float arc_j, float arc_k,
                                              float foot_r, float drop_r) {
    DepBox b;
    const float sr = fmax_(foot_r, drop_r);
    b.i0 = imax(0, (int)(arc_i - sr));
    b.i1 = imin(d.nx, (int)(arc_i + sr) + 1);
    b.j0 = imax(0, (int)(arc_j - sr));
    b.j1 = imin(d.ny, (int)(arc_j + sr) + 1);
    b.k0 = imax(0, (int)(arc_k - 1.0f));
    const float k_span = fmax_(drop_r + 3.0f, 4.0f);
    b.k1 = imin(d.nz, (int)(arc_k + k_span) + 1);
    b.drop_cz = arc_k + drop_r + 0.5f;
    b.rd2 = drop_r * drop_r;
    b.foot2 = sr * sr;
    return b;
}

struct DepFields {
    void* f_src;      // populations, elements per DepConsts::storage
    int32_t* flags;
    float* f_l;
    float* phi;
    float* H;
    float* T;
    float* rho;
};

struct DepConsts {
    float arc_i, arc_j, arc_k, drop_r, target_vol, T_drop, hdrop, rho0, cell_vol;
    int storage;   // PopStorage of f_src
};

// kernels.py:255-275 _has_metal_neighbor: a 6-neighbour in the grid that is
// FLUID or SOLID, or whose phi > 0.35 or f_l > 0.2.  The pointers are plain
// (not const __restrict__): the same kernel writes these fields, so the loads
// must not take the non-coherent path.
__device__ bool has_metal_nb(const Dims& d, const DepFields& F, int i, int j, int k) {
    const int sx = d.ny * d.nz, sy = d.nz;
    const int c = d.idx(i, j, k);
    int nb[6];
    bool ok[6];
    ok[0] = i > 0;           nb[0] = c - sx;
    ok[1] = i + 1 < d.nx;    nb[1] = c + sx;
    ok[2] = j > 0;           nb[2] = c - sy;
    ok[3] = j + 1 < d.ny;    nb[3] = c + sy;
    ok[4] = k > 0;           nb[4] = c - 1;
    ok[5] = k + 1 < d.nz;    nb[5] = c + 1;
    int fl[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) fl[m] = ok[m] ? F.flags[nb[m]] : GAS;
#pragma unroll
    for (int m = 0; m < 6; ++m)
        if (ok[m] && (fl[m] == FLUID || fl[m] == SOLID)) return true;
#pragma unroll
    for (int m = 0; m < 6; ++m)
        if (ok[m] && (F.phi[nb[m]] > 0.35f || F.f_l[nb[m]] > 0.2f)) return true;
    return false;
}

__device__ __forceinline__ void write_liquid(const DepFields& F, const DepConsts& K, size_t n,
                                             int c) {
    F.T[c] = K.T_drop;
    F.H[c] = K.hdrop;
    F.rho[c] = K.rho0;
#pragma unroll
    for (int q = 0; q < 19; ++q) pop_store(F.f_src, q * n + c, q, wq(q) * K.rho0, K.storage);
}

// Bits of e reachable from a bit of g by walking up (towards larger k) through
// consecutive bits of e; the bits of g outside e are ignored.
__device__ __forceinline__ u64 fill_up(u64 g, u64 e) {
    u64 p = e;
    g &= e;
    g |= p & (g << 1);
    p &= p << 1;
    g |= p & (g << 2);
    p &= p << 2;
    g |= p & (g << 4);
    p &= p << 4;
    g |= p & (g << 8);
    p &= p << 8;
    g |= p & (g << 16);
    p &= p << 16;
    g |= p & (g << 32);
    return g;
}

// One column of the wavefront: A holds E for this column and conv for the
// columns (i-1, j) and (i, j-1); S holds the seeds.  Writes conv in place.
__device__ __forceinline__ void wavefront_column(u64* A, const u64* S, int ci, int cj, int nj,
                                                 int nw) {
    const int col = ci * nj + cj;
    u64 carry = 0;
    for (int w = 0; w < nw; ++w) {
        const int x = col * nw + w;
        u64 a = S[x] | carry;
        if (ci > 0) a |= A[x - nj * nw];
        if (cj > 0) a |= A[x - nw];
        const u64 g = fill_up(a, A[x]);
        A[x] = g;
        carry = g >> 63;
    }
}

// conv over the whole box, diagonal by diagonal (column (i, j) depends only on
// diagonal i + j - 1).  Called by all threads; ends with a block barrier.
__device__ void wavefront(u64* A, const u64* S, int ni, int nj, int nw) {
    const int tid = threadIdx.x;
    const int ndiag = ni + nj - 1;
    if (imin(ni, nj) <= 32) {
        // every diagonal fits one warp: warp 0 walks them with warp barriers
        if (tid < 32) {
            for (int s = 0; s < ndiag; ++s) {
                const int lo = imax(0, s - (nj - 1)), hi = imin(s, ni - 1);
                const int ci = lo + tid;
                if (ci <= hi) wavefront_column(A, S, ci, s - ci, nj, nw);
                __syncwarp();
            }
        }
    } else {
        for (int s = 0; s < ndiag; ++s) {
            const int lo = imax(0, s - (nj - 1)), hi = imin(s, ni - 1);
            for (int ci = lo + tid; ci <= hi; ci += blockDim.x)
                wavefront_column(A, S, ci, s - ci, nj, nw);
            __syncthreads();
        }
    }
    __syncthreads();
}

// Exclusive scan of the popcounts of A[0, ncw) into P in visiting order (the
// column words are stored in that order); returns the total to every thread.
__device__ int popc_scan(const u64* A, int* P, int ncw, int* s_warp, int* s_total) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int per = (ncw + nt - 1) / nt;
    const int w0 = imin(ncw, tid * per), w1 = imin(ncw, w0 + per);
    int local = 0;
    for (int w = w0; w < w1; ++w) local += __popcll(A[w]);
    int incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const int v = lane < (nt >> 5) ? s_warp[lane] : 0;
        int inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += u;
        }
        s_warp[lane] = inc - v;
        if (lane == 31) *s_total = inc;
    }
    __syncthreads();
    int run = s_warp[warp] + incl - local;
    for (int w = w0; w < w1; ++w) {
        P[w] = run;
        run += __popcll(A[w]);
    }
    const int total = *s_total;
    __syncthreads();
    return total;
}

// Keep the first m set bits of A in visiting order.
__device__ void truncate_to(u64* A, const int* P, int ncw, int m) {
    for (int w = threadIdx.x; w < ncw; w += blockDim.x) {
        const int p = P[w];
        u64 x = A[w];
        if (p >= m) {
            A[w] = 0;
        } else if (p + __popcll(x) > m) {
            u64 out = 0;
            for (int q = p; q < m; ++q) {
                const u64 low = x & (~x + 1);
                out |= low;
                x ^= low;
            }
            A[w] = out;
        }
    }
}

// Budget of one pass (thread 0): convert while the running volume is below
// the target, one float32 addition per converted cell, at most `avail` cells.
__device__ int spend_budget(int avail, float target, float cell_vol, float* s_vol, float* s_real) {
    float v = *s_vol, r = *s_real;
    int m = 0;
    while (m < avail && !(v >= target)) {
        v = v + cell_vol;
        r = r + cell_vol;
        ++m;
    }
    *s_vol = v;
    *s_real = r;
    return m;
}

__device__ __forceinline__ void box_cell(const DepBox& b, int nj, int nk, int e, int& col, int& kk,
                                         int& i, int& j, int& k) {
    col = e / nk;
    kk = e - col * nk;
    const int ci = col / nj;
    i = b.i0 + ci;
    j = b.j0 + (col - ci * nj);
    k = b.k0 + kk;
}

__global__ void __launch_bounds__(kDepThreads)
    k_deposit_wavefront(Dims d, DepFields F, DepConsts K, DepositTries tries, float* vol_acc,
                        float* real_acc, int smem_words) {
    extern __shared__ u64 s_bits[];
    __shared__ int s_warp[32];
    __shared__ int s_total, s_m, s_go;
    __shared__ float s_vol, s_real;
    const int tid = threadIdx.x, nt = blockDim.x;
    const size_t n = (size_t)d.n();
    if (tid == 0) {
        s_vol = *vol_acc;
        s_real = *real_acc;
    }
    for (int t = 0; t < tries.n; ++t) {
        __syncthreads();
        const DepBox b = deposit_box(d, K.arc_i, K.arc_j, K.arc_k, tries.r[t], K.drop_r);
        const int ni = b.i1 - b.i0, nj = b.j1 - b.j0, nk = b.k1 - b.k0;
        // the host sized the shared bitmasks from the same boxes; the word
        // check only keeps an inconsistent launch inside its allocation
        if (ni > 0 && nj > 0 && nk > 0 && ni * nj * ((nk + 63) >> 6) <= smem_words) {
            const int nw = (nk + 63) >> 6;
            const int ncw = ni * nj * nw;
            const int ncell = ni * nj * nk;
            u64* A1 = s_bits;        // E of pass 1, then its conv
            u64* A2 = A1 + ncw;      // E of pass 2, then its conv
            u64* M = A2 + ncw;       // metal neighbour before the pass (+ pass-1 cells)
            int* P = reinterpret_cast<int*>(M + ncw);
            for (int x = tid; x < ncw; x += nt) A1[x] = A2[x] = M[x] = 0;
            __syncthreads();
            // eligibility and seeds from the state at the start of the attempt
            for (int e = tid; e < ncell; e += nt) {
                int col, kk, i, j, k;
                box_cell(b, nj, nk, e, col, kk, i, j, k);
                const int c = d.idx(i, j, k);
                if (F.flags[c] != GAS) continue;
                const float di = (float)i - K.arc_i, dj = (float)j - K.arc_j;
                const float rij2 = di * di + dj * dj;
                const float dk = (float)k - b.drop_cz;
                const float r2 = di * di + dj * dj + dk * dk;
                const bool in1 = !(rij2 > b.foot2 && r2 > b.rd2);
                const bool in2 = !(rij2 > b.foot2 * 1.44f);
                if (!in1 && !in2) continue;
                const u64 bit = 1ull << (kk & 63);
                const int x = col * nw + (kk >> 6);
                if (in1) atomicOr(&A1[x], bit);
                if (in2) atomicOr(&A2[x], bit);
                if (has_metal_nb(d, F, i, j, k)) atomicOr(&M[x], bit);
            }
            __syncthreads();
            // ---- pass 1 ----
            wavefront(A1, M, ni, nj, nw);
            int total = popc_scan(A1, P, ncw, s_warp, &s_total);
            if (tid == 0) {
                const int m = spend_budget(total, K.target_vol, K.cell_vol, &s_vol, &s_real);
                s_m = m;
                s_go = !(s_vol >= K.target_vol);
            }
            __syncthreads();
            truncate_to(A1, P, ncw, s_m);
            __syncthreads();
            for (int e = tid; e < ncell; e += nt) {
                int col, kk, i, j, k;
                box_cell(b, nj, nk, e, col, kk, i, j, k);
                if ((A1[col * nw + (kk >> 6)] >> (kk & 63)) & 1ull) {
                    const int c = d.idx(i, j, k);
                    F.flags[c] = FLUID;
                    F.f_l[c] = 1.0f;
                    F.phi[c] = 1.0f;
                    write_liquid(F, K, n, c);
                }
            }
            // ---- pass 2 (budget left): pass-1 cells are metal, no longer gas ----
            if (s_go) {
                for (int x = tid; x < ncw; x += nt) {
                    const int col = x / nw, w = x - col * nw;
                    const int ci = col / nj, cj = col - ci * nj;
                    const u64 c1 = A1[x];
                    u64 nbm = (c1 << 1) | (c1 >> 1);
                    if (w > 0) nbm |= A1[x - 1] >> 63;
                    if (w + 1 < nw) nbm |= A1[x + 1] << 63;
                    if (ci > 0) nbm |= A1[x - nj * nw];
                    if (ci + 1 < ni) nbm |= A1[x + nj * nw];
                    if (cj > 0) nbm |= A1[x - nw];
                    if (cj + 1 < nj) nbm |= A1[x + nw];
                    A2[x] &= ~c1;
                    M[x] |= nbm;
                }
                __syncthreads();
                wavefront(A2, M, ni, nj, nw);
                total = popc_scan(A2, P, ncw, s_warp, &s_total);
                if (tid == 0) s_m = spend_budget(total, K.target_vol, K.cell_vol, &s_vol, &s_real);
                __syncthreads();
                truncate_to(A2, P, ncw, s_m);
                __syncthreads();
                for (int e = tid; e < ncell; e += nt) {
                    int col, kk, i, j, k;
                    box_cell(b, nj, nk, e, col, kk, i, j, k);
                    if ((A2[col * nw + (kk >> 6)] >> (kk & 63)) & 1ull) {
                        const int c = d.idx(i, j, k);
                        F.flags[c] = FLUID;
                        F.f_l[c] = 1.0f;
                        F.phi[c] = 1.0f;
                        write_liquid(F, K, n, c);
                    }
                }
            }
            __syncthreads();
            // ---- pass 3: thermal top-up of the liquid footprint (no budget) ----
            const float foot_wide = b.foot2 * 1.44f;
            for (int e = tid; e < ncell; e += nt) {
                int col, kk, i, j, k;
                box_cell(b, nj, nk, e, col, kk, i, j, k);
                const int c = d.idx(i, j, k);
                if (F.flags[c] != FLUID || F.f_l[c] < 0.45f) continue;
                const float di = (float)i - K.arc_i, dj = (float)j - K.arc_j;
                if (di * di + dj * dj > foot_wide) continue;
                write_liquid(F, K, n, c);
            }
        }
        __syncthreads();
        if (tid == 0) {
            // the retry resumes the budget from the volume converted so far
            s_go = (t + 1 < tries.n) && !((double)s_real >= tries.accept);
            if (s_go) s_vol = s_real;
        }
        __syncthreads();
        if (!s_go) break;
    }
    if (tid == 0) {
        *vol_acc = s_vol;
        *real_acc = s_real;
    }
}

// The same semantics visited cell by cell on one thread, for search boxes
// whose bitmasks do not fit in shared memory.
__global__ void k_deposit_serial(Dims d, DepFields F, DepConsts K, DepositTries tries,
                                 float* vol_acc, float* real_acc) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const size_t n = (size_t)d.n();
    float vol = *vol_acc, real = *real_acc;
    for (int t = 0; t < tries.n; ++t) {
        if (t > 0) {
            if ((double)real >= tries.accept) break;
            vol = real;
        }
        const DepBox b = deposit_box(d, K.arc_i, K.arc_j, K.arc_k, tries.r[t], K.drop_r);
        for (int pass = 0; pass < 2; ++pass)
            for (int i = b.i0; i < b.i1; ++i)
                for (int j = b.j0; j < b.j1; ++j)
                    for (int k = b.k0; k < b.k1; ++k) {
                        if (vol >= K.target_vol) continue;
                        const int c = d.idx(i, j, k);
                        if (F.flags[c] != GAS) continue;
                        if (!has_metal_nb(d, F, i, j, k)) continue;
                        const float di = (float)i - K.arc_i, dj = (float)j - K.arc_j;
                        const float rij2 = di * di + dj * dj;
                        if (pass == 0) {
                            const float dk = (float)k - b.drop_cz;
                            const float r2 = di * di + dj * dj + dk * dk;
                            if (rij2 > b.foot2 && r2 > b.rd2) continue;
                        } else if (rij2 > b.foot2 * 1.44f) {
                            continue;
                        }
                        vol = vol + K.cell_vol;
                        F.flags[c] = FLUID;
                        F.f_l[c] = 1.0f;
                        F.phi[c] = 1.0f;
                        write_liquid(F, K, n, c);
                        real = real + K.cell_vol;
                    }
        for (int i = b.i0; i < b.i1; ++i)
            for (int j = b.j0; j < b.j1; ++j)
                for (int k = b.k0; k < b.k1; ++k) {
                    const int c = d.idx(i, j, k);
                    if (F.flags[c] != FLUID || F.f_l[c] < 0.45f) continue;
                    const float di = (float)i - K.arc_i, dj = (float)j - K.arc_j;
                    if (di * di + dj * dj > b.foot2 * 1.44f) continue;
                    write_liquid(F, K, n, c);
                }
    }
    *vol_acc = vol;
    *real_acc = real;
}

}  // namespace

int launch_deposit(Dims d, void* f_src, int f_storage, int32_t* flags, float* f_l, float* phi,
                   float* H, float* T, float* rho, float arc_i, float arc_j, float arc_k,
                   const float* foot_radii, int n_tries, double accept_volume, float drop_r,
                   float target_vol, float T_drop, float cp_rho, float L_rho, float rho0,
                   float* vol_acc, float* real_acc, float cell_vol, void* stream) {
    if (f_storage < kStoreF32 || f_storage > kStoreBF16)
        return fail(WAAM_ERR_INVALID, "deposit: f_storage must be 0, 1 or 2");
    if (n_tries < 1 || n_tries > WAAM_DEPOSIT_MAX_TRIES || !foot_radii)
        return fail(WAAM_ERR_INVALID, "deposit: footprint radii missing or too many tries");
    // the search box is cast to int: keep every coordinate well inside int range
    auto sane = [](float v) { return std::isfinite(v) && std::fabs(v) < 1.0e6f; };
    if (!sane(arc_i) || !sane(arc_j) || !sane(arc_k) || !sane(drop_r))
        return fail(WAAM_ERR_INVALID, "deposit: arc position or droplet radius not finite/sane");
    for (int t = 0; t < n_tries; ++t)
        if (!sane(foot_radii[t]))
            return fail(WAAM_ERR_INVALID, "deposit: footprint radius not finite/sane");
    DepositTries tries;
    for (int t = 0; t < n_tries; ++t) tries.r[t] = foot_radii[t];
    for (int t = n_tries; t < WAAM_DEPOSIT_MAX_TRIES; ++t) tries.r[t] = 0.0f;
    tries.n = n_tries;
    tries.accept = accept_volume;
    // the largest search box of the attempts sizes the shared bitmasks
    size_t words = 0;
    for (int t = 0; t < n_tries; ++t) {
        const DepBox b = deposit_box(d, arc_i, arc_j, arc_k, tries.r[t], drop_r);
        const int64_t ni = b.i1 - b.i0, nj = b.j1 - b.j0, nk = b.k1 - b.k0;
        if (ni > 0 && nj > 0 && nk > 0) {
            const size_t w = (size_t)(ni * nj) * (size_t)((nk + 63) / 64);
            words = w > words ? w : words;
        }
    }
    const DepFields F{f_src, flags, f_l, phi, H, T, rho};
    const DepConsts K{arc_i, arc_j, arc_k, drop_r, target_vol, T_drop, cp_rho * T_drop + L_rho,
                      rho0, cell_vol, f_storage};
    const size_t smem = words * kDepWordBytes;
    if (smem <= (size_t)kDepMaxSmem) {
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(
                k_deposit_wavefront, cudaFuncAttributeMaxDynamicSharedMemorySize, kDepMaxSmem);
            if (e != cudaSuccess) return fail(WAAM_ERR_CUDA, cudaGetErrorString(e));
        }
        k_deposit_wavefront<<<1, kDepThreads, smem, STREAM(stream)>>>(d, F, K, tries, vol_acc,
                                                                      real_acc, (int)words);
        return check_launch("k_deposit_wavefront");
    }
    k_deposit_serial<<<1, 32, 0, STREAM(stream)>>>(d, F, K, tries, vol_acc, real_acc);
    return check_launch("k_deposit_serial");
}

}  // namespace waam
