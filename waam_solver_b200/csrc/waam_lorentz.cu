// Electromagnetic (Lorentz) force of the welding current: kernels.py:1236-1513,
// driven by physics/weld_forces.py:196-281 solve_lorentz.
//
//   sigma map -> Gaussian current source normalised to I -> damped Jacobi
//   solve of div(sigma grad phi_e) = -source (the substrate below nz_solid
//   grounded, gas insulating) -> J = -sigma grad phi_e -> axial current binned
//   by radius per z slab, prefix-summed -> B_theta = mu0 I_enc / (2 pi r)
//   -> F += f_l (J x B) dt^2 / (rho dx).
//
// The Jacobi sweep optionally accumulates the L1 change and the L1 norm of its
// input (elec_l1_diff, kernels.py:1387-1398) in the same pass, so the host's
// convergence check every ten sweeps costs no extra grid read.  Grid sums are
// accumulated in double in a fixed block order (the reference's float atomics
// have no fixed order); the radial bins use double atomics and are rounded to
// float before the float prefix sum, as the oracle does.
#include <cmath>

#include "../../include/waam_b200.h"
#include "waam_common.cuh"
#include "waam_internal.cuh"

namespace waam {

#define STREAM(s) reinterpret_cast<cudaStream_t>(s)

namespace {

constexpr int kRedGridMax = kWsMaxPartials / 2;   // two sums share the partials
constexpr int kMaxBins = 1024;
constexpr int kOpScalarSourceScale = 16;          // ws.scalars slot of the source scale

// k slab of the arc current source (kernels.py:1261-1284): cells outside
// [k_min, k_max] get 0.  The same float arithmetic on host and device.
__host__ __device__ __forceinline__ void source_slab(float arc_k, float sigma_cells, int nz,
                                                     int& k_min, int& k_max) {
    k_max = imin(nz, (int)(arc_k + sigma_cells * 4.0f) + 1);
    k_min = imax(0, (int)(arc_k - sigma_cells));
}

// Reduction tiles: the 32 x 8 (k, j) tiles with loops over the tiles and i,
// so the grid stays at <= kRedGridMax blocks (one partial per block).
inline dim3 red_tile_grid(const Dims& d) {
    int gx = imin((d.nz + kTileK - 1) / kTileK, 16);
    int gy = imin((d.ny + kTileJ - 1) / kTileJ, 16);
    int gz = imax(1, imin(d.nx, kRedGridMax / (gx * gy)));
    return dim3(gx, gy, gz);
}

__device__ __forceinline__ double2 block_sum2(double a, double b) {
    __shared__ double sh[2][kTileK * kTileJ / 32];
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
    }
    const int t = threadIdx.y * blockDim.x + threadIdx.x;
    const int lane = t & 31, wid = t >> 5;
    if (lane == 0) {
        sh[0][wid] = a;
        sh[1][wid] = b;
    }
    __syncthreads();
    double2 r = make_double2(0.0, 0.0);
    if (t == 0)
        for (int w = 0; w < kTileK * kTileJ / 32; ++w) {
            r.x += sh[0][w];
            r.y += sh[1][w];
        }
    __syncthreads();
    return r;   // valid in thread 0
}

// Last-block combine of two per-block sums: every thread of the last block
// adds a fixed strided subset of the partials in order, then the fixed tree
// of block_sum2 (the same order on every run).  Returns true in the thread
// that holds the totals.  Blocks of kTileK x kTileJ threads.
__device__ bool finish_sum2(Workspace ws, double2 part, double2& total) {
    __shared__ bool last;
    const int t = threadIdx.y * blockDim.x + threadIdx.x;
    const unsigned nb = gridDim.x * gridDim.y * gridDim.z;
    const unsigned b = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
    if (t == 0) {
        ws.partials[b] = part.x;
        ws.partials[nb + b] = part.y;
        __threadfence();
        unsigned prev = atomicAdd(ws.counter, 1u);
        last = prev == nb - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double x = 0.0, y = 0.0;
    for (unsigned q = t; q < nb; q += kTileK * kTileJ) {
        x += ((volatile double*)ws.partials)[q];
        y += ((volatile double*)ws.partials)[nb + q];
    }
    const double2 r = block_sum2(x, y);
    if (t != 0) return false;
    total = r;
    *ws.counter = 0u;
    return true;
}

// kernels.py:1237-1251
__global__ void k_elec_sigma(float* sigma, const float* f_l, const int32_t* flags, int64_t n,
                             float s_liq, float s_sol) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        int fl = flags[c];
        sigma[c] = fl == GAS ? 1e-8f : (f_l[c] > 0.55f ? s_liq : s_sol);
    }
}

// The arc source value of cell (i, j, k) (kernels.py:1261-1284).
__device__ __forceinline__ float elec_source_value(int i, int j, int k, float arc_i, float arc_j,
                                                  float arc_k, float inv2s2, float current,
                                                  float vol_eps, int k_min, int k_max) {
    if (k < k_min || k > k_max) return 0.0f;
    float di = (float)i - arc_i, dj = (float)j - arc_j, dk = (float)k - arc_k;
    float r2 = di * di + dj * dj + 0.25f * dk * dk;
    return current * waam_expf(-r2 * inv2s2) / vol_eps;
}

// kernels.py:1255-1284 (clear + inject in one pass)
__global__ void k_elec_source(Dims d, float* src, float arc_i, float arc_j, float arc_k,
                              float inv2s2, float current, float vol_eps, int k_min, int k_max) {
    int i, j, k, c;
    if (!tile_cell(d, i, j, k, c)) return;
    src[c] = elec_source_value(i, j, k, arc_i, arc_j, arc_k, inv2s2, current, vol_eps, k_min,
                               k_max);
}

// kernels.py:1288-1301, pass 1: sum(source * cell_vol) -> scale in ws scalars
__global__ void k_elec_source_sum(const float* src, int64_t n, float cell_vol, float current,
                                  Workspace ws) {
    double part = 0.0;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x)
        part += (double)(src[c] * cell_vol);
    __shared__ double sh[kThreads / 32];
    for (int o = 16; o > 0; o >>= 1) part += __shfl_down_sync(0xffffffffu, part, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = part;
    __syncthreads();
    __shared__ bool last;
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) t += sh[w];
        ws.partials[blockIdx.x] = t;
        __threadfence();
        last = atomicAdd(ws.counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double t = 0.0;
    for (unsigned b = 0; b < gridDim.x; ++b) t += ((volatile double*)ws.partials)[b];
    float total = (float)t;
    ws.scalars[kOpScalarSourceScale] = current / fmax_(total, 1e-12f);
    *ws.counter = 0u;
}

// Clear + inject + normalise in two passes that read nothing: pass 1 sums
// value * cell_vol over the slab k_min..k_max (every other cell is 0) in
// double, fixed order; pass 2 writes value * scale everywhere, the float the
// reference's in-place scaling leaves.
__global__ void __launch_bounds__(kTileK* kTileJ)
    k_elec_source_fused_sum(Dims d, float arc_i, float arc_j, float arc_k, const float* arc_k_dev,
                            float sigma_cells, float inv2s2, float current, float vol_eps,
                            float cell_vol, float target, Workspace ws) {
    if (arc_k_dev) arc_k = *arc_k_dev;
    int k_min, k_max;
    source_slab(arc_k, sigma_cells, d.nz, k_min, k_max);
    double part = 0.0;
    const int ks = imax(k_min, 0), ke = imin(k_max, d.nz - 1);
    for (int i = blockIdx.z; i < d.nx; i += gridDim.z)
        for (int jt = blockIdx.y; jt * kTileJ < d.ny; jt += gridDim.y)
            for (int kt = blockIdx.x; ks + kt * kTileK <= ke; kt += gridDim.x) {
                const int k = ks + kt * kTileK + threadIdx.x, j = jt * kTileJ + threadIdx.y;
                if (k > ke || j >= d.ny) continue;
                const float v = elec_source_value(i, j, k, arc_i, arc_j, arc_k, inv2s2, current,
                                                  vol_eps, k_min, k_max);
                part += (double)(v * cell_vol);
            }
    double2 tot;
    if (finish_sum2(ws, block_sum2(part, 0.0), tot)) {
        const float total = (float)tot.x;
        ws.scalars[kOpScalarSourceScale] = target / fmax_(total, 1e-12f);
    }
}

__global__ void k_elec_source_fused_write(Dims d, float* src, float arc_i, float arc_j,
                                          float arc_k, const float* arc_k_dev, float sigma_cells,
                                          float inv2s2, float current, float vol_eps,
                                          Workspace ws) {
    int i, j, k, c;
    if (!tile_cell(d, i, j, k, c)) return;
    if (arc_k_dev) arc_k = *arc_k_dev;
    int k_min, k_max;
    source_slab(arc_k, sigma_cells, d.nz, k_min, k_max);
    const float s = ws.scalars[kOpScalarSourceScale];
    const float v = elec_source_value(i, j, k, arc_i, arc_j, arc_k, inv2s2, current, vol_eps,
                                      k_min, k_max);
    src[c] = v * s;
}

// kernels.py:1288-1301, pass 2
__global__ void k_elec_source_scale(float* src, int64_t n, Workspace ws) {
    const float s = ws.scalars[kOpScalarSourceScale];
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x)
        src[c] *= s;
}

// kernels.py:1315-1355 elec_jacobi_step (+ kernels.py:1387-1398 elec_l1_diff
// of (phi_out, phi_in) when L1 is set).
template <bool L1>
__global__ void __launch_bounds__(kTileK* kTileJ)
    k_elec_jacobi(Dims d, const float* __restrict__ phi_in, float* __restrict__ phi_out,
                  const float* __restrict__ sigma, const float* __restrict__ src,
                  const int32_t* __restrict__ flags, float dx, float omega_j, int nz_solid,
                  float* diff_out, float* norm_out, Workspace ws) {
    const float eps = 1e-12f;
    const int sx = d.ny * d.nz, sy = d.nz;
    double dsum = 0.0, nsum = 0.0;
    for (int i = blockIdx.z; i < d.nx; i += gridDim.z)
        for (int jt = blockIdx.y; jt * kTileJ < d.ny; jt += gridDim.y)
            for (int kt = blockIdx.x; kt * kTileK < d.nz; kt += gridDim.x) {
                const int k = kt * kTileK + threadIdx.x, j = jt * kTileJ + threadIdx.y;
                if (k >= d.nz || j >= d.ny) continue;
                const int c = (i * d.ny + j) * d.nz + k;
                const int fl = flags[c];
                const float pin = phi_in[c];
                float out;
                if (fl == GAS || (k <= nz_solid && fl == SOLID)) {
                    out = 0.0f;
                } else {
                    const int ip = c + (i + 1 < d.nx ? sx : 0), im = c - (i > 0 ? sx : 0);
                    const int jp = c + (j + 1 < d.ny ? sy : 0), jm = c - (j > 0 ? sy : 0);
                    const int kp = c + (k + 1 < d.nz ? 1 : 0), km = c - (k > 0 ? 1 : 0);
                    const float sp = sigma[ip], sm = sigma[im], sn = sigma[jp], ss = sigma[jm];
                    const float st = sigma[kp], sb = sigma[km];
                    const float denom = sp + sm + sn + ss + st + sb + eps;
                    const float nb = sp * phi_in[ip] + sm * phi_in[im] + sn * phi_in[jp] +
                                     ss * phi_in[jm] + st * phi_in[kp] + sb * phi_in[km];
                    const float pn = (nb + src[c] * dx * dx) / denom;
                    out = (1.0f - omega_j) * pin + omega_j * pn;
                }
                phi_out[c] = out;
                if (L1) {
                    dsum += (double)fabsf(out - pin);
                    nsum += (double)fabsf(pin);
                }
            }
    if (L1) {
        double2 part = block_sum2(dsum, nsum);
        double2 tot;
        if (finish_sum2(ws, part, tot)) {
            *diff_out = (float)tot.x;
            *norm_out = (float)tot.y;
        }
    }
}

// The sweep of the fused solve: the same arithmetic as k_elec_jacobi, with
// the fixed cells (GAS, and SOLID at k <= nz_solid) read from a byte mask
// built with sigma, and the source read only inside its k slab (it is 0
// elsewhere).  A tile grid (one cell per thread) for the plain sweeps; the
// L1 sweep keeps the fixed reduction grid.
template <bool L1>
__global__ void __launch_bounds__(kTileK* kTileJ)
    k_elec_jacobi_m(Dims d, const float* __restrict__ phi_in, float* __restrict__ phi_out,
                    const float* __restrict__ sigma, const float* __restrict__ src,
                    const uint8_t* __restrict__ fixed, float dx, float omega_j, int k_src_lo,
                    int k_src_hi, float* diff_out, float* norm_out, Workspace ws) {
    const float eps = 1e-12f;
    const int sx = d.ny * d.nz, sy = d.nz;
    double dsum = 0.0, nsum = 0.0;
    const int i_step = L1 ? gridDim.z : d.nx, j_step = L1 ? gridDim.y : d.ny,
              k_step = L1 ? gridDim.x : d.nz;
    for (int i = blockIdx.z; i < d.nx; i += i_step)
        for (int jt = blockIdx.y; jt * kTileJ < d.ny; jt += j_step)
            for (int kt = blockIdx.x; kt * kTileK < d.nz; kt += k_step) {
                const int k = kt * kTileK + threadIdx.x, j = jt * kTileJ + threadIdx.y;
                if (k >= d.nz || j >= d.ny) continue;
                const int c = (i * d.ny + j) * d.nz + k;
                const float pin = phi_in[c];
                float out;
                if (fixed[c]) {
                    out = 0.0f;
                } else {
                    const int ip = c + (i + 1 < d.nx ? sx : 0), im = c - (i > 0 ? sx : 0);
                    const int jp = c + (j + 1 < d.ny ? sy : 0), jm = c - (j > 0 ? sy : 0);
                    const int kp = c + (k + 1 < d.nz ? 1 : 0), km = c - (k > 0 ? 1 : 0);
                    const float sp = sigma[ip], sm = sigma[im], sn = sigma[jp], ss = sigma[jm];
                    const float st = sigma[kp], sb = sigma[km];
                    const float sc = (k >= k_src_lo && k <= k_src_hi) ? src[c] : 0.0f;
                    const float denom = sp + sm + sn + ss + st + sb + eps;
                    const float nb = sp * phi_in[ip] + sm * phi_in[im] + sn * phi_in[jp] +
                                     ss * phi_in[jm] + st * phi_in[kp] + sb * phi_in[km];
                    const float pn = (nb + sc * dx * dx) / denom;
                    out = (1.0f - omega_j) * pin + omega_j * pn;
                }
                phi_out[c] = out;
                if (L1) {
                    dsum += (double)fabsf(out - pin);
                    nsum += (double)fabsf(pin);
                }
            }
    if (L1) {
        double2 part = block_sum2(dsum, nsum);
        double2 tot;
        if (finish_sum2(ws, part, tot)) {
            *diff_out = (float)tot.x;
            *norm_out = (float)tot.y;
        }
    }
}

// One cell of the masked sweep from its neighbour values, in the reference's
// expression order (kernels.py:1315-1355).
__device__ __forceinline__ float jacobi_cell(float pin, float sp, float sm, float sn, float ss,
                                            float st, float sb, float pp, float pm, float pn_,
                                            float ps, float pt, float pb, float sc, float dx,
                                            float omega_j) {
    const float eps = 1e-12f;
    const float denom = sp + sm + sn + ss + st + sb + eps;
    const float nb = sp * pp + sm * pm + sn * pn_ + ss * ps + st * pt + sb * pb;
    const float pn = (nb + sc * dx * dx) / denom;
    return (1.0f - omega_j) * pin + omega_j * pn;
}

// ---- the potential solve over its live cells ---------------------------------
// Only the cells the sweep does not hold at 0 (metal above the grounded
// plate) change: the sweeps walk a list of them.  The fixed cells stay exact
// because both potential buffers hold 0 at every fixed cell: k_elec_prepare
// zeroes the output buffer of the first sweep at cells that became fixed
// since the previous solve (old mask 0, new mask 1), the zero list zeroes the
// other buffer after that sweep, and every later sweep writes 0 there in the
// reference anyway.  Fixed cells then add exactly 0 to the L1 sums of every
// sweep after the first.  counts: [0] live cells, [1] newly fixed cells,
// [2 + b] live cells of tile block b, then (after the scan) its list offset;
// after those the per-block live bitmaps (one word per warp) and the totals
// of the scan's 1024-block groups.
constexpr int kCntLive = 0, kCntZero = 1, kCntBlocks = 2;
constexpr int kLiveBlocks = 148 * 8;
constexpr int kWarpsPerTile = kTileK * kTileJ / 32;
constexpr int kScanGroup = 1024;

inline int64_t counts_bitmap_offset(int64_t nb) { return kCntBlocks + nb; }
inline int64_t counts_group_offset(int64_t nb) { return kCntBlocks + nb + nb * kWarpsPerTile; }
inline int64_t counts_total_len(int64_t nb) {
    return counts_group_offset(nb) + (nb + kScanGroup - 1) / kScanGroup;
}

__device__ __forceinline__ int tile_block_linear() {
    return (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
}

__global__ void __launch_bounds__(kTileK* kTileJ)
    k_elec_prepare(Dims d, float* __restrict__ sigma, uint8_t* __restrict__ fixed,
                   float* __restrict__ phi_b, const float* __restrict__ f_l,
                   const int32_t* __restrict__ flags, float s_liq, float s_sol, int nz_solid,
                   int* __restrict__ zero_list, int* __restrict__ counts,
                   unsigned* __restrict__ bitmaps) {
    int i, j, k, c;
    const bool ok = tile_cell(d, i, j, k, c);
    bool live = false, newly = false;
    if (ok) {
        const int fl = flags[c];
        sigma[c] = fl == GAS ? 1e-8f : (f_l[c] > 0.55f ? s_liq : s_sol);
        const uint8_t nf = (fl == GAS || (k <= nz_solid && fl == SOLID)) ? 1 : 0;
        const uint8_t of = fixed[c];
        if (nf != of) fixed[c] = nf;
        newly = nf && !of;
        if (newly) phi_b[c] = 0.0f;
        live = !nf;
    }
    // newly fixed cells: one atomic per warp
    const unsigned m = __ballot_sync(0xffffffffu, newly);
    const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
    int base = 0;
    if (m && lane == 0) base = atomicAdd(&counts[kCntZero], __popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (newly) zero_list[base + __popc(m & ((1u << lane) - 1u))] = c;
    const unsigned lm = __ballot_sync(0xffffffffu, live);
    const int b = tile_block_linear();
    if (lane == 0) bitmaps[(int64_t)b * kWarpsPerTile + ((threadIdx.y * blockDim.x) >> 5)] = lm;
    const int nlive = __syncthreads_count(live);
    if (threadIdx.x == 0 && threadIdx.y == 0) counts[kCntBlocks + b] = nlive;
}

// Exclusive scan of the per-block live counts in two levels: each block of
// 1024 threads scans a group of 1024 counts (coalesced) and leaves the group
// total; k_elec_scan_groups scans the totals; k_elec_list adds both.
__device__ __forceinline__ int block_exclusive_scan_1024(int v, int& total) {
    __shared__ int warp_sums[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_sums[w] = incl;
    __syncthreads();
    if (w == 0) {
        int ws_ = warp_sums[lane], wincl = ws_;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, wincl, o);
            if (lane >= o) wincl += y;
        }
        warp_sums[lane] = wincl - ws_;
        if (lane == 31) total = wincl;
    }
    __syncthreads();
    const int out = warp_sums[w] + incl - v;
    return out;
}

__global__ void __launch_bounds__(kScanGroup) k_elec_scan(int* counts, int nb, int* groups) {
    const int b = blockIdx.x * kScanGroup + threadIdx.x;
    const int v = b < nb ? counts[kCntBlocks + b] : 0;
    int t = 0;
    const int ex = block_exclusive_scan_1024(v, t);
    if (b < nb) counts[kCntBlocks + b] = ex;
    if (threadIdx.x == 31) groups[blockIdx.x] = t;   // thread 31 holds the group total
}

// Exclusive scan of the group totals (one block), total live count to counts[0].
__global__ void __launch_bounds__(kScanGroup) k_elec_scan_groups(int* counts, int* groups,
                                                                 int n_groups) {
    int running = 0;
    for (int g0 = 0; g0 < n_groups; g0 += kScanGroup) {
        const int g = g0 + threadIdx.x;
        const int v = g < n_groups ? groups[g] : 0;
        __shared__ int tot;
        int t = 0;
        const int ex = block_exclusive_scan_1024(v, t);
        if (threadIdx.x == 31) tot = t;
        __syncthreads();
        if (g < n_groups) groups[g] = running + ex;
        running += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) counts[kCntLive] = running;
}

// The live list in tile-block order (a fixed order), from the blocks' bitmaps:
// one warp per tile block (grid-stride), which leaves at once when the block
// has no live cells.
__global__ void __launch_bounds__(256)
    k_elec_list(Dims d, const int* __restrict__ counts, const unsigned* __restrict__ bitmaps,
                const int* __restrict__ groups, int nb, int gx, int gy,
                int* __restrict__ live_list) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nb; b += nwarps) {
        const int off = counts[kCntBlocks + b] + groups[b / kScanGroup];
        const int next = b + 1 < nb ? counts[kCntBlocks + b + 1] + groups[(b + 1) / kScanGroup]
                                    : counts[kCntLive];
        if (next == off) continue;
        const int bx = b % gx, by = (b / gx) % gy, i = b / (gx * gy);
        int base = off;
        for (int w = 0; w < kWarpsPerTile; ++w) {
            const unsigned m = bitmaps[(int64_t)b * kWarpsPerTile + w];
            if ((m >> lane) & 1u) {
                const int k = bx * kTileK + lane, j = by * kTileJ + w;
                live_list[base + __popc(m & ((1u << lane) - 1u))] = (i * d.ny + j) * d.nz + k;
            }
            base += __popc(m);
        }
    }
}

// One sweep over the live list (a fixed grid: the L1 sums in a fixed order).
template <bool L1>
__global__ void __launch_bounds__(256)
    k_elec_jacobi_live(Dims d, const float* __restrict__ phi_in, float* __restrict__ phi_out,
                       const float* __restrict__ sigma, const float* __restrict__ src,
                       const int* __restrict__ live_list, const int* __restrict__ counts,
                       float dx, float omega_j, const float* __restrict__ arc_k_dev,
                       float sigma_cells, float* diff_out, float* norm_out, Workspace ws) {
    const int cnt = counts[kCntLive];
    int k_src_lo, k_src_hi;
    source_slab(*arc_k_dev, sigma_cells, d.nz, k_src_lo, k_src_hi);
    const int sx = d.ny * d.nz, sy = d.nz;
    double dsum = 0.0, nsum = 0.0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        const int c = live_list[t];
        const int k = c % d.nz;
        const int r = c / d.nz;
        const int j = r % d.ny, i = r / d.ny;
        const int ip = c + (i + 1 < d.nx ? sx : 0), im = c - (i > 0 ? sx : 0);
        const int jp = c + (j + 1 < d.ny ? sy : 0), jm = c - (j > 0 ? sy : 0);
        const int kp = c + (k + 1 < d.nz ? 1 : 0), km = c - (k > 0 ? 1 : 0);
        const float pin = phi_in[c];
        const float sc = (k >= k_src_lo && k <= k_src_hi) ? src[c] : 0.0f;
        const float out = jacobi_cell(pin, sigma[ip], sigma[im], sigma[jp], sigma[jm], sigma[kp],
                                      sigma[km], phi_in[ip], phi_in[im], phi_in[jp], phi_in[jm],
                                      phi_in[kp], phi_in[km], sc, dx, omega_j);
        phi_out[c] = out;
        if (L1) {
            dsum += (double)fabsf(out - pin);
            nsum += (double)fabsf(pin);
        }
    }
    if (L1) {
        double2 part = block_sum2(dsum, nsum);
        double2 tot;
        if (finish_sum2(ws, part, tot)) {
            *diff_out = (float)tot.x;
            *norm_out = (float)tot.y;
        }
    }
}

__global__ void k_elec_zero_list(const int* __restrict__ zero_list, const int* __restrict__ counts,
                                 float* phi) {
    const int cnt = counts[kCntZero];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x)
        phi[zero_list[t]] = 0.0f;
}

// kernels.py:1237-1251 elec_build_sigma, plus the byte mask of the cells the
// Jacobi sweep holds at 0 (kernels.py:1315-1355: GAS, SOLID at k <= nz_solid).
__global__ void k_elec_sigma_mask(Dims d, float* sigma, uint8_t* fixed, const float* f_l,
                                  const int32_t* flags, float s_liq, float s_sol, int nz_solid) {
    int i, j, k, c;
    if (!tile_cell(d, i, j, k, c)) return;
    const int fl = flags[c];
    sigma[c] = fl == GAS ? 1e-8f : (f_l[c] > 0.55f ? s_liq : s_sol);
    fixed[c] = (fl == GAS || (k <= nz_solid && fl == SOLID)) ? 1 : 0;
}

// kernels.py:1387-1398 elec_l1_diff as an operator
__global__ void __launch_bounds__(kTileK* kTileJ)
    k_elec_l1(Dims d, const float* __restrict__ a, const float* __restrict__ b, float* diff_out,
              float* norm_out, Workspace ws) {
    double dsum = 0.0, nsum = 0.0;
    for (int i = blockIdx.z; i < d.nx; i += gridDim.z)
        for (int jt = blockIdx.y; jt * kTileJ < d.ny; jt += gridDim.y)
            for (int kt = blockIdx.x; kt * kTileK < d.nz; kt += gridDim.x) {
                const int k = kt * kTileK + threadIdx.x, j = jt * kTileJ + threadIdx.y;
                if (k >= d.nz || j >= d.ny) continue;
                const int c = (i * d.ny + j) * d.nz + k;
                const float bv = b[c];
                dsum += (double)fabsf(a[c] - bv);
                nsum += (double)fabsf(bv);
            }
    double2 part = block_sum2(dsum, nsum);
    double2 tot;
    if (finish_sum2(ws, part, tot)) {
        *diff_out = (float)tot.x;
        *norm_out = (float)tot.y;
    }
}

// kernels.py:1358-1383 elec_compute_J
__global__ void k_elec_J(Dims d, float* Jx, float* Jy, float* Jz, const float* __restrict__ phi,
                         const float* __restrict__ sigma, const int32_t* __restrict__ flags,
                         float dx) {
    int i, j, k, c;
    if (!tile_cell(d, i, j, k, c)) return;
    if (flags[c] == GAS) {
        Jx[c] = 0.0f;
        Jy[c] = 0.0f;
        Jz[c] = 0.0f;
        return;
    }
    const int sx = d.ny * d.nz, sy = d.nz;
    const float sg = sigma[c];
    const float two_dx = 2.0f * dx;
    const float gx = (phi[c + (i + 1 < d.nx ? sx : 0)] - phi[c - (i > 0 ? sx : 0)]) / two_dx;
    const float gy = (phi[c + (j + 1 < d.ny ? sy : 0)] - phi[c - (j > 0 ? sy : 0)]) / two_dx;
    const float gz = (phi[c + (k + 1 < d.nz ? 1 : 0)] - phi[c - (k > 0 ? 1 : 0)]) / two_dx;
    Jx[c] = -sg * gx;
    Jy[c] = -sg * gy;
    Jz[c] = -sg * gz;
}

__device__ __forceinline__ int radial_bin(float di, float dj, float bin_dr, int n_bins,
                                          float& r) {
    r = sqrtf(di * di + dj * dj);
    return imin((int)(r / bin_dr), n_bins - 1);
}

// kernels.py:1402-1421 elec_bin_axial_current: per z slab, sum of Jz dx^2 by
// radius bin.  Block (s, k) sums a strip of columns of slab k in shared
// double bins, then adds them to the slab's double accumulators.
__global__ void k_elec_bin(Dims d, const float* __restrict__ Jz, double* acc, float arc_i,
                           float arc_j, float dx2, float bin_dr, int n_bins) {
    extern __shared__ double sbin[];
    const int k = blockIdx.y;
    for (int b = threadIdx.x; b < n_bins; b += blockDim.x) sbin[b] = 0.0;
    __syncthreads();
    const int ncol = d.nx * d.ny;
    for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < ncol;
         col += gridDim.x * blockDim.x) {
        const int i = col / d.ny, j = col - i * d.ny;
        float r;
        const int b = radial_bin((float)i - arc_i, (float)j - arc_j, bin_dr, n_bins, r);
        atomicAdd(&sbin[b], (double)(Jz[(int64_t)col * d.nz + k] * dx2));
    }
    __syncthreads();
    for (int b = threadIdx.x; b < n_bins; b += blockDim.x)
        if (sbin[b] != 0.0) atomicAdd(&acc[(int64_t)k * n_bins + b], sbin[b]);
}

// The same sums without atomics: block (kt, ch) is one warp that owns k in
// [32 kt, 32 kt + 32) of a contiguous chunk of columns and adds each column's
// Jz dx^2 into its private shared double bins (lane k touches only its own
// slots), column after column; the loads of 32 columns are in flight at a
// time, coalesced along k, and lane u finds the bin of the u-th of them.  The
// per-chunk bins go to partials[ch][b][k]; k_elec_bin_combine adds the chunks
// in a fixed order, so the bins are the same on every run.
constexpr int kBinUnroll = 32;

__global__ void __launch_bounds__(32) k_elec_bin_cols(Dims d, const float* __restrict__ Jz,
                                                      double* __restrict__ partials, float arc_i,
                                                      float arc_j, float dx2, float bin_dr,
                                                      int n_bins, int chunk) {
    extern __shared__ double sacc[];   // [n_bins][32]
    const int lane = threadIdx.x;
    const int k = blockIdx.x * 32 + lane;
    for (int b = 0; b < n_bins; ++b) sacc[b * 32 + lane] = 0.0;
    const int ncol = d.nx * d.ny;
    const int c0 = blockIdx.y * chunk, c1 = imin(ncol, c0 + chunk);
    const bool kin = k < d.nz;
    for (int col = c0; col < c1; col += kBinUnroll) {
        float v[kBinUnroll];
#pragma unroll
        for (int u = 0; u < kBinUnroll; ++u)
            v[u] = (kin && col + u < c1) ? Jz[(int64_t)(col + u) * d.nz + k] : 0.0f;
        int my_bin = 0;
        if (col + lane < c1) {
            const int i = (col + lane) / d.ny, j = (col + lane) - i * d.ny;
            float r;
            my_bin = radial_bin((float)i - arc_i, (float)j - arc_j, bin_dr, n_bins, r);
        }
#pragma unroll
        for (int u = 0; u < kBinUnroll; ++u) {
            const int b = __shfl_sync(0xffffffffu, my_bin, u);
            if (col + u < c1) sacc[b * 32 + lane] += (double)(v[u] * dx2);
        }
    }
    if (!kin) return;
    double* out = partials + (int64_t)blockIdx.y * n_bins * d.nz;
    for (int b = 0; b < n_bins; ++b) out[(int64_t)b * d.nz + k] = sacc[b * 32 + lane];
}

// One warp per bin entry: lane l adds chunks l, l + 32, ... in order, then a
// fixed shuffle tree.
__global__ void k_elec_bin_combine(const double* __restrict__ partials, float* bins, int nz,
                                   int n_bins, int chunks) {
    const int64_t m = (int64_t)nz * n_bins;
    const int lane = threadIdx.x & 31;
    for (int64_t q = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < m;
         q += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int b = (int)(q % n_bins), k = (int)(q / n_bins);
        double s = 0.0;
        for (int ch = lane; ch < chunks; ch += 32) s += partials[((int64_t)ch * n_bins + b) * nz + k];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) bins[q] = (float)s;
    }
}

__global__ void k_elec_bin_store(const double* acc, float* bins, int64_t m) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < m;
         q += (int64_t)gridDim.x * blockDim.x)
        bins[q] = (float)acc[q];
}

// kernels.py:1424-1435 elec_prefix_bins (float, in place)
__global__ void k_elec_prefix(float* bins, int n_bins, int nz) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nz) return;
    float a = 0.0f;
    for (int b = 0; b < n_bins; ++b) {
        a += bins[(int64_t)k * n_bins + b];
        bins[(int64_t)k * n_bins + b] = a;
    }
}

// kernels.py:1438-1475 elec_B_axisymmetric, one warp per (i, j) column with
// lanes over k: the column's radius, bin and r * dx come once per lane, and
// each cell takes the reference's three divisions in its order (measured on
// 512x256x160: 9 us per step less than one thread per cell).
__global__ void __launch_bounds__(256) k_elec_B_cols(Dims d, float* Bx, float* By, float* Bz,
                                                     const float* __restrict__ bins, float arc_i,
                                                     float arc_j, float dx, float bin_dr,
                                                     float mu0, int n_bins) {
    const int col = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (col >= d.nx * d.ny) return;
    const int lane = threadIdx.x & 31;
    const int i = col / d.ny, j = col - i * d.ny;
    const float di = (float)i - arc_i, dj = (float)j - arc_j;
    float rc;
    const int b = radial_bin(di, dj, bin_dr, n_bins, rc);
    const bool on = rc > 1e-3f;
    const float rm = rc * dx;
    const float two_pi = 6.28318530717958647692f;
    const int64_t c0 = (int64_t)col * d.nz;
    for (int k = lane; k < d.nz; k += 32) {
        float bx = 0.0f, by = 0.0f;
        if (on) {
            const float I = bins[(int64_t)k * n_bins + b];
            const float Bt = mu0 * I / (two_pi * rm);
            bx = -Bt * dj / rc;
            by = Bt * di / rc;
        }
        Bx[c0 + k] = bx;
        By[c0 + k] = by;
        Bz[c0 + k] = 0.0f;
    }
}

// kernels.py:1479-1513 apply_lorentz_JxB
__global__ void k_lorentz_JxB(float* Fx, float* Fy, float* Fz, const float* __restrict__ Jx,
                              const float* __restrict__ Jy, const float* __restrict__ Jz,
                              const float* __restrict__ Bx, const float* __restrict__ By,
                              const float* __restrict__ Bz, const float* __restrict__ f_l,
                              const int32_t* __restrict__ flags, int64_t n, float dt, float dx,
                              float rho_ref) {
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        const float fl = f_l[c];
        if (flags[c] == GAS || fl < 0.05f) continue;
        const float jx = Jx[c], jy = Jy[c], jz = Jz[c], bx = Bx[c], by = By[c], bz = Bz[c];
        const float fxp = jy * bz - jz * by, fyp = jz * bx - jx * bz, fzp = jx * by - jy * bx;
        const float flw = fmin_(1.0f, fl);
        const float scale = flw * dt * dt / (rho_ref * dx);
        Fx[c] += fxp * scale;
        Fy[c] += fyp * scale;
        Fz[c] += fzp * scale;
    }
}

}  // namespace
}  // namespace waam

using namespace waam;


#define REQUIRE(cond, msg) \
    if (!(cond)) return waam::fail(WAAM_ERR_INVALID, msg)

extern "C" {

int waam_elec_build_sigma(float* sigma, const float* f_l, const int32_t* flags, int64_t n,
                          float sigma_liquid, float sigma_solid, void* stream) {
    REQUIRE(sigma && f_l && flags && n > 0, "elec_build_sigma: null field or empty grid");
    k_elec_sigma<<<elem_blocks(n), kThreads, 0, STREAM(stream)>>>(sigma, f_l, flags, n,
                                                                  sigma_liquid, sigma_solid);
    return check_launch("k_elec_sigma");
}

int waam_elec_inject_arc_source(float* source, int nx, int ny, int nz, float arc_i, float arc_j,
                                float arc_k, float sigma_cells, float current_A, float dx,
                                void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "elec_inject_arc_source: bad dims");
    REQUIRE(source, "elec_inject_arc_source: null field");
    REQUIRE(std::isfinite(arc_k) && std::isfinite(sigma_cells) && std::fabs(arc_k) < 1e6f &&
                std::fabs(sigma_cells) < 1e6f,
            "elec_inject_arc_source: arc k / sigma not finite");
    const float eps = 1e-6f;
    const float inv2s2 = 1.0f / (2.0f * sigma_cells * sigma_cells + eps);
    const float cell_vol = dx * dx * dx;
    int k_min, k_max;
    source_slab(arc_k, sigma_cells, nz, k_min, k_max);
    Dims d{nx, ny, nz};
    k_elec_source<<<tile_grid(d), tile_block(), 0, STREAM(stream)>>>(
        d, source, arc_i, arc_j, arc_k, inv2s2, current_A, cell_vol + eps, k_min, k_max);
    return check_launch("k_elec_source");
}

static int arc_source_impl(float* source, int nx, int ny, int nz, float arc_i, float arc_j,
                           float arc_k, const float* arc_k_dev, float sigma_cells,
                           float current_A, float dx, void* workspace, size_t workspace_bytes,
                           void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "elec_arc_source: bad dims");
    REQUIRE(source, "elec_arc_source: null field");
    REQUIRE(std::isfinite(arc_k) && std::isfinite(sigma_cells) && std::fabs(arc_k) < 1e6f &&
                std::fabs(sigma_cells) < 1e6f,
            "elec_arc_source: arc k / sigma not finite");
    Dims d{nx, ny, nz};
    REQUIRE(workspace_ok(workspace, workspace_bytes, d.n()),
            "elec_arc_source: workspace too small or misaligned");
    Workspace ws = Workspace::at(workspace);
    const float eps = 1e-6f;
    const float inv2s2 = 1.0f / (2.0f * sigma_cells * sigma_cells + eps);
    const float cell_vol = dx * dx * dx;
    // a fixed grid: the sum order does not depend on the GPU
    dim3 grid(imin((nz + kTileK - 1) / kTileK, 4), imin((ny + kTileJ - 1) / kTileJ, 16),
              imin(nx, 64));
    k_elec_source_fused_sum<<<grid, tile_block(), 0, STREAM(stream)>>>(
        d, arc_i, arc_j, arc_k, arc_k_dev, sigma_cells, inv2s2, current_A, cell_vol + eps,
        cell_vol, current_A, ws);
    int rc = check_launch("k_elec_source_fused_sum");
    if (rc) return rc;
    k_elec_source_fused_write<<<tile_grid(d), tile_block(), 0, STREAM(stream)>>>(
        d, source, arc_i, arc_j, arc_k, arc_k_dev, sigma_cells, inv2s2, current_A,
        cell_vol + eps, ws);
    return check_launch("k_elec_source_fused_write");
}

int waam_elec_arc_source(float* source, int nx, int ny, int nz, float arc_i, float arc_j,
                         float arc_k, float sigma_cells, float current_A, float dx,
                         void* workspace, size_t workspace_bytes, void* stream) {
    return arc_source_impl(source, nx, ny, nz, arc_i, arc_j, arc_k, nullptr, sigma_cells,
                           current_A, dx, workspace, workspace_bytes, stream);
}

int waam_elec_arc_source_dev(float* source, int nx, int ny, int nz, float arc_i, float arc_j,
                             const float* arc_k_dev, float sigma_cells, float current_A,
                             float dx, void* workspace, size_t workspace_bytes, void* stream) {
    REQUIRE(arc_k_dev, "elec_arc_source_dev: null arc k");
    return arc_source_impl(source, nx, ny, nz, arc_i, arc_j, 0.0f, arc_k_dev, sigma_cells,
                           current_A, dx, workspace, workspace_bytes, stream);
}

int waam_elec_normalize_source(float* source, int64_t n, float target_current_A, float dx,
                               void* workspace, size_t workspace_bytes, void* stream) {
    REQUIRE(source && n > 0, "elec_normalize_source: null field or empty grid");
    REQUIRE(workspace_ok(workspace, workspace_bytes, n),
            "elec_normalize_source: workspace too small or misaligned");
    Workspace ws = Workspace::at(workspace);
    const float cell_vol = dx * dx * dx;
    k_elec_source_sum<<<red_blocks(n), kThreads, 0, STREAM(stream)>>>(source, n, cell_vol,
                                                                      target_current_A, ws);
    int rc = check_launch("k_elec_source_sum");
    if (rc) return rc;
    k_elec_source_scale<<<elem_blocks(n), kThreads, 0, STREAM(stream)>>>(source, n, ws);
    return check_launch("k_elec_source_scale");
}

int waam_elec_init_ground(float* phi, int64_t n, void* stream) {
    REQUIRE(phi && n > 0, "elec_init_ground: null field or empty grid");
    cudaError_t e = cudaMemsetAsync(phi, 0, (size_t)n * sizeof(float), STREAM(stream));
    if (e != cudaSuccess) return fail(WAAM_ERR_CUDA, cudaGetErrorString(e));
    return WAAM_OK;
}

int waam_elec_jacobi_step(const float* phi_in, float* phi_out, const float* sigma,
                          const float* source, const int32_t* flags, int nx, int ny, int nz,
                          float dx, float omega_j, int nz_solid, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "elec_jacobi_step: bad dims");
    REQUIRE(phi_in && phi_out && sigma && source && flags && phi_in != phi_out,
            "elec_jacobi_step: null or aliased field");
    Dims d{nx, ny, nz};
    k_elec_jacobi<false><<<red_tile_grid(d), tile_block(), 0, STREAM(stream)>>>(
        d, phi_in, phi_out, sigma, source, flags, dx, omega_j, nz_solid, nullptr, nullptr,
        Workspace{});
    return check_launch("k_elec_jacobi");
}

int waam_elec_jacobi_step_l1(const float* phi_in, float* phi_out, const float* sigma,
                             const float* source, const int32_t* flags, int nx, int ny, int nz,
                             float dx, float omega_j, int nz_solid, float* diff_buf,
                             float* norm_buf, void* workspace, size_t workspace_bytes,
                             void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "elec_jacobi_step_l1: bad dims");
    REQUIRE(phi_in && phi_out && sigma && source && flags && diff_buf && norm_buf &&
                phi_in != phi_out,
            "elec_jacobi_step_l1: null or aliased field");
    Dims d{nx, ny, nz};
    REQUIRE(workspace_ok(workspace, workspace_bytes, d.n()),
            "elec_jacobi_step_l1: workspace too small or misaligned");
    k_elec_jacobi<true><<<red_tile_grid(d), tile_block(), 0, STREAM(stream)>>>(
        d, phi_in, phi_out, sigma, source, flags, dx, omega_j, nz_solid, diff_buf, norm_buf,
        Workspace::at(workspace));
    return check_launch("k_elec_jacobi_l1");
}

int waam_elec_build_sigma_mask(float* sigma, uint8_t* fixed, const float* f_l,
                               const int32_t* flags, int nx, int ny, int nz, float sigma_liquid,
                               float sigma_solid, int nz_solid, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "elec_build_sigma_mask: bad dims");
    REQUIRE(sigma && fixed && f_l && flags, "elec_build_sigma_mask: null field");
    Dims d{nx, ny, nz};
    k_elec_sigma_mask<<<tile_grid(d), tile_block(), 0, STREAM(stream)>>>(
        d, sigma, fixed, f_l, flags, sigma_liquid, sigma_solid, nz_solid);
    return check_launch("k_elec_sigma_mask");
}

int waam_elec_jacobi_chunk(float* phi_a, float* phi_b, const float* sigma, const float* source,
                           const uint8_t* fixed, int nx, int ny, int nz, float dx, float omega_j,
                           int n_sweeps, float arc_k, float sigma_cells, float* diff_buf,
                           float* norm_buf, void* workspace, size_t workspace_bytes,
                           void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "elec_jacobi_chunk: bad dims");
    REQUIRE(phi_a && phi_b && sigma && source && fixed && diff_buf && norm_buf && phi_a != phi_b,
            "elec_jacobi_chunk: null or aliased field");
    REQUIRE(n_sweeps >= 1, "elec_jacobi_chunk: n_sweeps must be >= 1");
    REQUIRE(std::isfinite(arc_k) && std::isfinite(sigma_cells) && std::fabs(arc_k) < 1e6f &&
                std::fabs(sigma_cells) < 1e6f,
            "elec_jacobi_chunk: arc k / sigma not finite");
    Dims d{nx, ny, nz};
    REQUIRE(workspace_ok(workspace, workspace_bytes, d.n()),
            "elec_jacobi_chunk: workspace too small or misaligned");
    int k_lo, k_hi;
    source_slab(arc_k, sigma_cells, nz, k_lo, k_hi);
    float* in = phi_a;
    float* out = phi_b;
    for (int s = 0; s < n_sweeps; ++s) {
        if (s + 1 < n_sweeps) {
            k_elec_jacobi_m<false><<<tile_grid(d), tile_block(), 0, STREAM(stream)>>>(
                d, in, out, sigma, source, fixed, dx, omega_j, k_lo, k_hi, nullptr, nullptr,
                Workspace{});
        } else {
            k_elec_jacobi_m<true><<<red_tile_grid(d), tile_block(), 0, STREAM(stream)>>>(
                d, in, out, sigma, source, fixed, dx, omega_j, k_lo, k_hi, diff_buf, norm_buf,
                Workspace::at(workspace));
        }
        int rc = check_launch("k_elec_jacobi_m");
        if (rc) return rc;
        float* t = in;
        in = out;
        out = t;
    }
    return WAAM_OK;
}

int64_t waam_elec_counts_len(int nx, int ny, int nz) {
    if (!dims_ok(nx, ny, nz)) return 0;
    const dim3 g = tile_grid(Dims{nx, ny, nz});
    return counts_total_len((int64_t)g.x * g.y * g.z);
}

int waam_elec_prepare(float* sigma, uint8_t* fixed, float* phi_b, const float* f_l,
                      const int32_t* flags, int nx, int ny, int nz, float sigma_liquid,
                      float sigma_solid, int nz_solid, int32_t* live_list, int32_t* zero_list,
                      int32_t* counts, int64_t counts_len, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "elec_prepare: bad dims");
    REQUIRE(sigma && fixed && phi_b && f_l && flags && live_list && zero_list && counts,
            "elec_prepare: null field");
    REQUIRE(counts_len >= waam_elec_counts_len(nx, ny, nz), "elec_prepare: counts too short");
    Dims d{nx, ny, nz};
    const dim3 g = tile_grid(d);
    const int nb = (int)(g.x * g.y * g.z);
    cudaError_t e = cudaMemsetAsync(counts, 0, kCntBlocks * sizeof(int32_t), STREAM(stream));
    if (e != cudaSuccess) return fail(WAAM_ERR_CUDA, cudaGetErrorString(e));
    unsigned* bitmaps = reinterpret_cast<unsigned*>(counts + counts_bitmap_offset(nb));
    int* groups = counts + counts_group_offset(nb);
    const int n_groups = (nb + kScanGroup - 1) / kScanGroup;
    k_elec_prepare<<<g, tile_block(), 0, STREAM(stream)>>>(d, sigma, fixed, phi_b, f_l, flags,
                                                           sigma_liquid, sigma_solid, nz_solid,
                                                           zero_list, counts, bitmaps);
    int rc = check_launch("k_elec_prepare");
    if (rc) return rc;
    k_elec_scan<<<n_groups, kScanGroup, 0, STREAM(stream)>>>(counts, nb, groups);
    rc = check_launch("k_elec_scan");
    if (rc) return rc;
    k_elec_scan_groups<<<1, kScanGroup, 0, STREAM(stream)>>>(counts, groups, n_groups);
    rc = check_launch("k_elec_scan_groups");
    if (rc) return rc;
    k_elec_list<<<kLiveBlocks, 256, 0, STREAM(stream)>>>(d, counts, bitmaps, groups, nb,
                                                         (int)g.x, (int)g.y, live_list);
    return check_launch("k_elec_list");
}

int waam_elec_jacobi_live(float* phi_a, float* phi_b, const float* sigma, const float* source,
                          const int32_t* live_list, const int32_t* zero_list,
                          const int32_t* counts, int nx, int ny, int nz, float dx,
                          float omega_j, int n_sweeps, int first_chunk, const float* arc_k_dev,
                          float sigma_cells, float* diff_buf, float* norm_buf, void* workspace,
                          size_t workspace_bytes, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "elec_jacobi_live: bad dims");
    REQUIRE(phi_a && phi_b && sigma && source && live_list && zero_list && counts && diff_buf &&
                norm_buf && phi_a != phi_b,
            "elec_jacobi_live: null or aliased field");
    REQUIRE(n_sweeps >= 1, "elec_jacobi_live: n_sweeps must be >= 1");
    REQUIRE(!first_chunk || n_sweeps >= 2,
            "elec_jacobi_live: the first chunk of a solve needs at least 2 sweeps");
    REQUIRE(arc_k_dev && std::isfinite(sigma_cells) && std::fabs(sigma_cells) < 1e6f,
            "elec_jacobi_live: null arc k or sigma not finite");
    Dims d{nx, ny, nz};
    REQUIRE(workspace_ok(workspace, workspace_bytes, d.n()),
            "elec_jacobi_live: workspace too small or misaligned");
    float* in = phi_a;
    float* out = phi_b;
    for (int s = 0; s < n_sweeps; ++s) {
        if (s + 1 < n_sweeps)
            k_elec_jacobi_live<false><<<kLiveBlocks, 256, 0, STREAM(stream)>>>(
                d, in, out, sigma, source, live_list, counts, dx, omega_j, arc_k_dev,
                sigma_cells, nullptr, nullptr, Workspace{});
        else
            k_elec_jacobi_live<true><<<kLiveBlocks, 256, 0, STREAM(stream)>>>(
                d, in, out, sigma, source, live_list, counts, dx, omega_j, arc_k_dev,
                sigma_cells, diff_buf, norm_buf, Workspace::at(workspace));
        int rc = check_launch("k_elec_jacobi_live");
        if (rc) return rc;
        if (first_chunk && s == 0) {
            // the input of the first sweep: its newly fixed cells become 0
            k_elec_zero_list<<<kLiveBlocks, 256, 0, STREAM(stream)>>>(zero_list, counts, in);
            rc = check_launch("k_elec_zero_list");
            if (rc) return rc;
        }
        float* t = in;
        in = out;
        out = t;
    }
    return WAAM_OK;
}

int waam_elec_l1_diff(const float* a, const float* b, float* diff_buf, float* norm_buf, int nx,
                      int ny, int nz, void* workspace, size_t workspace_bytes, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "elec_l1_diff: bad dims");
    REQUIRE(a && b && diff_buf && norm_buf, "elec_l1_diff: null field");
    Dims d{nx, ny, nz};
    REQUIRE(workspace_ok(workspace, workspace_bytes, d.n()),
            "elec_l1_diff: workspace too small or misaligned");
    k_elec_l1<<<red_tile_grid(d), tile_block(), 0, STREAM(stream)>>>(d, a, b, diff_buf, norm_buf,
                                                                     Workspace::at(workspace));
    return check_launch("k_elec_l1");
}

int waam_elec_compute_J(float* Jx, float* Jy, float* Jz, const float* phi, const float* sigma,
                        const int32_t* flags, int nx, int ny, int nz, float dx, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "elec_compute_J: bad dims");
    REQUIRE(Jx && Jy && Jz && phi && sigma && flags, "elec_compute_J: null field");
    Dims d{nx, ny, nz};
    k_elec_J<<<tile_grid(d), tile_block(), 0, STREAM(stream)>>>(d, Jx, Jy, Jz, phi, sigma, flags,
                                                               dx);
    return check_launch("k_elec_J");
}

int waam_elec_bin_axial_current(const float* Jz, float* bins, int nx, int ny, int nz, float arc_i,
                                float arc_j, float dx, float bin_dr_cells, int n_bins,
                                void* workspace, size_t workspace_bytes, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "elec_bin_axial_current: bad dims");
    REQUIRE(Jz && bins, "elec_bin_axial_current: null field");
    REQUIRE(n_bins >= 1 && n_bins <= kMaxBins, "elec_bin_axial_current: n_bins out of range");
    Dims d{nx, ny, nz};
    REQUIRE(workspace_ok(workspace, workspace_bytes, d.n()),
            "elec_bin_axial_current: workspace too small or misaligned");
    // double accumulators in the workspace's field scratch
    const int64_t m = (int64_t)nz * n_bins;
    REQUIRE((size_t)m * sizeof(double) <= (size_t)(d.n() + kFieldSlack) * sizeof(float),
            "elec_bin_axial_current: nz * n_bins accumulators exceed the workspace");
    Workspace ws = Workspace::at(workspace);
    double* acc = reinterpret_cast<double*>(ws.field);
    const int ncol = nx * ny;
    {
        // chunked per-warp bins in the field scratch, when they fit
        const size_t field_bytes = (size_t)(d.n() + kFieldSlack) * sizeof(float);
        const int ktiles = (nz + 31) / 32;
        int chunks = imax(1, (148 * 12) / ktiles);
        chunks = imin(chunks, ncol);
        chunks = (int)std::min<int64_t>(chunks, (int64_t)(field_bytes / ((size_t)m * sizeof(double))));
        if (chunks >= 1 && (size_t)n_bins * 32 * sizeof(double) <= 48 * 1024) {
            const int chunk = (ncol + chunks - 1) / chunks;
            chunks = (ncol + chunk - 1) / chunk;
            k_elec_bin_cols<<<dim3(ktiles, chunks), 32, (size_t)n_bins * 32 * sizeof(double),
                              STREAM(stream)>>>(d, Jz, acc, arc_i, arc_j, dx * dx, bin_dr_cells,
                                                n_bins, chunk);
            int rc = check_launch("k_elec_bin_cols");
            if (rc) return rc;
            k_elec_bin_combine<<<elem_blocks(m * 32), kThreads, 0, STREAM(stream)>>>(
                acc, bins, nz, n_bins, chunks);
            return check_launch("k_elec_bin_combine");
        }
    }
    cudaError_t e = cudaMemsetAsync(acc, 0, (size_t)m * sizeof(double), STREAM(stream));
    if (e != cudaSuccess) return fail(WAAM_ERR_CUDA, cudaGetErrorString(e));
    const int strips = imax(1, imin((ncol + kThreads - 1) / kThreads, imax(1, 1184 / nz)));
    k_elec_bin<<<dim3(strips, nz), kThreads, n_bins * sizeof(double), STREAM(stream)>>>(
        d, Jz, acc, arc_i, arc_j, dx * dx, bin_dr_cells, n_bins);
    int rc = check_launch("k_elec_bin");
    if (rc) return rc;
    k_elec_bin_store<<<elem_blocks(m), kThreads, 0, STREAM(stream)>>>(acc, bins, m);
    return check_launch("k_elec_bin_store");
}

int waam_elec_prefix_bins(float* bins, int n_bins, int nz, void* stream) {
    REQUIRE(bins && n_bins >= 1 && nz >= 1, "elec_prefix_bins: bad arguments");
    k_elec_prefix<<<(nz + 127) / 128, 128, 0, STREAM(stream)>>>(bins, n_bins, nz);
    return check_launch("k_elec_prefix");
}

int waam_elec_B_axisymmetric(float* Bx, float* By, float* Bz, const float* bins, int nx, int ny,
                             int nz, float arc_i, float arc_j, float dx, float bin_dr_cells,
                             float mu0, int n_bins, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "elec_B_axisymmetric: bad dims");
    REQUIRE(Bx && By && Bz && bins, "elec_B_axisymmetric: null field");
    REQUIRE(n_bins >= 1, "elec_B_axisymmetric: n_bins out of range");
    Dims d{nx, ny, nz};
    const int64_t warps = (int64_t)nx * ny;
    k_elec_B_cols<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, STREAM(stream)>>>(
        d, Bx, By, Bz, bins, arc_i, arc_j, dx, bin_dr_cells, mu0, n_bins);
    return check_launch("k_elec_B_cols");
}

int waam_elec_fields(float* Jx, float* Jy, float* Jz, float* Bx, float* By, float* Bz,
                     float* bins, const float* phi, const float* sigma, const int32_t* flags,
                     int nx, int ny, int nz, float arc_i, float arc_j, float dx,
                     float bin_dr_cells, float mu0, int n_bins, void* workspace,
                     size_t workspace_bytes, void* stream) {
    int rc = waam_elec_compute_J(Jx, Jy, Jz, phi, sigma, flags, nx, ny, nz, dx, stream);
    if (rc) return rc;
    rc = waam_elec_bin_axial_current(Jz, bins, nx, ny, nz, arc_i, arc_j, dx, bin_dr_cells,
                                     n_bins, workspace, workspace_bytes, stream);
    if (rc) return rc;
    rc = waam_elec_prefix_bins(bins, n_bins, nz, stream);
    if (rc) return rc;
    return waam_elec_B_axisymmetric(Bx, By, Bz, bins, nx, ny, nz, arc_i, arc_j, dx, bin_dr_cells,
                                    mu0, n_bins, stream);
}

int waam_apply_lorentz_JxB(float* Fx, float* Fy, float* Fz, const float* Jx, const float* Jy,
                           const float* Jz, const float* Bx, const float* By, const float* Bz,
                           const float* f_l, const int32_t* flags, int64_t n, float dt, float dx,
                           float rho_ref, void* stream) {
    REQUIRE(Fx && Fy && Fz && Jx && Jy && Jz && Bx && By && Bz && f_l && flags && n > 0,
            "apply_lorentz_JxB: null field or empty grid");
    k_lorentz_JxB<<<elem_blocks(n), kThreads, 0, STREAM(stream)>>>(Fx, Fy, Fz, Jx, Jy, Jz, Bx, By,
                                                                   Bz, f_l, flags, n, dt, dx,
                                                                   rho_ref);
    return check_launch("k_lorentz_JxB");
}

}  // extern "C"
