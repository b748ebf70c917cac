// Pool telemetry on the device (twin.py:706-821 get_telemetry,
// kernels.py:3424-3481 telemetry_pool_reduce / extract_fl_yz_slice,
// physics/electrical_stickout.py:39-50 bead height, physics/bead_geometry.py:13-40
// toe column, export/probes.py:90-107 probe samples).
//
// One reduction pass over the grid and one single-block finish produce every
// aggregate in a WaamTelemetry record in device memory, so a telemetry call
// costs two launches and one small device-to-host read instead of the
// reference's atomics plus slice and volume copies.  All reductions are
// deterministic: maxima and integer sums do not depend on order, and the
// FP64 enthalpy sum uses a fixed block count, a fixed cell-to-thread map and
// fixed-order block and partial combination.
#include <climits>

#include "../../include/waam_b200.h"
#include "waam_common.cuh"
#include "waam_internal.cuh"

namespace waam {

#define STREAM(s) reinterpret_cast<cudaStream_t>(s)

namespace {

constexpr int kTelemBlocks = 592;   // fixed: the FP64 sum order never depends on the GPU
constexpr int kTelemThreads = 256;
constexpr int kTelemSlots = 10;     // partial values per block

struct TelemAcc {
    double h_sum, n, i_sum;
    float T_global, T_peak, cool, u2;
    int i_min, i_max, bead;
};

__device__ __forceinline__ void acc_init(TelemAcc& a) {
    a.h_sum = 0.0;
    a.n = 0.0;
    a.i_sum = 0.0;
    // the reference's buffers start at 0 (kernels.py:3440-3447): maxima are
    // at least 0
    a.T_global = 0.0f;
    a.T_peak = 0.0f;
    a.cool = 0.0f;
    a.u2 = 0.0f;
    a.i_min = INT_MAX;
    a.i_max = INT_MIN;
    a.bead = -1;
}

__device__ __forceinline__ void acc_merge(TelemAcc& a, const TelemAcc& b) {
    a.h_sum += b.h_sum;
    a.n += b.n;
    a.i_sum += b.i_sum;
    a.T_global = fmaxf(a.T_global, b.T_global);
    a.T_peak = fmaxf(a.T_peak, b.T_peak);
    a.cool = fmaxf(a.cool, b.cool);
    a.u2 = fmaxf(a.u2, b.u2);
    a.i_min = min(a.i_min, b.i_min);
    a.i_max = max(a.i_max, b.i_max);
    a.bead = max(a.bead, b.bead);
}

__device__ __forceinline__ TelemAcc acc_shfl_down(const TelemAcc& a, int o) {
    TelemAcc b;
    b.h_sum = __shfl_down_sync(0xffffffffu, a.h_sum, o);
    b.n = __shfl_down_sync(0xffffffffu, a.n, o);
    b.i_sum = __shfl_down_sync(0xffffffffu, a.i_sum, o);
    b.T_global = __shfl_down_sync(0xffffffffu, a.T_global, o);
    b.T_peak = __shfl_down_sync(0xffffffffu, a.T_peak, o);
    b.cool = __shfl_down_sync(0xffffffffu, a.cool, o);
    b.u2 = __shfl_down_sync(0xffffffffu, a.u2, o);
    b.i_min = __shfl_down_sync(0xffffffffu, a.i_min, o);
    b.i_max = __shfl_down_sync(0xffffffffu, a.i_max, o);
    b.bead = __shfl_down_sync(0xffffffffu, a.bead, o);
    return b;
}

// Block combination in a fixed order: a shuffle tree inside each warp, then
// thread 0 merges the warps in index order.  The result is valid in thread 0.
__device__ TelemAcc acc_block(TelemAcc a) {
    __shared__ TelemAcc sh[kTelemThreads / 32];
    for (int o = 16; o > 0; o >>= 1) acc_merge(a, acc_shfl_down(a, o));
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int w = 1; w < kTelemThreads / 32; ++w) acc_merge(a, sh[w]);
    __syncthreads();
    return a;
}

__device__ __forceinline__ void acc_store(double* part, int nb, int b, const TelemAcc& a) {
    part[0 * nb + b] = a.h_sum;
    part[1 * nb + b] = a.n;
    part[2 * nb + b] = a.i_sum;
    part[3 * nb + b] = (double)a.T_global;
    part[4 * nb + b] = (double)a.T_peak;
    part[5 * nb + b] = (double)a.cool;
    part[6 * nb + b] = (double)a.u2;
    part[7 * nb + b] = (double)a.i_min;
    part[8 * nb + b] = (double)a.i_max;
    part[9 * nb + b] = (double)a.bead;
}

__device__ __forceinline__ TelemAcc acc_load(const volatile double* part, int nb, int b) {
    TelemAcc a;
    a.h_sum = part[0 * nb + b];
    a.n = part[1 * nb + b];
    a.i_sum = part[2 * nb + b];
    a.T_global = (float)part[3 * nb + b];
    a.T_peak = (float)part[4 * nb + b];
    a.cool = (float)part[5 * nb + b];
    a.u2 = (float)part[6 * nb + b];
    a.i_min = (int)part[7 * nb + b];
    a.i_max = (int)part[8 * nb + b];
    a.bead = (int)part[9 * nb + b];
    return a;
}

// kernels.py:3424-3468 plus the bead height and the FP64 total enthalpy.
// Cells are visited in a fixed grid-stride order; the last block to finish
// combines the per-block partials in block order and writes the record.
__global__ void __launch_bounds__(kTelemThreads) k_telemetry_reduce(
    Dims d, const float* __restrict__ T, const float* __restrict__ f_l,
    const float* __restrict__ phi, const float* __restrict__ dT_dt,
    const float* __restrict__ ux, const float* __restrict__ uy, const float* __restrict__ uz,
    const float* __restrict__ H, const int32_t* __restrict__ flags, int nz_solid,
    WaamTelemetry* out, Workspace ws) {
    TelemAcc a;
    acc_init(a);
    const int64_t n = d.n();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t plane = (int64_t)d.ny * d.nz;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += stride) {
        const float Tc = T[c];
        a.T_global = fmaxf(a.T_global, Tc);
        if (H) a.h_sum += (double)H[c];
        if (phi[c] > 0.05f) a.cool = fmaxf(a.cool, -dT_dt[c]);
        const int i = (int)(c / plane);
        if (f_l[c] > 0.5f) {
            a.n += 1.0;
            a.T_peak = fmaxf(a.T_peak, Tc);
            const float u = ux[c], v = uy[c], w = uz[c];
            a.u2 = fmaxf(a.u2, u * u + v * v + w * w);
            a.i_sum += (double)i;
            a.i_min = min(a.i_min, i);
            a.i_max = max(a.i_max, i);
        }
        const int k = (int)(c % d.nz);
        if (flags && k >= nz_solid && flags[c] == SOLID) a.bead = max(a.bead, k);
    }
    a = acc_block(a);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        acc_store(ws.partials, gridDim.x, blockIdx.x, a);
        __threadfence();
        last = atomicAdd(ws.counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    TelemAcc t;
    acc_init(t);
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
        acc_merge(t, acc_load((volatile double*)ws.partials, gridDim.x, b));
    t = acc_block(t);
    if (threadIdx.x == 0) {
        *ws.counter = 0u;
        out->H_sum = t.h_sum;
        out->T_global = (double)t.T_global;
        out->T_peak = (double)t.T_peak;
        out->peak_cool = (double)t.cool;
        out->u2_max = (double)t.u2;
        out->n_liquid = (int64_t)t.n;
        out->i_sum = (int64_t)t.i_sum;
        out->i_min = t.n > 0.0 ? t.i_min : -1;
        out->i_max = t.n > 0.0 ? t.i_max : -1;
        out->bead_k_max = t.bead;
    }
}

// twin.py:723-744: the slice through the pool centroid (rounded half to even,
// as Python's round) and the y / z extent of f_l > 0.5 in it; the porosity
// tracer counts (twin.py:746-749); the toe-angle column (bead_geometry.py:21-29).
__global__ void __launch_bounds__(kTelemThreads) k_telemetry_finish(
    Dims d, const float* __restrict__ f_l, const float* __restrict__ phi,
    const int32_t* __restrict__ flags, const int32_t* __restrict__ tracer_active,
    int max_tracers, int nz_solid, WaamTelemetry* out) {
    __shared__ int y_min, y_max, z_min, n_act, n_trap;
    __shared__ int i_c;
    if (threadIdx.x == 0) {
        y_min = INT_MAX;
        y_max = INT_MIN;
        z_min = INT_MAX;
        n_act = 0;
        n_trap = 0;
        const int64_t nl = out->n_liquid;
        int ic = -1;
        if (nl > 0) {
            ic = (int)rint((double)out->i_sum / (double)nl);
            ic = max(0, min(d.nx - 1, ic));
        }
        i_c = ic;
    }
    __syncthreads();
    if (i_c >= 0) {
        const int64_t base = (int64_t)i_c * d.ny * d.nz;
        for (int s = threadIdx.x; s < d.ny * d.nz; s += blockDim.x) {
            if (f_l[base + s] > 0.5f) {
                const int j = s / d.nz, k = s % d.nz;
                atomicMin(&y_min, j);
                atomicMax(&y_max, j);
                atomicMin(&z_min, k);
            }
        }
    }
    if (tracer_active) {
        int a1 = 0, a2 = 0;
        for (int p = threadIdx.x; p < max_tracers; p += blockDim.x) {
            const int v = tracer_active[p];
            a1 += v == 1;
            a2 += v == 2;
        }
        atomicAdd(&n_act, a1);
        atomicAdd(&n_trap, a2);
    }
    // toe column: i = nx / 3, j = ny / 2, k in [max(0, nz_solid - 1), min(nz - 1, nz_solid + 8))
    const int k0 = max(0, nz_solid - 1), k1 = min(d.nz - 1, nz_solid + 8);
    const int nt = flags ? max(0, min(k1 - k0, WAAM_TOE_CELLS)) : 0;
    if ((int)threadIdx.x < nt) {
        const int64_t c = ((int64_t)(d.nx / 3) * d.ny + d.ny / 2) * d.nz + k0 + threadIdx.x;
        out->toe_phi[threadIdx.x] = phi[c];
        out->toe_flags[threadIdx.x] = flags[c];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        out->i_c = i_c;
        const bool any = y_min != INT_MAX;
        out->y_min = any ? y_min : -1;
        out->y_max = any ? y_max : -1;
        out->z_min = any ? z_min : -1;
        out->n_tracers_active = n_act;
        out->n_tracers_trapped = n_trap;
        out->toe_k0 = k0;
        out->toe_n = nt;
    }
}

// export/probes.py:90-107: T and f_l at each probe cell (index < 0: NaN).
__global__ void k_probe_sample(const float* __restrict__ T, const float* __restrict__ f_l,
                               WaamProbeSet ps, float* __restrict__ row) {
    const int p = threadIdx.x;
    if (p >= ps.n_probes) return;
    const int64_t c = ps.cell[p];
    row[2 * p] = c >= 0 ? T[c] : __int_as_float(0x7fc00000);
    row[2 * p + 1] = c >= 0 ? f_l[c] : __int_as_float(0x7fc00000);
}

__global__ void k_bead_height(Dims d, const int32_t* __restrict__ flags, int nz_solid,
                              int32_t* out) {
    const int64_t n = d.n();
    int best = -1;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(c % d.nz);
        if (k >= nz_solid && flags[c] == SOLID) best = max(best, k);
    }
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_down_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0 && best >= 0) atomicMax(out, best);
}

}  // namespace

}  // namespace waam

using namespace waam;

#define REQUIRE(cond, msg) \
    if (!(cond)) return waam::fail(WAAM_ERR_INVALID, msg)

extern "C" {

int waam_telemetry_pool(const float* T, const float* f_l, const float* phi, const float* dT_dt,
                        const float* ux, const float* uy, const float* uz, const float* H,
                        const int32_t* flags, const int32_t* tracer_active, int max_tracers,
                        int nx, int ny, int nz, int nz_solid, WaamTelemetry* out,
                        void* workspace, size_t workspace_bytes, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "telemetry: bad dims");
    REQUIRE(T && f_l && phi && dT_dt && ux && uy && uz && out, "telemetry: null field");
    REQUIRE(max_tracers >= 0, "telemetry: bad tracer count");
    Dims d{nx, ny, nz};
    REQUIRE(workspace_ok(workspace, workspace_bytes, d.n()), "telemetry: workspace too small");
    static_assert(kTelemBlocks * kTelemSlots <= kWsMaxPartials, "partials do not fit");
    Workspace ws = Workspace::at(workspace);
    k_telemetry_reduce<<<kTelemBlocks, kTelemThreads, 0, STREAM(stream)>>>(
        d, T, f_l, phi, dT_dt, ux, uy, uz, H, flags, nz_solid, out, ws);
    int e = check_launch("k_telemetry_reduce");
    if (e) return e;
    k_telemetry_finish<<<1, kTelemThreads, 0, STREAM(stream)>>>(
        d, f_l, phi, flags, max_tracers > 0 ? tracer_active : nullptr, max_tracers, nz_solid,
        out);
    return check_launch("k_telemetry_finish");
}

int waam_probe_sample(const float* T, const float* f_l, const WaamProbeSet* probes, float* row,
                      void* stream) {
    REQUIRE(T && f_l && probes && row, "probe_sample: null pointer");
    REQUIRE(probes->n_probes >= 0 && probes->n_probes <= WAAM_MAX_PROBES,
            "probe_sample: bad probe count");
    if (probes->n_probes == 0) return WAAM_OK;
    k_probe_sample<<<1, WAAM_MAX_PROBES, 0, STREAM(stream)>>>(T, f_l, *probes, row);
    return check_launch("k_probe_sample");
}

int waam_bead_height(const int32_t* flags, int nx, int ny, int nz, int nz_solid, int32_t* out,
                     void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "bead_height: bad dims");
    REQUIRE(flags && out, "bead_height: null pointer");
    Dims d{nx, ny, nz};
    cudaError_t ce = cudaMemsetAsync(out, 0xff, sizeof(int32_t), STREAM(stream));
    if (ce != cudaSuccess) return fail(WAAM_ERR_CUDA, cudaGetErrorString(ce));
    k_bead_height<<<elem_blocks(d.n()), kThreads, 0, STREAM(stream)>>>(d, flags, nz_solid, out);
    return check_launch("k_bead_height");
}

}  // extern "C"
