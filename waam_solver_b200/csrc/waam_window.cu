// Moving simulation window (kernels.py:2620-2723 shift_simulation_window_x,
// twin.py:599-631): every listed field moves n_shift cells towards i = 0 and
// the right strip is reset.
//
// One launch moves all fields.  Each thread owns one (j, k) column of one
// field plane and walks i upwards, as the reference's serial inner loop does,
// so the in-place move has no cross-thread hazard: index m is loaded at
// iteration m - n_shift and stored at iteration m.  Groups of four loads are
// issued before their four stores (a load of index m always precedes the store
// to m), which keeps several requests in flight per thread.  Consecutive
// threads hold consecutive k, so every access is coalesced.  The planes (up to
// WAAM_MAX_SHIFT_PLANES, float, int32 or 16-bit) travel in the launch
// parameters.
#include "../../include/waam_b200.h"
#include "waam_common.cuh"
#include "waam_internal.cuh"

namespace waam {

#define STREAM(s) reinterpret_cast<cudaStream_t>(s)

namespace {

struct ShiftTable {
    WaamShiftPlane p[WAAM_MAX_SHIFT_PLANES];
};

template <typename E>
__device__ __forceinline__ void shift_column(E* base, int64_t plane, int64_t col, int nx,
                                             int n_shift, int nz, int nz_solid, int mode,
                                             E below, E above) {
    const int keep = nx - n_shift;   // cells that receive a moved value
    int i = 0;
    for (; i + 4 <= keep; i += 4) {
        E v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = base[(int64_t)(i + u + n_shift) * plane + col];
#pragma unroll
        for (int u = 0; u < 4; ++u) base[(int64_t)(i + u) * plane + col] = v[u];
    }
    for (; i < keep; ++i) base[(int64_t)i * plane + col] = base[(int64_t)(i + n_shift) * plane + col];
    if (mode == WAAM_SHIFT_KEEP) return;
    const int k = (int)(col % nz);
    const E fill = (mode == WAAM_SHIFT_BY_K && k >= nz_solid) ? above : below;
    for (int r = keep < 0 ? 0 : keep; r < nx; ++r) base[(int64_t)r * plane + col] = fill;
}

__global__ void __launch_bounds__(256) k_shift_window(Dims d, const __grid_constant__ ShiftTable T,
                                                      int n_shift, int nz_solid) {
    const WaamShiftPlane& p = T.p[blockIdx.y];
    const int64_t plane = (int64_t)d.ny * d.nz;
    const int64_t col = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= plane) return;
    if (p.elem_bytes == 4) {
        shift_column<uint32_t>(static_cast<uint32_t*>(p.ptr), plane, col, d.nx, n_shift, d.nz,
                               nz_solid, p.mode, p.below, p.above);
    } else {
        shift_column<uint16_t>(static_cast<uint16_t*>(p.ptr), plane, col, d.nx, n_shift, d.nz,
                               nz_solid, p.mode, (uint16_t)p.below, (uint16_t)p.above);
    }
}

// twin.py:624-626: tracer x positions follow the window (all slots, as the
// reference shifts the whole position array).
__global__ void k_shift_tracers(float* pos, int max_tracers, float shift_m) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < max_tracers) pos[3 * t] = pos[3 * t] - shift_m;
}

}  // namespace

}  // namespace waam

using namespace waam;

#define REQUIRE(cond, msg) \
    if (!(cond)) return waam::fail(WAAM_ERR_INVALID, msg)

extern "C" {

int waam_shift_window_x(const WaamShiftPlane* planes, int n_planes, int n_shift, int nx, int ny,
                        int nz, int nz_solid, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "shift_window: bad dims");
    REQUIRE(planes && n_planes >= 0 && n_planes <= WAAM_MAX_SHIFT_PLANES,
            "shift_window: bad plane table");
    REQUIRE(n_shift >= 0, "shift_window: n_shift must be >= 0");
    ShiftTable t{};
    for (int q = 0; q < n_planes; ++q) {
        const WaamShiftPlane& p = planes[q];
        REQUIRE(p.ptr && (p.elem_bytes == 4 || p.elem_bytes == 2), "shift_window: bad plane");
        REQUIRE(p.mode >= WAAM_SHIFT_KEEP && p.mode <= WAAM_SHIFT_BY_K, "shift_window: bad mode");
        REQUIRE(((uintptr_t)p.ptr % (uintptr_t)p.elem_bytes) == 0, "shift_window: misaligned");
        t.p[q] = p;
    }
    if (n_planes == 0) return WAAM_OK;
    const int64_t cols = (int64_t)ny * nz;
    dim3 grid((unsigned)((cols + 255) / 256), (unsigned)n_planes);
    k_shift_window<<<grid, 256, 0, STREAM(stream)>>>(Dims{nx, ny, nz}, t, n_shift, nz_solid);
    return check_launch("k_shift_window");
}

int waam_shift_tracers_x(float* pos, int max_tracers, float shift_m, void* stream) {
    REQUIRE(pos && max_tracers >= 0, "shift_tracers: bad arguments");
    if (max_tracers == 0) return WAAM_OK;
    k_shift_tracers<<<(max_tracers + 255) / 256, 256, 0, STREAM(stream)>>>(pos, max_tracers,
                                                                          shift_m);
    return check_launch("k_shift_tracers");
}

}  // extern "C"
