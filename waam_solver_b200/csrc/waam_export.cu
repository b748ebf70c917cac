// Export fields (export/vtk_io.py:62-166; kernels.py:3354-3418).
//
// The derived fields (VOF curvature, vorticity magnitude) are per-cell
// stencils.  The volume export gathers every requested array, already in the
// physical units the VTK file carries and already in VTK cell order (x
// fastest), into one staging buffer with a single launch, so the host makes
// one device-to-host copy and writes it out unchanged.  The reorder is a
// 32 x 32 shared-memory transpose of each (i, k) tile of a j plane: reads are
// coalesced along k (the grid's fastest index), writes along i (VTK's).
#include "../../include/waam_b200.h"
#include "waam_common.cuh"
#include "waam_internal.cuh"

namespace waam {

#define STREAM(s) reinterpret_cast<cudaStream_t>(s)

namespace {

// kernels.py:3354-3376 compute_curvature_field
__global__ void k_curvature_field(Dims d, const float* __restrict__ phi,
                                  const int32_t* __restrict__ flags, float* __restrict__ kappa) {
    int i, j, k, c;
    if (!tile_cell(d, i, j, k, c)) return;
    float out = 0.0f;
    if (flags[c] != GAS && !(i < 1 || j < 1 || k < 1 || i > d.nx - 2 || j > d.ny - 2 ||
                             k > d.nz - 2)) {
        float g0;
        const float kv = brackbill_kappa(d, phi, i, j, k, g0);
        if (g0 >= 1e-6f) out = kv;
    }
    kappa[c] = out;
}

// kernels.py:3379-3418 compute_vorticity_magnitude (physical 1/s)
__global__ void k_vorticity(Dims d, const float* __restrict__ ux, const float* __restrict__ uy,
                            const float* __restrict__ uz, const int32_t* __restrict__ flags,
                            float* __restrict__ vort, float scale) {
    int i, j, k, c;
    if (!tile_cell(d, i, j, k, c)) return;
    float out = 0.0f;
    if (flags[c] != GAS) {
        const int ip = imin(i + 1, d.nx - 1), im = imax(i - 1, 0);
        const int jp = imin(j + 1, d.ny - 1), jm = imax(j - 1, 0);
        const int kp = imin(k + 1, d.nz - 1), km = imax(k - 1, 0);
        const float duz_dy = 0.5f * (uz[d.idx(i, jp, k)] - uz[d.idx(i, jm, k)]);
        const float duy_dz = 0.5f * (uy[d.idx(i, j, kp)] - uy[d.idx(i, j, km)]);
        const float dux_dz = 0.5f * (ux[d.idx(i, j, kp)] - ux[d.idx(i, j, km)]);
        const float duz_dx = 0.5f * (uz[d.idx(ip, j, k)] - uz[d.idx(im, j, k)]);
        const float duy_dx = 0.5f * (uy[d.idx(ip, j, k)] - uy[d.idx(im, j, k)]);
        const float dux_dy = 0.5f * (ux[d.idx(i, jp, k)] - ux[d.idx(i, jm, k)]);
        const float wx = (duz_dy - duy_dz) * scale;
        const float wy = (dux_dz - duz_dx) * scale;
        const float wz = (duy_dx - dux_dy) * scale;
        out = sqrtf(wx * wx + wy * wy + wz * wz);
    }
    vort[c] = out;
}

struct ChannelTable {
    WaamExportChannel ch[WAAM_MAX_EXPORT_CHANNELS];
};

// One channel value at grid cell c (numpy float32 order of vtk_io.py).
__device__ __forceinline__ uint32_t channel_value(const WaamExportChannel& ch, int64_t c) {
    const float* s0 = static_cast<const float*>(ch.src[0]);
    switch (ch.op) {
        case WAAM_EXPORT_COPY:
        case WAAM_EXPORT_COPY_I32:
            return static_cast<const uint32_t*>(ch.src[0])[c];
        case WAAM_EXPORT_ADD:
            return __float_as_uint(s0[c] + ch.a);
        case WAAM_EXPORT_NEG:
            return __float_as_uint(-s0[c]);
        case WAAM_EXPORT_LU_VEL:   // u * dx / dt
            return __float_as_uint((s0[c] * ch.a) / ch.b);
        case WAAM_EXPORT_LU_ACC:   // F * dx / dt / dt
            return __float_as_uint(((s0[c] * ch.a) / ch.b) / ch.b);
        case WAAM_EXPORT_SPEED:
        case WAAM_EXPORT_ACC_MAG: {
            float v[3];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const float x = static_cast<const float*>(ch.src[q])[c];
                v[q] = (x * ch.a) / ch.b;
                if (ch.op == WAAM_EXPORT_ACC_MAG) v[q] = v[q] / ch.b;
            }
            return __float_as_uint(sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
        }
        case WAAM_EXPORT_PRESSURE:  // (rho - 1) * cs2 * rho_phys * (dx / dt)^2
            return __float_as_uint((((s0[c] - 1.0f) * ch.a) * ch.b) * ch.c);
        case WAAM_EXPORT_MUSHY: {
            const float fl = s0[c];
            return __float_as_uint((fl > 0.05f && fl < 0.95f) ? 1.0f : 0.0f);
        }
        default:
            return 0u;
    }
}

// blockIdx.x: i tile, blockIdx.y: k tile, blockIdx.z: j; threads 32 x 8.
__global__ void __launch_bounds__(256) k_export_pack(Dims d, const __grid_constant__ ChannelTable T,
                                                     int n_channels, uint32_t* __restrict__ out) {
    __shared__ uint32_t tile[32][33];
    const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32, j = blockIdx.z;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int64_t n = d.n();
    for (int ch = 0; ch < n_channels; ++ch) {
        const WaamExportChannel& C = T.ch[ch];
#pragma unroll
        for (int r = 0; r < 32; r += 8) {
            const int i = i0 + r + ty, k = k0 + tx;
            if (i < d.nx && k < d.nz) tile[r + ty][tx] = channel_value(C, d.idx(i, j, k));
        }
        __syncthreads();
        uint32_t* o = out + (int64_t)ch * n;
#pragma unroll
        for (int r = 0; r < 32; r += 8) {
            const int k = k0 + r + ty, i = i0 + tx;
            if (i < d.nx && k < d.nz)
                o[i + (int64_t)d.nx * (j + (int64_t)d.ny * k)] = tile[tx][r + ty];
        }
        __syncthreads();
    }
}

}  // namespace

}  // namespace waam

using namespace waam;

#define REQUIRE(cond, msg) \
    if (!(cond)) return waam::fail(WAAM_ERR_INVALID, msg)

extern "C" {

int waam_compute_curvature_field(const float* phi, const int32_t* flags, float* kappa_out, int nx,
                                 int ny, int nz, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "curvature_field: bad dims");
    REQUIRE(phi && flags && kappa_out, "curvature_field: null field");
    Dims d{nx, ny, nz};
    k_curvature_field<<<tile_grid(d), tile_block(), 0, STREAM(stream)>>>(d, phi, flags, kappa_out);
    return check_launch("k_curvature_field");
}

int waam_compute_vorticity_magnitude(const float* ux, const float* uy, const float* uz,
                                     const int32_t* flags, float* vort_out, int nx, int ny, int nz,
                                     float dx, float dt, void* stream) {
    (void)dx;
    REQUIRE(dims_ok(nx, ny, nz), "vorticity: bad dims");
    REQUIRE(ux && uy && uz && flags && vort_out, "vorticity: null field");
    Dims d{nx, ny, nz};
    const float scale = 1.0f / (dt + 1e-12f);
    k_vorticity<<<tile_grid(d), tile_block(), 0, STREAM(stream)>>>(d, ux, uy, uz, flags, vort_out,
                                                                   scale);
    return check_launch("k_vorticity");
}

int waam_export_pack(const WaamExportChannel* channels, int n_channels, int nx, int ny, int nz,
                     void* out, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "export_pack: bad dims");
    REQUIRE(channels && out && n_channels >= 0 && n_channels <= WAAM_MAX_EXPORT_CHANNELS,
            "export_pack: bad channel table");
    ChannelTable t{};
    for (int q = 0; q < n_channels; ++q) {
        const WaamExportChannel& c = channels[q];
        REQUIRE(c.op >= WAAM_EXPORT_COPY && c.op <= WAAM_EXPORT_MUSHY, "export_pack: bad op");
        const int nsrc = (c.op == WAAM_EXPORT_SPEED || c.op == WAAM_EXPORT_ACC_MAG) ? 3 : 1;
        for (int s = 0; s < nsrc; ++s) REQUIRE(c.src[s], "export_pack: null source");
        t.ch[q] = c;
    }
    if (n_channels == 0) return WAAM_OK;
    Dims d{nx, ny, nz};
    dim3 grid((unsigned)((nx + 31) / 32), (unsigned)((nz + 31) / 32), (unsigned)ny);
    k_export_pack<<<grid, dim3(32, 8), 0, STREAM(stream)>>>(d, t, n_channels,
                                                            static_cast<uint32_t*>(out));
    return check_launch("k_export_pack");
}

}  // extern "C"
