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

// ---- phi = 0.5 surface (export/vtk_io.py:180-224) -----------------------------
// Point values on the (nx+1)(ny+1)(nz+1) lattice of cell corners: the mean of
// the cells that share the point (what VTK's cell_data_to_point_data does),
// for up to four fields.  Point index (I * (ny+1) + J) * (nz+1) + K.
struct FourPtrs {
    const float* c[4];
    float* p[4];
};

__global__ void k_cell_to_point(Dims d, FourPtrs f, int n_fields) {
    const int PX = d.nx + 1, PY = d.ny + 1, PZ = d.nz + 1;
    const int64_t np = (int64_t)PX * PY * PZ;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < np;
         q += (int64_t)gridDim.x * blockDim.x) {
        const int K = (int)(q % PZ);
        const int64_t r = q / PZ;
        const int J = (int)(r % PY), I = (int)(r / PY);
        float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        int cnt = 0;
        for (int i = I - 1; i <= I; ++i) {
            if (i < 0 || i >= d.nx) continue;
            for (int j = J - 1; j <= J; ++j) {
                if (j < 0 || j >= d.ny) continue;
                for (int k = K - 1; k <= K; ++k) {
                    if (k < 0 || k >= d.nz) continue;
                    const int64_t c = d.idx(i, j, k);
                    for (int m = 0; m < n_fields; ++m) acc[m] += f.c[m][c];
                    ++cnt;
                }
            }
        }
        for (int m = 0; m < n_fields; ++m) f.p[m][q] = acc[m] / (float)cnt;
    }
}

// Marching tetrahedra: each cube of eight lattice points is cut into the six
// tetrahedra around its 0-7 diagonal (corner bit 0 = +x, bit 1 = +y,
// bit 2 = +z), the same cut in every cube, so shared faces are triangulated
// alike and the surface is closed.  A tetrahedron with one (three) corners
// above iso yields one triangle, two corners two triangles.  Each triangle
// vertex is written with its edge key (lower point index * n_points + upper),
// its position and the interpolated point fields; triangles are numbered by
// an atomic counter and carry the sort key cube * 16 + tet * 2 + part, so the
// host restores a fixed order.  Triangles face from above-iso to below-iso.
__constant__ int kTets[6][4] = {{0, 1, 3, 7}, {0, 1, 5, 7}, {0, 2, 3, 7},
                                {0, 2, 6, 7}, {0, 4, 5, 7}, {0, 4, 6, 7}};

struct IsoOut {
    int64_t* keys;     // [3 * cap] edge keys
    float* vals;       // [3 * cap][6]: x, y, z, a0, a1, a2
    int64_t* order;    // [cap] sort keys
    unsigned long long* count;
    int64_t cap;
};

__device__ __forceinline__ void iso_vertex(const float* const* a, int na, const float* pos_a,
                                           const float* pos_b, int64_t pa, int64_t pb, float va,
                                           float vb, float iso, int64_t np, int64_t slot,
                                           const IsoOut& o) {
    const float t = (iso - va) / (vb - va);
    float* v = o.vals + slot * 6;
    for (int q = 0; q < 3; ++q) v[q] = pos_a[q] + t * (pos_b[q] - pos_a[q]);
    for (int m = 0; m < 3; ++m)
        v[3 + m] = m < na ? a[m][pa] + t * (a[m][pb] - a[m][pa]) : 0.0f;
    o.keys[slot] = pa < pb ? pa * np + pb : pb * np + pa;
}

__global__ void k_marching_tets(Dims d, const float* __restrict__ iso_f, FourPtrs attr, int na,
                                float iso, float h, float ox, float oy, float oz, IsoOut o) {
    const int PY = d.ny + 1, PZ = d.nz + 1;
    const int64_t np = (int64_t)(d.nx + 1) * PY * PZ;
    const int64_t ncube = (int64_t)d.nx * d.ny * d.nz;
    for (int64_t cube = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; cube < ncube;
         cube += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(cube % d.nz);
        const int64_t r = cube / d.nz;
        const int j = (int)(r % d.ny), i = (int)(r / d.ny);
        int64_t pid[8];
        float val[8];
        unsigned above = 0;
        for (int c = 0; c < 8; ++c) {
            pid[c] = ((int64_t)(i + (c & 1)) * PY + (j + ((c >> 1) & 1))) * PZ + (k + (c >> 2));
            val[c] = iso_f[pid[c]];
            if (val[c] > iso) above |= 1u << c;
        }
        if (above == 0 || above == 0xFFu) continue;
        float pos[8][3];
        for (int c = 0; c < 8; ++c) {
            pos[c][0] = ox + h * (float)(i + (c & 1));
            pos[c][1] = oy + h * (float)(j + ((c >> 1) & 1));
            pos[c][2] = oz + h * (float)(k + (c >> 2));
        }
        for (int t = 0; t < 6; ++t) {
            int in[4], out[4], ni = 0, no = 0;
            for (int q = 0; q < 4; ++q) {
                const int c = kTets[t][q];
                if ((above >> c) & 1u) in[ni++] = c; else out[no++] = c;
            }
            if (ni == 0 || ni == 4) continue;
            // triangles as corner pairs (above, below) per vertex
            int tri[2][3][2];
            int ntri;
            if (ni == 1) {
                for (int v = 0; v < 3; ++v) { tri[0][v][0] = in[0]; tri[0][v][1] = out[v]; }
                ntri = 1;
            } else if (ni == 3) {
                for (int v = 0; v < 3; ++v) { tri[0][v][0] = in[v]; tri[0][v][1] = out[0]; }
                ntri = 1;
            } else {
                // quad in[0]-out[0], in[0]-out[1], in[1]-out[1], in[1]-out[0]
                tri[0][0][0] = in[0]; tri[0][0][1] = out[0];
                tri[0][1][0] = in[0]; tri[0][1][1] = out[1];
                tri[0][2][0] = in[1]; tri[0][2][1] = out[1];
                tri[1][0][0] = in[0]; tri[1][0][1] = out[0];
                tri[1][1][0] = in[1]; tri[1][1][1] = out[1];
                tri[1][2][0] = in[1]; tri[1][2][1] = out[0];
                ntri = 2;
            }
            for (int m = 0; m < ntri; ++m) {
                const unsigned long long slot = atomicAdd(o.count, 1ull);
                if ((int64_t)slot >= o.cap) continue;
                float pv[3][3];
                for (int v = 0; v < 3; ++v) {
                    const int ca = tri[m][v][0], cb = tri[m][v][1];
                    const float tt = (iso - val[cb]) / (val[ca] - val[cb]);
                    for (int q = 0; q < 3; ++q)
                        pv[v][q] = pos[cb][q] + tt * (pos[ca][q] - pos[cb][q]);
                }
                // orientation: the normal points from above-iso to below-iso
                const float e1[3] = {pv[1][0] - pv[0][0], pv[1][1] - pv[0][1], pv[1][2] - pv[0][2]};
                const float e2[3] = {pv[2][0] - pv[0][0], pv[2][1] - pv[0][1], pv[2][2] - pv[0][2]};
                const float nrm[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                                      e1[0] * e2[1] - e1[1] * e2[0]};
                const int ca0 = tri[m][0][0], cb0 = tri[m][0][1];
                const float dir = nrm[0] * (pos[cb0][0] - pos[ca0][0]) +
                                  nrm[1] * (pos[cb0][1] - pos[ca0][1]) +
                                  nrm[2] * (pos[cb0][2] - pos[ca0][2]);
                int ord[3] = {0, 1, 2};
                if (dir < 0.0f) { ord[1] = 2; ord[2] = 1; }
                for (int v = 0; v < 3; ++v) {
                    const int ca = tri[m][ord[v]][0], cb = tri[m][ord[v]][1];
                    iso_vertex(attr.c, na, pos[cb], pos[ca], pid[cb], pid[ca], val[cb], val[ca],
                               iso, np, (int64_t)slot * 3 + v, o);
                }
                o.order[slot] = cube * 16 + t * 2 + m;
            }
        }
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

int waam_cell_to_point(const float* c0, const float* c1, const float* c2, const float* c3,
                       float* p0, float* p1, float* p2, float* p3, int nx, int ny, int nz,
                       void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "cell_to_point: bad dims");
    FourPtrs f{{c0, c1, c2, c3}, {p0, p1, p2, p3}};
    int n = 0;
    while (n < 4 && f.c[n]) {
        REQUIRE(f.p[n], "cell_to_point: null output");
        ++n;
    }
    REQUIRE(n >= 1, "cell_to_point: no field");
    const int64_t np = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
    k_cell_to_point<<<elem_blocks(np), kThreads, 0, STREAM(stream)>>>(Dims{nx, ny, nz}, f, n);
    return check_launch("k_cell_to_point");
}

int waam_isosurface(const float* iso_points, const float* a0, const float* a1, const float* a2,
                    int nx, int ny, int nz, float iso, float spacing, float ox, float oy,
                    float oz, int64_t* keys, float* vals, int64_t* order,
                    unsigned long long* count, int64_t capacity, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "isosurface: bad dims");
    REQUIRE(iso_points && keys && vals && order && count && capacity >= 0,
            "isosurface: null buffer");
    FourPtrs attr{{a0, a1, a2, nullptr}, {nullptr, nullptr, nullptr, nullptr}};
    int na = 0;
    while (na < 3 && attr.c[na]) ++na;
    IsoOut o{keys, vals, order, count, capacity};
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(unsigned long long), STREAM(stream));
    if (e != cudaSuccess) return waam::fail(WAAM_ERR_CUDA, cudaGetErrorString(e));
    const int64_t ncube = (int64_t)nx * ny * nz;
    k_marching_tets<<<elem_blocks(ncube), kThreads, 0, STREAM(stream)>>>(
        Dims{nx, ny, nz}, iso_points, attr, na, iso, spacing, ox, oy, oz, o);
    return check_launch("k_marching_tets");
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
