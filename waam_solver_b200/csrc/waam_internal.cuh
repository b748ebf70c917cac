// Internal declarations shared by the CUDA translation units.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "waam_common.cuh"

namespace waam {

constexpr int kThreads = 256;
constexpr int kMaxElemBlocks = 148 * 16;  // grid-stride cap: 16 CTAs per SM
constexpr int kRedBlocks = 592;           // fixed so reduction order never depends on the GPU

// Caller-provided workspace layout (waam_workspace_bytes):
//   [0, 512)            unsigned counters: [0] last-block reduction,
//                       [kActiveShardSlot, +kActiveShards) active-cell counts per shard
//   [512, 1024)         float scalars of the operator-level reductions
//   [1024, 132096)      double partial sums, one per reduction block (<= 16384)
//   [132096, ...)       one field-sized scratch (n + kFieldSlack elements): a float
//                       snapshot (operator API) or the int32 active-cell list (fused step)
//   [ws_shape_offset(n), +4n)  the fused step's arc shape factors
constexpr size_t kWsScalarsOffset = 512;
constexpr size_t kWsPartialsOffset = 1024;
constexpr int kWsMaxPartials = 16384;
constexpr size_t kWsFieldOffset = kWsPartialsOffset + kWsMaxPartials * sizeof(double);
constexpr int64_t kFieldSlack = 65536;
constexpr int kActiveShards = 64;     // power of two

inline size_t ws_field_bytes(int64_t n) {
    size_t field = (size_t)((n > 0 ? n : 0) + kFieldSlack) * sizeof(float);
    return (field + 255) & ~(size_t)255;
}
// a second field-sized region after the first: the arc pass's per-cell shape
// factors (so they never share memory with the active-cell list a pending
// collision still reads)
inline size_t ws_shape_offset(int64_t n) { return kWsFieldOffset + ws_field_bytes(n); }
inline size_t ws_total_bytes(int64_t n) {
    size_t shape = ((size_t)(n > 0 ? n : 0) * sizeof(float) + 255) & ~(size_t)255;
    return ws_shape_offset(n) + shape;
}
constexpr int kActiveShardSlot = 64;  // first shard counter in the counter block

// Cell tiles of the stencil kernels: 32 (k) x 8 (j) threads, one grid z-slice
// per i, so a cell's coordinates come from the launch geometry without
// integer division and consecutive lanes touch consecutive k (coalesced).
constexpr int kTileK = 32;
constexpr int kTileJ = 8;

inline dim3 tile_grid(const Dims& d) {
    return dim3((d.nz + kTileK - 1) / kTileK, (d.ny + kTileJ - 1) / kTileJ, d.nx);
}
inline dim3 tile_block() { return dim3(kTileK, kTileJ, 1); }

__device__ __forceinline__ bool tile_cell(const Dims& d, int& i, int& j, int& k, int& c) {
    k = blockIdx.x * kTileK + threadIdx.x;
    j = blockIdx.y * kTileJ + threadIdx.y;
    i = blockIdx.z;
    if (k >= d.nz || j >= d.ny) return false;
    c = (i * d.ny + j) * d.nz + k;
    return true;
}

// Tile numbering of the quiet-tile lists: t = (i * tiles_j + j / kTileJ) *
// tiles_k + k / kTileK (WaamFields.tile_bits / tile_list).
__host__ __device__ inline int tiles_k(const Dims& d) { return (d.nz + kTileK - 1) / kTileK; }
__host__ __device__ inline int tiles_j(const Dims& d) { return (d.ny + kTileJ - 1) / kTileJ; }
__host__ __device__ inline int64_t tile_total(const Dims& d) {
    return (int64_t)tiles_k(d) * tiles_j(d) * d.nx;
}

// Work-list entries pack a tile as (i << 16) | (j / kTileJ << 6) | k / kTileK, so
// the list kernels decode them with shifts; quiet-tile skipping therefore
// needs tiles_k <= 64 and tiles_j <= 1024 (nz <= 2048, ny <= 8192).
__host__ __device__ inline bool tiles_packable(const Dims& d) {
    return tiles_k(d) <= 64 && tiles_j(d) <= 1024 && d.nx <= 65535;
}
__host__ __device__ inline int pack_tile(int i, int jt, int kt) { return (i << 16) | (jt << 6) | kt; }
__host__ __device__ inline int64_t tile_index(const Dims& d, int e) {
    return ((int64_t)(e >> 16) * tiles_j(d) + ((e >> 6) & 1023)) * tiles_k(d) + (e & 63);
}

// The cell of this thread (threadIdx.x along k, threadIdx.y along j) in the
// tile of packed work-list entry e.
__device__ __forceinline__ bool list_tile_cell(const Dims& d, int e, int& i, int& j, int& k,
                                               int& c) {
    k = (e & 63) * kTileK + threadIdx.x;
    j = ((e >> 6) & 1023) * kTileJ + threadIdx.y;
    i = e >> 16;
    if (k >= d.nz || j >= d.ny) return false;
    c = (i * d.ny + j) * d.nz + k;
    return true;
}

// This block's share of the first cnt work-list entries (blockIdx.x, then every
// gridDim.x-th), handed to f(entry) one after the other; the next entry is
// requested before f works the current one, so that its load overlaps.
template <class F>
__device__ __forceinline__ void for_list_tiles(const int32_t* __restrict__ list, int cnt, F f) {
    int e = blockIdx.x;
    int ent = e < cnt ? list[1 + e] : -1;
    while (e < cnt) {
        const int e2 = e + (int)gridDim.x;
        const int ent2 = e2 < cnt ? list[1 + e2] : -1;
        f(ent);
        e = e2;
        ent = ent2;
    }
}

// Slots of the fused step's device scalars (WaamFields::step_scalars).
constexpr int kScalarArcK = 0;   // resolved arc k (written by the surface query)
constexpr int kScalarWsum = 1;   // arc weight sum
constexpr int kScalarEpw = 2;    // energy per unit weight
constexpr int kScalarArcI = 4;   // torch x in cells (copied in by the host every step)
constexpr int kScalarArcJ = 5;   // torch y in cells
// the arc position of the step as its collision sees it, copied by the column
// pass: a collision left pending for the next step's first stages must not
// see that step's position (slots 0, 4, 5 are rewritten by then)
constexpr int kScalarCollideArcK = 8;
constexpr int kScalarCollideArcI = 9;
constexpr int kScalarCollideArcJ = 10;

struct Workspace {
    unsigned* counter;        // counter[0]: reduction, counter[kActiveCountSlot]: active cells
    double* partials;
    float* scalars;
    float* field;
    static Workspace at(void* base) {
        char* b = static_cast<char*>(base);
        Workspace w;
        w.counter = reinterpret_cast<unsigned*>(b);
        w.partials = reinterpret_cast<double*>(b + kWsPartialsOffset);
        w.scalars = reinterpret_cast<float*>(b + kWsScalarsOffset);
        w.field = reinterpret_cast<float*>(b + kWsFieldOffset);
        return w;
    }
};

int fail(int code, const char* what);
int check_launch(const char* what);
int elem_blocks(int64_t n);
int red_blocks(int64_t n);
bool dims_ok(int nx, int ny, int nz);
bool workspace_ok(void* ws, size_t bytes, int64_t n);

__global__ void k_arc_norm(Dims d, const int32_t* __restrict__ flags, const float* __restrict__ f_l,
                           ArcParams p, const float* arc_k_dev, float arc_k_offset, float Qe_dt,
                           float dx3, float* norm_out, float* scalars, Workspace ws);
__global__ void k_arc_inject(Dims d, float* __restrict__ H, const int32_t* __restrict__ flags,
                             const float* __restrict__ f_l, ArcParams p, const float* arc_k_dev,
                             float arc_k_offset, const float* scalars, int cap, PhaseParams ph);

int launch_contact_columns(Dims d, const float* snap, float* phi, const int32_t* flags,
                           float theta, void* stream);
int launch_stream(Dims d, const float* f_src, float* f_dst, const int32_t* flags, void* stream);
int launch_advect_tracers(Dims d, float* pos, int32_t* active, const float* ux, const float* uy,
                          const float* uz, const float* f_l, const int32_t* flags, float dx,
                          int max_tracers, void* stream);
// Droplet deposition with up to WAAM_DEPOSIT_MAX_TRIES footprint radii; attempt
// t > 0 runs only while the converted volume is below accept_volume.
int launch_deposit(Dims d, void* f_src, int f_storage, int32_t* flags, float* f_l, float* phi,
                   float* H, float* T, float* rho, float arc_i, float arc_j, float arc_k,
                   const float* foot_radii, int n_tries, double accept_volume, float drop_r,
                   float target_vol, float T_drop, float cp_rho, float L_rho, float rho0,
                   float* vol_acc, float* real_acc, float cell_vol, void* stream);

}  // namespace waam
