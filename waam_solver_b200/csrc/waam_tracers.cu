// Porosity tracers: kernels.py:3182-3255 inject_tracers / advect_tracers.
//
// Spawning fills consecutive ring-buffer slots from the head pointer (the
// reference takes them with an atomic increment per particle; the set of
// slots is the same, the order fixed) at random offsets in a square of half
// width sigma around the torch.  The random numbers come from a counter-based
// hash of (seed, spawn index, component) -- the reference's ti.random() has no
// reproducible stream, so a seed makes runs repeatable instead.  Advection
// moves each active particle by the velocity of the cell it sits in
// (u * dx per step, nearest cell); a particle that leaves the grid or enters
// gas is dropped (active = 0), one in a solid or mushy cell is trapped
// (active = 2).
#include "../../include/waam_b200.h"
#include "waam_common.cuh"
#include "waam_internal.cuh"

namespace waam {

#define STREAM(s) reinterpret_cast<cudaStream_t>(s)

namespace {

// SplitMix64 finaliser: a bijective mix of a 64-bit counter.
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Uniform float in [0, 1) with 24 random bits.
__device__ __forceinline__ float uniform01(uint64_t seed, uint64_t index, int component) {
    const uint64_t h = mix64(seed ^ mix64(index * 2ull + (uint64_t)component));
    return (float)(uint32_t)(h >> 40) * (1.0f / 16777216.0f);
}

__global__ void k_inject_tracers(float* pos, int32_t* active, int32_t* head, int max_tracers,
                                 float arc_x, float arc_y, float arc_z, float sigma_m,
                                 int spawn_count, uint64_t seed) {
    __shared__ int base;
    if (threadIdx.x == 0) base = *head;
    __syncthreads();
    for (int t = threadIdx.x; t < spawn_count; t += blockDim.x) {
        const uint64_t index = (uint64_t)(uint32_t)base + (uint64_t)t;
        const int slot = (int)(index % (uint64_t)max_tracers);
        active[slot] = 1;
        const float rdx = (uniform01(seed, index, 0) * 2.0f - 1.0f) * sigma_m;
        const float rdy = (uniform01(seed, index, 1) * 2.0f - 1.0f) * sigma_m;
        pos[3 * slot + 0] = arc_x + rdx;
        pos[3 * slot + 1] = arc_y + rdy;
        pos[3 * slot + 2] = arc_z;
    }
    __syncthreads();
    if (threadIdx.x == 0) *head = base + spawn_count;
}

}  // namespace

__global__ void k_advect_tracers(Dims d, float* __restrict__ pos, int32_t* __restrict__ active,
                                 const float* __restrict__ ux, const float* __restrict__ uy,
                                 const float* __restrict__ uz, const float* __restrict__ f_l,
                                 const int32_t* __restrict__ flags, float dx, int max_tracers) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= max_tracers || active[p] != 1) return;
    float x = pos[3 * p], y = pos[3 * p + 1], z = pos[3 * p + 2];
    // ti.cast(f32 -> i32) truncates towards zero, as (int) does
    const int i = (int)(x / dx), j = (int)(y / dx), k = (int)(z / dx);
    if (i < 0 || i >= d.nx || j < 0 || j >= d.ny || k < 0 || k >= d.nz) {
        active[p] = 0;
        return;
    }
    const int c = d.idx(i, j, k);
    const int flag = flags[c];
    if (flag == GAS) {
        active[p] = 0;
        return;
    }
    if (f_l[c] < 0.05f || flag == SOLID) {
        active[p] = 2;
        return;
    }
    pos[3 * p] = x + ux[c] * dx;
    pos[3 * p + 1] = y + uy[c] * dx;
    pos[3 * p + 2] = z + uz[c] * dx;
}

int launch_advect_tracers(Dims d, float* pos, int32_t* active, const float* ux, const float* uy,
                          const float* uz, const float* f_l, const int32_t* flags, float dx,
                          int max_tracers, void* stream) {
    if (max_tracers <= 0) return WAAM_OK;
    k_advect_tracers<<<(max_tracers + kThreads - 1) / kThreads, kThreads, 0, STREAM(stream)>>>(
        d, pos, active, ux, uy, uz, f_l, flags, dx, max_tracers);
    return check_launch("k_advect_tracers");
}

}  // namespace waam

using namespace waam;

#define REQUIRE(cond, msg) \
    if (!(cond)) return waam::fail(WAAM_ERR_INVALID, msg)

extern "C" {

int waam_inject_tracers(float* pos, int32_t* active, int32_t* head, int max_tracers, float arc_x,
                        float arc_y, float arc_z, float sigma_m, int spawn_count, uint64_t seed,
                        void* stream) {
    REQUIRE(pos && active && head, "inject_tracers: null field");
    REQUIRE(max_tracers > 0 && spawn_count >= 0, "inject_tracers: bad counts");
    if (spawn_count == 0) return WAAM_OK;
    k_inject_tracers<<<1, 256, 0, STREAM(stream)>>>(pos, active, head, max_tracers, arc_x, arc_y,
                                                    arc_z, sigma_m, spawn_count, seed);
    return check_launch("k_inject_tracers");
}

int waam_advect_tracers(float* pos, int32_t* active, const float* ux, const float* uy,
                        const float* uz, const float* f_l, const int32_t* flags, int nx, int ny,
                        int nz, float dx, int max_tracers, void* stream) {
    REQUIRE(dims_ok(nx, ny, nz), "advect_tracers: bad dims");
    REQUIRE(pos && active && ux && uy && uz && f_l && flags, "advect_tracers: null field");
    REQUIRE(max_tracers >= 0, "advect_tracers: bad count");
    return launch_advect_tracers(Dims{nx, ny, nz}, pos, active, ux, uy, uz, f_l, flags, dx,
                                 max_tracers, stream);
}

}  // extern "C"
