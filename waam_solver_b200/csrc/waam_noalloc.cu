// Goldak arc-heat injection that allocates nothing: its reduction scratch
// (block partial sums, the last-block counter and the energy scalars) lives
// in a file-scope static device array instead of a caller workspace.
//
// Who needs it: a host that hands the library only its own input/output
// buffers and must not create device allocations after set-up -- for example
// an FFI host that owns no CUDA allocator, or a step loop running under a
// fixed device-memory budget where a cudaMalloc (or a torch caching-allocator
// growth) in the middle of a run is not acceptable.
//
// Limits and rules:
//  * the array holds kNoAllocMaxBlocks partial sums; one reduction block
//    covers kNoAllocCellsPerBlock cells, so grids above
//    kNoAllocMaxBlocks * kNoAllocCellsPerBlock = 16,777,216 cells are
//    rejected with WAAM_ERR_INVALID;
//  * every GPU that loads the library holds the array (about 66 KB) until
//    the process exits;
//  * all calls share the array: calls that overlap on the GPU (different
//    streams without ordering) race on it and must not be issued;
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it; make
//    that first call before any stream capture.
#include <cstdint>
#include <mutex>

#include "../../include/waam_b200.h"
#include "waam_common.cuh"
#include "waam_internal.cuh"

using namespace waam;

namespace {

constexpr int kNoAllocMaxBlocks = 8192;
constexpr int kNoAllocCellsPerBlock = 2048;  // 256 threads x 8 cells (grid-stride)
constexpr size_t kCounterBytes = 256;
constexpr size_t kScalarBytes = 256;
constexpr size_t kScratchBytes = kCounterBytes + kScalarBytes + kNoAllocMaxBlocks * sizeof(double);
constexpr int kMaxDevices = 64;

// Host code must not use this name as an address (it is a host-side stand-in);
// device code may name it directly.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Resolve (once per device, with that device current) the device address of
// the static scratch array.
int scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(WAAM_ERR_CUDA, "inject_goldak_heat_noalloc: cudaGetDevice failed");
    if (dev < 0 || dev >= kMaxDevices)
        return fail(WAAM_ERR_INVALID, "inject_goldak_heat_noalloc: device index out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (g_scratch_ptr[dev] == nullptr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            return fail(WAAM_ERR_CUDA, "inject_goldak_heat_noalloc: cudaGetSymbolAddress failed");
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return WAAM_OK;
}

// The counter must start at zero; partials and scalars are overwritten.
__global__ void k_noalloc_reset() {
    if (threadIdx.x == 0) *reinterpret_cast<unsigned*>(g_noalloc_scratch) = 0u;
}

}  // namespace

extern "C" int waam_inject_goldak_heat_noalloc(
    float* H, const int32_t* flags, const float* f_l, float* norm_buf, int nx, int ny, int nz,
    float arc_i, float arc_j, float arc_k, float Q_w, float dt, float dx3, float eta, float sign,
    float ff, float fr, float a_f, float a_r, float b, float c, float pen, int enable,
    void* stream) {
    if (!dims_ok(nx, ny, nz)) return fail(WAAM_ERR_INVALID, "inject_goldak_heat_noalloc: bad dims");
    if (!H || !flags || !f_l) return fail(WAAM_ERR_INVALID, "inject_goldak_heat_noalloc: null field");
    const int64_t n = (int64_t)nx * ny * nz;
    const int64_t blocks = (n + kNoAllocCellsPerBlock - 1) / kNoAllocCellsPerBlock;
    if (blocks > kNoAllocMaxBlocks)
        return fail(WAAM_ERR_INVALID,
                    "inject_goldak_heat_noalloc: grid exceeds the static scratch limit of "
                    "16777216 cells; use waam_inject_goldak_heat with a workspace");
    void* base = nullptr;
    int rc = scratch_address(&base);
    if (rc != WAAM_OK) return rc;
    char* bp = static_cast<char*>(base);
    Workspace ws;
    ws.counter = reinterpret_cast<unsigned*>(bp);
    ws.scalars = reinterpret_cast<float*>(bp + kCounterBytes);
    ws.partials = reinterpret_cast<double*>(bp + kCounterBytes + kScalarBytes);
    ws.field = nullptr;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);

    ArcParams p{};
    p.kind = 1;
    p.arc_i = arc_i;
    p.arc_j = arc_j;
    p.arc_k = arc_k;
    p.sign = sign;
    p.ff = ff;
    p.fr = fr;
    p.a_f = a_f;
    p.a_r = a_r;
    p.b = b;
    p.c = c;
    p.pen = pen;
    p.enable = enable;
    const float Qe_dt = Q_w * eta * dt;
    const Dims d{nx, ny, nz};

    k_noalloc_reset<<<1, 32, 0, s>>>();
    rc = check_launch("k_noalloc_reset");
    if (rc) return rc;
    k_arc_norm<<<(int)blocks, kThreads, 0, s>>>(d, flags, f_l, p, nullptr, 0.0f, Qe_dt, dx3,
                                                 norm_buf, ws.scalars, ws);
    rc = check_launch("k_arc_norm (no-alloc)");
    if (rc) return rc;
    PhaseParams unused{};
    k_arc_inject<<<elem_blocks(n), kThreads, 0, s>>>(d, H, flags, f_l, p, nullptr, 0.0f, ws.scalars,
                                                     0, unused);
    return check_launch("k_arc_inject (no-alloc)");
}
