// noalloc_stage.cu — the pencil-sweep RK3 stage with library-owned scratch.
//
// flame_rk_stage_tiled with configuration 3 needs a scratch buffer from the caller (the
// right-hand-side accumulator and the sensor / mass-fraction arrays).  Some callers cannot
// provide one: a Julia program whose device memory all belongs to CUDA.jl's pool, or a serving
// loop that has committed its whole HBM budget up front, must not cudaMalloc behind its back,
// and a cudaMalloc issued while other work runs can synchronize the device.  For them this file
// keeps the scratch in a fixed array in device memory, created when the library's GPU code is
// loaded on a device and held until the process exits.
//
// Limits and rules (also stated in include/flame3d_b200.h):
//   * at most FLAME_NOALLOC_SCRATCH_BYTES of scratch, i.e. grids whose
//     flame_stage_scratch_bytes() fits; larger grids are rejected with FLAME_EINVAL;
//   * the first call on a device looks up the array's device address (cudaGetSymbolAddress) with
//     that device current, so it should be made before any stream capture; the address is cached
//     for the life of the process, so cudaDeviceReset between calls is not supported;
//   * every call on a device shares the one array, so calls that overlap on the GPU (different
//     streams, or different host threads) race and must be serialised by the caller;
//   * nothing in the array has to start at zero: each stage writes the accumulator and the
//     sensor arrays completely before it reads them, so the contents left by the previous call
//     are never used.

#include <mutex>

#include "common.cuh"

namespace {

constexpr size_t kScratchBytes = (size_t)FLAME_NOALLOC_SCRATCH_BYTES;

// The shared scratch.  Host code must not use this name as a pointer: on the host it stands for
// the symbol, not for device memory; its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_stage_scratch[kScratchBytes];

std::mutex g_mu;
void *g_addr[64] = {};  // device address of g_stage_scratch per device, once looked up

int scratch_address(void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return flame_fail(FLAME_ELAUNCH, "flame_rk_stage_noalloc: cudaGetDevice: %s",
                          cudaGetErrorString(e));
    if (dev < 0 || dev >= 64)
        return flame_fail(FLAME_EUNSUPPORTED, "flame_rk_stage_noalloc: device %d >= 64", dev);
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_stage_scratch);
        if (e != cudaSuccess || !p)
            return flame_fail(FLAME_ELAUNCH,
                              "flame_rk_stage_noalloc: cudaGetSymbolAddress on device %d: %s",
                              dev, cudaGetErrorString(e));
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return FLAME_OK;
}

}  // namespace

extern "C" int flame_rk_stage_noalloc(const FlameGrid *g, flame_stream_t s, int stage, double dt,
                                      const FlameStageBuffers *b, const FlameMetrics *m,
                                      const FlameThermo *th, const FlameTransport *tr,
                                      int precision) {
    if (int e = flame_check_grid(g, "flame_rk_stage_noalloc")) return e;
    if (!b) return flame_fail(FLAME_EINVAL, "flame_rk_stage_noalloc: NULL buffers");
    // the stage checks the rest; this one comes before the array's address lookup, so that a
    // grid no configuration takes is refused without touching the device
    if (g->nx < FLAME_NG || g->ny < FLAME_NG || g->nz < FLAME_NG)
        return flame_fail(FLAME_EINVAL, "flame_rk_stage_noalloc: extents must be >= %d", FLAME_NG);
    if (precision != 0 && precision != 1)
        return flame_fail(FLAME_EINVAL, "flame_rk_stage_noalloc: precision=%d must be 0 or 1",
                          precision);
    const size_t need = flame_stage_scratch_bytes(g, precision);
    if (need > kScratchBytes)
        return flame_fail(FLAME_EINVAL,
                          "flame_rk_stage_noalloc: this grid needs %zu bytes of scratch, more than "
                          "the %zu bytes the library holds; use flame_rk_stage_tiled with a "
                          "caller-owned scratch buffer",
                          need, kScratchBytes);
    void *scratch = nullptr;
    if (int e = scratch_address(&scratch)) return e;
    FlameStageBuffers bb = *b;
    bb.scratch = scratch;
    return flame_rk_stage_tiled(g, s, stage, dt, &bb, m, th, tr, precision, 3);
}
