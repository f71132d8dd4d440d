// Brick flags of caller-owned scalar fields, with no device allocation.
//
// fx_brick_flags_noalloc computes the reference's active-brick flags
// (shaders/compute-active-bricks.wgsl.ts:35-58: a brick is active when one of its
// sample voxels, every second voxel along each axis, or its centre voxel has
// density + 0.7 temperature + 0.9 reaction above 0.012; an active brick whose
// peak exceeds 0.05, or whose centre exceeds 0.035, also flags its 26
// neighbours, clamped to the grid) for fields that the caller owns, on the
// caller's stream.
//
// Its callers are the ones that cannot allocate device memory at the time of
// the call. One is a frame loop that recomputes occupancy every frame: a
// cudaFree waits for all work on the device and would stall the frame. Another
// is a process whose device memory is fully reserved up front by its own arena:
// an allocation there fails or evicts. So the call allocates nothing. It makes no
// cudaMalloc, cudaFree or cudaMallocAsync call and uses no library routine that
// allocates, torch's included. The one scratch buffer it needs (a summary byte
// per brick between the two kernels) is the static device array below, which
// the driver places when it loads this library's module on a device.
//
// Limits and ordering:
//  - at most kNoAllocMaxBricks bricks (8^3 voxels each, ragged edges count as
//    bricks), i.e. 1 MiB of scratch; larger grids are rejected before any CUDA call;
//  - the first call on a device is its set-up: with that device current it looks
//    up the scratch address with cudaGetSymbolAddress, once per device. CUDA 12
//    loads modules lazily by default, so that first call is also when the module
//    (its code and the 1 MiB array) is loaded onto the device, and its first
//    launches load the two kernels. A caller that reserves the rest of the
//    device's memory up front makes one call (on any small grid) before it
//    reserves, or runs with CUDA_MODULE_LOADING=EAGER; later calls then take no
//    device memory at all. The first call should also come before any stream
//    capture;
//  - the scratch address is cached per device ordinal for the life of the
//    process. A cudaDeviceReset destroys the context that holds the array, so a
//    process that resets a device must not call this entry point on it again;
//  - launch errors are taken from the launches themselves (cudaLaunchKernel's
//    return value), so an error left pending by unrelated earlier work is neither
//    reported as this call's nor cleared;
//  - nothing has to start at zero: the summary kernel writes every scratch byte
//    that the dilation kernel reads, and the dilation kernel writes every flag;
//  - the scratch is one per device, so two calls in flight at once on one
//    device (different streams or host threads without ordering between them)
//    race. Calls on the same stream are ordered and safe.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/fenix_cuda.h"
#include "fx_math.cuh"

namespace fx {
void set_last_error(const std::string& msg);
}

namespace {

constexpr uint32_t kNoAllocMaxBricks = 1u << 20;
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) uint8_t g_noalloc_summary[kNoAllocMaxBricks];

std::mutex g_noalloc_mu;
void* g_noalloc_scratch[kNoAllocMaxDevices] = {};

// One warp per brick: lanes take the 64 sample voxels (local coordinates all
// even) two each, and every lane also evaluates the centre voxel. Writes
// bit 0 (active) and bit 1 (dilates) of the brick's summary byte.
__global__ void __launch_bounds__(256) k_noalloc_summary(fx::Dims dm, uint3 bc, const float* __restrict__ dens,
                                                        const float* __restrict__ temp, const float* __restrict__ reac,
                                                        uint8_t* __restrict__ summary) {
  const uint32_t nb = bc.x * bc.y * bc.z;
  const uint32_t b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (b >= nb) return;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t bx = b % bc.x, by = (b / bc.x) % bc.y, bz = b / (bc.x * bc.y);
  const uint32_t x0 = bx * 8u, y0 = by * 8u, z0 = bz * 8u;
  bool active = false, peak = false;
#pragma unroll
  for (uint32_t k = 0; k < 2; ++k) {
    const uint32_t s = lane + 32u * k;
    const uint32_t x = x0 + 2u * (s & 3u), y = y0 + 2u * ((s >> 2) & 3u), z = z0 + 2u * (s >> 4);
    if (x < dm.w && y < dm.h && z < dm.d) {
      const uint32_t i = fx::flat(dm, x, y, z);
      const float e = __ldg(dens + i) + __ldg(temp + i) * 0.7f + __ldg(reac + i) * 0.9f;
      active = active || e > 0.012f;
      peak = peak || e > 0.05f;
    }
  }
  const uint32_t ci = fx::flat(dm, min(x0 + 4u, dm.w - 1u), min(y0 + 4u, dm.h - 1u), min(z0 + 4u, dm.d - 1u));
  const float ce = __ldg(dens + ci) + __ldg(temp + ci) * 0.7f + __ldg(reac + ci) * 0.9f;
  active = active || ce > 0.012f;
  peak = peak || ce > 0.05f;
  const bool any_active = __any_sync(0xffffffffu, active);
  const bool dilates = __any_sync(0xffffffffu, peak) || ce > 0.035f;
  if (lane == 0) summary[b] = any_active ? (uint8_t)(1u | (dilates ? 2u : 0u)) : (uint8_t)0u;
}

// flags[b] = active[b] || any neighbour within Chebyshev distance 1 that is
// active and dilates (the gather form of the reference's clamped scatter).
__global__ void __launch_bounds__(256) k_noalloc_dilate(uint3 bc, const uint8_t* __restrict__ summary, uint32_t* __restrict__ flags) {
  const uint32_t nb = bc.x * bc.y * bc.z;
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const uint32_t bx = b % bc.x, by = (b / bc.x) % bc.y, bz = b / (bc.x * bc.y);
  bool flag = (summary[b] & 1u) != 0u;
  const uint32_t zlo = bz ? bz - 1 : 0, zhi = min(bz + 1, bc.z - 1);
  const uint32_t ylo = by ? by - 1 : 0, yhi = min(by + 1, bc.y - 1);
  const uint32_t xlo = bx ? bx - 1 : 0, xhi = min(bx + 1, bc.x - 1);
  for (uint32_t z = zlo; z <= zhi && !flag; ++z)
    for (uint32_t y = ylo; y <= yhi && !flag; ++y)
      for (uint32_t x = xlo; x <= xhi && !flag; ++x) flag = summary[x + bc.x * (y + bc.y * z)] == 3u;
  flags[b] = flag ? 1u : 0u;
}

fx_status noalloc_fail(fx_status code, const std::string& msg) {
  fx::set_last_error("fx_brick_flags_noalloc: " + msg);
  return code;
}

}  // namespace

extern "C" fx_status fx_brick_flags_noalloc(const float* density, const float* temperature, const float* reaction, uint32_t width,
                                            uint32_t height, uint32_t depth, uint32_t* flags, void* stream) {
  if (!density || !temperature || !reaction || !flags) return noalloc_fail(FX_ERR_INVALID_ARGUMENT, "NULL buffer");
  if (width == 0 || height == 0 || depth == 0) return noalloc_fail(FX_ERR_INVALID_ARGUMENT, "every dimension must be >= 1");
  const uint64_t bcx = (width + 7ull) / 8ull, bcy = (height + 7ull) / 8ull, bcz = (depth + 7ull) / 8ull;
  const uint64_t nb = bcx * bcy * bcz;
  if (nb > kNoAllocMaxBricks)
    return noalloc_fail(FX_ERR_INVALID_ARGUMENT, "the grid has " + std::to_string(nb) + " bricks; the static scratch holds at most " +
                                                     std::to_string(kNoAllocMaxBricks) + " (1 MiB, one byte per 8^3 brick)");
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(FX_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return noalloc_fail(FX_ERR_UNSUPPORTED, "device ordinal beyond the per-device scratch table");
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_scratch[dev]) {
      e = cudaGetSymbolAddress(&g_noalloc_scratch[dev], g_noalloc_summary);
      if (e != cudaSuccess) {
        g_noalloc_scratch[dev] = nullptr;
        return noalloc_fail(FX_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      }
    }
    scratch = g_noalloc_scratch[dev];
  }
  const fx::Dims dm{width, height, depth};
  const uint3 bc = make_uint3((uint32_t)bcx, (uint32_t)bcy, (uint32_t)bcz);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const uint32_t n = (uint32_t)nb;
  uint8_t* summary = static_cast<uint8_t*>(scratch);
  const uint8_t* summary_in = summary;
  void* sum_args[] = {(void*)&dm, (void*)&bc, (void*)&density, (void*)&temperature, (void*)&reaction, (void*)&summary};
  e = cudaLaunchKernel((const void*)k_noalloc_summary, dim3((n + 7u) / 8u), dim3(256), sum_args, 0, s);
  if (e != cudaSuccess) return noalloc_fail(FX_ERR_CUDA, std::string("summary launch: ") + cudaGetErrorString(e));
  void* dil_args[] = {(void*)&bc, (void*)&summary_in, (void*)&flags};
  e = cudaLaunchKernel((const void*)k_noalloc_dilate, dim3((n + 255u) / 256u), dim3(256), dil_args, 0, s);
  if (e != cudaSuccess) return noalloc_fail(FX_ERR_CUDA, std::string("dilation launch: ") + cudaGetErrorString(e));
  return FX_OK;
}
