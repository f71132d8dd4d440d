// Weighted-Jacobi V-cycle pressure solver with FP64 norms (see fx_vcycle.h).
//
// Per level k the cycle runs `pre` weighted sweeps, restricts 4 x the mean of
// the 8 fine residuals under each coarse voxel (the mean and the clamped
// children of pressure-restriction.wgsl.ts:27-50; the 4 rescales the unscaled
// 7-point operator to the doubled spacing), solves the coarse correction from
// zero, adds its trilinear prolongation (the sample position of
// pressure-prolongation.wgsl.ts:29-44) and runs `post` sweeps. The coarsest
// level runs `coarse` sweeps. Values are f32 and computed in the same order as
// the oracle, so the iterates agree bit for bit; the norms are FP64 sums whose
// order differs between the two, which matters only for a residual within
// rounding of the tolerance.
//
// The loop runs as a WHILE conditional node of the step's CUDA graph: the
// finalize kernel sets the condition from the FP64 residual, and it is 0 once
// max_cycles cycles have run, so the loop always ends.
#include <algorithm>
#include <cmath>

#include "fx_vcycle.h"

namespace fx {
namespace {

constexpr int kVZ = 4;

// dst = src + w ((sum of the 6 neighbours - rhs) / 6 - src) at interior voxels
// (dst = the Jacobi value when w is 1), 0 on the boundary. Warp layout of the
// fine sweep kernel: 32 consecutive x per warp, x neighbours by shuffles, z
// neighbours from a register column; the sum keeps the order +x, -x, +y, -y, +z, -z.
__global__ void __launch_bounds__(256) k_wjacobi(Dims dm, const float* __restrict__ rhs, const float* __restrict__ src, float* __restrict__ dst,
                                                 float w, int one) {
  const uint32_t lane = threadIdx.x;
  const uint32_t x = blockIdx.x * 32 + lane, y = blockIdx.y * 8 + threadIdx.y, z0 = blockIdx.z * kVZ;
  if (y >= dm.h) return;  // whole warp
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const bool xin = x < dm.w;
  const uint32_t base = (xin ? x : dm.w - 1) + dm.w * y;
  const bool yint = y > 0 && y < dm.h - 1;
  const bool xint = x > 0 && x < dm.w - 1;
  const int nz = min(kVZ, (int)dm.d - (int)z0);
  if (!yint) {
    if (xin)
      for (int k = 0; k < nz; ++k) dst[base + sz * (z0 + k)] = 0.0f;
    return;
  }
  float c[kVZ + 2], yp[kVZ], ym[kVZ], dv[kVZ], xe[kVZ];
  const bool left_end = lane == 0 && x > 0, right_end = (lane == 31 || x == dm.w - 1) && x + 1 < dm.w;
#pragma unroll
  for (int k = 0; k < kVZ + 2; ++k) {
    const int z = (int)z0 + k - 1;
    c[k] = (z >= 0 && z < (int)dm.d) ? __ldg(src + base + sz * (uint32_t)z) : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < kVZ; ++k) {
    const uint32_t z = min(z0 + k, dm.d - 1);
    const uint32_t i = base + sz * z;
    dv[k] = __ldg(rhs + i);
    yp[k] = __ldg(src + i + sy);
    ym[k] = __ldg(src + i - sy);
    xe[k] = 0.0f;
    if (left_end) xe[k] = __ldg(src + i - 1);
    if (right_end) xe[k] = __ldg(src + i + 1);
  }
#pragma unroll
  for (int k = 0; k < kVZ; ++k) {
    const float cm = c[k + 1];
    float xr = __shfl_down_sync(0xffffffffu, cm, 1);
    float xl = __shfl_up_sync(0xffffffffu, cm, 1);
    if (right_end) xr = xe[k];
    if (left_end) xl = xe[k];
    const uint32_t z = z0 + k;
    if (k >= nz || !xin) continue;
    float v = 0.0f;
    if (xint && z > 0 && z < dm.d - 1) {
      const float s = xr + xl + yp[k] + ym[k] + c[k + 2] + c[k];
      const float j = div6(s - dv[k]);
      v = one ? j : cm + w * (j - cm);
    }
    dst[base + sz * z] = v;
  }
}

FX_DEV float resid_at(const Dims& f, const float* __restrict__ rhs, const float* __restrict__ e, uint32_t x, uint32_t y, uint32_t z) {
  if (is_boundary(f, x, y, z)) return 0.0f;
  const uint32_t W1 = f.w - 1u, H1 = f.h - 1u, D1 = f.d - 1u;
  const uint32_t i = flat(f, x, y, z);
  const float s = __ldg(e + flat(f, inc(x, W1), y, z)) + __ldg(e + flat(f, dec(x), y, z)) + __ldg(e + flat(f, x, inc(y, H1), z)) +
                  __ldg(e + flat(f, x, dec(y), z)) + __ldg(e + flat(f, x, y, inc(z, D1))) + __ldg(e + flat(f, x, y, dec(z)));
  const float lap = s - __ldg(e + i) * 6.0f;
  return __ldg(rhs + i) - lap;
}

__global__ void __launch_bounds__(256) k_resid_restrict(Dims f, const float* __restrict__ rhs_f, const float* __restrict__ e_f, Dims c,
                                                        float* __restrict__ rhs_c) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y,
                 z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= c.w || y >= c.h || z >= c.d) return;
  const uint32_t i = flat(c, x, y, z);
  if (x == 0u || y == 0u || z == 0u || x == c.w - 1u || y == c.h - 1u || z == c.d - 1u) {
    rhs_c[i] = 0.0f;
    return;
  }
  float sum = 0.0f;
#pragma unroll
  for (uint32_t dz = 0; dz < 2; ++dz)
#pragma unroll
    for (uint32_t dy = 0; dy < 2; ++dy)
#pragma unroll
      for (uint32_t dx = 0; dx < 2; ++dx)
        sum += resid_at(f, rhs_f, e_f, min(2u * x + dx, f.w - 1u), min(2u * y + dy, f.h - 1u), min(2u * z + dz, f.d - 1u));
  rhs_c[i] = (sum * 0.125f) * 4.0f;
}

// dst = src + trilinear(ec) at interior fine voxels, dst = src on the boundary
// (src and dst may be the same buffer).
__global__ void __launch_bounds__(256) k_prolong_add(Dims c, const float* __restrict__ ec, Dims f, const float* src, float* dst) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y,
                 z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= f.w || y >= f.h || z >= f.d) return;
  const uint32_t i = flat(f, x, y, z);
  const float v = src[i];
  if (x == 0u || y == 0u || z == 0u || x == f.w - 1u || y == f.h - 1u || z == f.d - 1u) {
    dst[i] = v;
    return;
  }
  const float px = ((float)x + 0.5f) * 0.5f - 0.5f;
  const float py = ((float)y + 0.5f) * 0.5f - 0.5f;
  const float pz = ((float)z + 0.5f) * 0.5f - 0.5f;
  dst[i] = v + tri_interp(ec, tri_corners(c, px, py, pz));
}

__global__ void __launch_bounds__(256) k_fill0(float* __restrict__ p, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = 0.0f;
}

// Block sum of one double per thread into *acc (one atomic per block).
FX_DEV void block_sum_to(double v, double* acc) {
  __shared__ double part[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) part[warp] = v;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    v = lane < nw ? part[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) atomicAdd(acc, v);
  }
}

__global__ void __launch_bounds__(256) k_sumsq(const float* __restrict__ a, uint32_t n, double* acc) {
  double s = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = (double)__ldg(a + i);
    s += v * v;
  }
  block_sum_to(s, acc);
}

// Sum over interior voxels of (rhs - (sum of the 6 neighbours - 6 p))^2, each
// term in double from the stored f32 values.
__global__ void __launch_bounds__(256) k_resid_norm(Dims f, const float* __restrict__ rhs, const float* __restrict__ p, double* acc) {
  const uint32_t iw = f.w - 2u, ih = f.h - 2u, id = f.d - 2u;
  const uint32_t n = iw * ih * id;
  const uint32_t sy = f.w, sz = f.w * f.h;
  double s2 = 0.0;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const uint32_t x = 1u + t % iw, y = 1u + (t / iw) % ih, z = 1u + t / (iw * ih);
    const uint32_t i = flat(f, x, y, z);
    const double s = (double)__ldg(p + i + 1) + (double)__ldg(p + i - 1) + (double)__ldg(p + i + sy) + (double)__ldg(p + i - sy) +
                     (double)__ldg(p + i + sz) + (double)__ldg(p + i - sz);
    const double r = (double)__ldg(rhs + i) - (s - 6.0 * (double)__ldg(p + i));
    s2 += r * r;
  }
  block_sum_to(s2, acc);
}

// Takes the accumulated residual, counts the cycle, decides whether another
// cycle is due and hands the decision to the graph's WHILE node.
__global__ void k_finalize(SolverDev* st, double tol, int max_cycles, int count, cudaGraphConditionalHandle cond) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (count) st->cycles += 1;
  st->res2 = st->res2_acc;
  st->res2_acc = 0.0;
  const bool done = sqrt(st->res2) <= tol * sqrt(st->rhs2);
  st->converged = done ? 1 : 0;
  const int cont = (!done && st->cycles < max_cycles) ? 1 : 0;
  st->cont = cont;
  if (cond) cudaGraphSetConditional(cond, (unsigned)cont);
}

__global__ void __launch_bounds__(256) k_maxdiv(Dims dm, VelField v, unsigned long long* bits) {
  const uint32_t iw = dm.w - 2u, ih = dm.h - 2u, id = dm.d - 2u;
  const uint32_t n = iw * ih * id;
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  double m = 0.0;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const uint32_t x = 1u + t % iw, y = 1u + (t / iw) % ih, z = 1u + t / (iw * ih);
    const uint32_t i = flat(dm, x, y, z);
    const double ddx = (double)__ldg(v.c[0] + i + 1) - (double)__ldg(v.c[0] + i - 1);
    const double ddy = (double)__ldg(v.c[1] + i + sy) - (double)__ldg(v.c[1] + i - sy);
    const double ddz = (double)__ldg(v.c[2] + i + sz) - (double)__ldg(v.c[2] + i - sz);
    m = fmax(m, fabs(0.5 * (ddx + ddy + ddz)));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  // non-negative doubles order like their bit patterns
  if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(bits, (unsigned long long)__double_as_longlong(m));
}

inline uint32_t reduce_blocks() { return (uint32_t)device_sm_count() * 4u; }

inline dim3 vz_grid(Dims d) { return dim3((d.w + 31) / 32, (d.h + 7) / 8, (d.d + kVZ - 1) / kVZ); }
inline dim3 pt_grid(Dims d) { return dim3((d.w + 31) / 32, (d.h + 3) / 4, (d.d + 1) / 2); }
const dim3 kPtBlock(32, 4, 2);

inline uint32_t count_of(Dims d) { return d.w * d.h * d.d; }

void fill0(cudaStream_t s, float* p, Dims d) {
  const uint32_t n = count_of(d);
  k_fill0<<<std::min<uint32_t>((n + 255) / 256, reduce_blocks() * 2), 256, 0, s>>>(p, n);
}

int smooth(cudaStream_t s, const LevelBuf& B, int sweeps, int start, const VCycleConfig& c, uint32_t* launches) {
  int a = start;
  for (int k = 0; k < sweeps; ++k) {
    k_wjacobi<<<vz_grid(B.dm), dim3(32, 8, 1), 0, s>>>(B.dm, B.div, B.p[a], B.p[a ^ 1], c.omega, c.omega_one ? 1 : 0);
    a ^= 1;
    ++*launches;
  }
  return a;
}

int level_cycle(cudaStream_t s, const VCycleLevels& L, const VCycleConfig& c, int k, int start, uint32_t* launches) {
  const LevelBuf& B = L.lv[k];
  if (k == c.levels - 1) return smooth(s, B, c.coarse, start, c, launches);
  const int a = smooth(s, B, c.pre, start, c, launches);
  const LevelBuf& C = L.lv[k + 1];
  k_resid_restrict<<<pt_grid(C.dm), kPtBlock, 0, s>>>(B.dm, B.div, B.p[a], C.dm, C.div);
  fill0(s, C.p[0], C.dm);
  *launches += 2;
  const int ce = level_cycle(s, L, c, k + 1, 0, launches);
  const int b = ((c.pre + c.post) & 1) ? a ^ 1 : a;
  k_prolong_add<<<pt_grid(B.dm), kPtBlock, 0, s>>>(C.dm, C.p[ce], B.dm, B.p[a], B.p[b]);
  ++*launches;
  return smooth(s, B, c.post, b, c, launches);
}

}  // namespace

cudaError_t vcycle_prologue(cudaStream_t s, const VCycleLevels& L, const VCycleConfig& c, int start, SolverDev* st,
                            cudaGraphConditionalHandle cond) {
  const LevelBuf& F = L.lv[0];
  cudaError_t e = cudaMemsetAsync(st, 0, sizeof(SolverDev), s);
  if (e != cudaSuccess) return e;
  if (!c.warm) fill0(s, F.p[start], F.dm);
  k_sumsq<<<reduce_blocks(), 256, 0, s>>>(F.div, count_of(F.dm), &st->rhs2);
  k_resid_norm<<<reduce_blocks(), 256, 0, s>>>(F.dm, F.div, F.p[start], &st->res2_acc);
  k_finalize<<<1, 32, 0, s>>>(st, c.tol, c.max_cycles, 0, cond);
  return cudaGetLastError();
}

cudaError_t vcycle_body(cudaStream_t s, const VCycleLevels& L, const VCycleConfig& c, int start, SolverDev* st,
                        cudaGraphConditionalHandle cond, uint32_t* launches) {
  const LevelBuf& F = L.lv[0];
  const int fin = level_cycle(s, L, c, 0, start, launches);
  (void)fin;  // == start: the fine level ends in the buffer it started from
  k_resid_norm<<<reduce_blocks(), 256, 0, s>>>(F.dm, F.div, F.p[start], &st->res2_acc);
  k_finalize<<<1, 32, 0, s>>>(st, c.tol, c.max_cycles, 1, cond);
  *launches += 2;
  return cudaGetLastError();
}

cudaError_t solver_norms(cudaStream_t s, Dims dm, const float* div, const float* p, double tol, SolverDev* st) {
  cudaError_t e = cudaMemsetAsync(st, 0, sizeof(SolverDev), s);
  if (e != cudaSuccess) return e;
  k_sumsq<<<reduce_blocks(), 256, 0, s>>>(div, count_of(dm), &st->rhs2);
  k_resid_norm<<<reduce_blocks(), 256, 0, s>>>(dm, div, p, &st->res2_acc);
  k_finalize<<<1, 32, 0, s>>>(st, tol, 0, 0, 0);
  return cudaGetLastError();
}

cudaError_t max_divergence(cudaStream_t s, Dims dm, VelField v, SolverDev* st) {
  k_maxdiv<<<reduce_blocks(), 256, 0, s>>>(dm, v, &st->maxdiv_bits);
  return cudaGetLastError();
}

}  // namespace fx
