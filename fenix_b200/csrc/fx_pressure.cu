// Fine-level pressure passes of the fused path: up to four Jacobi sweeps
// (pressure-jacobi.wgsl.ts:15-36) temporally blocked on chip, with the
// divergence (compute-divergence.wgsl.ts:22-42), the fine->mid restriction
// (pressure-restriction.wgsl.ts:27-50), the mid->fine prolongation
// (pressure-prolongation.wgsl.ts:29-44) and the projection
// (project-velocity.wgsl.ts:21-43) fused where the reference runs them next to
// the sweeps.
//
// A block owns a TX x TY column of the grid and marches along z through a chunk
// of planes. Stage 0 is the pass input and stage j the j-th sweep; stage j at
// plane z needs stage j-1 at planes z-1..z+1, so stage j runs j planes behind
// the input (one more when the divergence is computed in the block). Each thread
// owns fixed (x, y) positions of a frame = the column widened by H voxels (H =
// number of stencil stages after stage 0). For its positions it keeps every
// stage's last three planes in registers (the z neighbours) and publishes the
// newest plane to a double-buffered shared plane (the x and y neighbours).
// Stage j is valid on the frame shrunk by j, which is all the next stage needs.
// A stage at clock t reads only planes published at clock t-1, so one barrier
// per plane suffices.
//
// Every value is computed with the reference's operations in its order: the
// result equals the sweep-by-sweep evaluation bit for bit. The division by 6 is
// the exact IEEE quotient (div6, fx_math.cuh).
#include <algorithm>
#include <cstdlib>

#include "fx_fused.h"
#include "fx_pressure.h"

namespace fx {
namespace {

constexpr int TX = 32, TY = 16, NT = TX * TY;

// Integer tuning knob from the environment (defaults come from measurement).
int env_int(const char* name, int dflt, int lo, int hi) {
  const char* v = std::getenv(name);
  if (!v || !*v) return dflt;
  const int x = std::atoi(v);
  return (x >= lo && x <= hi) ? x : dflt;
}

enum { IN_ZERO = 0, IN_BUF = 1, IN_BUF_PROLONG = 2, IN_ZERO_PROLONG = 3 };

struct ZArgs {
  Dims dm;
  Dims mid;
  int zchunk;
  const float* p_in;
  const float* div_in;
  float* div_out;
  float* mid_div;
  const float* mid_p;
  float* p_out;
  VelField vfin;
  VelField vcur;
  float* vmag;
  int write_vmag;
  int restrict_mid;
};

// Prolongation term of pressure-prolongation.wgsl.ts:42-43 at fine voxel (x,y,z).
FX_DEV float prolong_sample(const Dims& mid, const float* __restrict__ mp, int x, int y, int z) {
  const float px = ((float)x + 0.5f) * 0.5f - 0.5f;
  const float py = ((float)y + 0.5f) * 0.5f - 0.5f;
  const float pz = ((float)z + 0.5f) * 0.5f - 0.5f;
  return tri_interp(mp, tri_corners(mid, px, py, pz));
}

template <int S, int IN, bool DIVV, bool PROJ>
struct Frame {
  static constexpr int H = S + (PROJ ? 1 : 0);
  static constexpr int EX = TX + 2 * H;
  static constexpr int EY = TY + 2 * H;
  static constexpr int P = EX * EY;
  static constexpr int RP = (P + NT - 1) / NT;
  static constexpr bool stage0 = IN != IN_ZERO;
  static constexpr int first = stage0 ? 0 : 1;  // first stage held in registers
  // Shared planes (P floats each): 2 per published stage (stages first..S-1, and
  // S when projecting), 2 each for vx and vy and 3 for the divergence when it is
  // computed in the block.
  static constexpr int pub_last = PROJ ? S : S - 1;
  static constexpr int npub = pub_last >= first ? pub_last - first + 1 : 0;
  static constexpr int floats = P * (2 * npub + (DIVV ? 7 : 0));
};

template <int S, int IN, bool DIVV, bool PROJ>
__global__ void __launch_bounds__(NT, 1) k_zjacobi(ZArgs a) {
  using Fr = Frame<S, IN, DIVV, PROJ>;
  constexpr int H = Fr::H, EX = Fr::EX, EY = Fr::EY, P = Fr::P, RP = Fr::RP;
  constexpr int dl = DIVV ? 1 : 0;
  constexpr int L = S + (PROJ ? 1 : 0);
  extern __shared__ float sm[];
  const Dims dm = a.dm;
  const int W = (int)dm.w, Hh = (int)dm.h, D = (int)dm.d;
  const int tid = threadIdx.x + TX * threadIdx.y;
  const int gx0 = (int)blockIdx.x * TX - H, gy0 = (int)blockIdx.y * TY - H;
  const int za = (int)blockIdx.z * a.zchunk;
  const int zb = min(za + a.zchunk, D);
  const size_t plane = (size_t)W * (size_t)Hh;

  // shared planes
  auto pub = [&](int j, int buf) -> float* { return sm + ((j - Fr::first) * 2 + buf) * P; };
  float* vxs = sm + 2 * Fr::npub * P;  // [2][P]
  float* vys = vxs + 2 * P;            // [2][P]
  float* dvs = vys + 2 * P;            // [3][P]

  // per-position constants
  int pidx[RP], dist[RP], gxr[RP], gyr[RP], gxy[RP];
  bool valid[RP], indom[RP], xyint[RP];
#pragma unroll
  for (int r = 0; r < RP; ++r) {
    const int p = tid + NT * r;
    valid[r] = p < P;
    const int lx = p % EX, ly = p / EX;
    pidx[r] = p;
    dist[r] = min(min(lx, EX - 1 - lx), min(ly, EY - 1 - ly));
    const int gx = gx0 + lx, gy = gy0 + ly;
    indom[r] = valid[r] && gx >= 0 && gy >= 0 && gx < W && gy < Hh;
    xyint[r] = valid[r] && gx > 0 && gy > 0 && gx < W - 1 && gy < Hh - 1;
    gxy[r] = indom[r] ? gx + W * gy : 0;
    gxr[r] = gx;
    gyr[r] = gy;
  }
  for (int k = tid; k < Fr::floats; k += NT) sm[k] = 0.0f;

  // register rings: ring[j][r][0..2] = stage j at planes q_j-2, q_j-1, q_j
  float ring[S + 1][RP][3];
  float divr[RP][S + 1];  // divr[r][k] = divergence at plane (t - dl - k)
  float vzr[RP][3];       // vz at planes t-2, t-1, t (divergence in block)
#pragma unroll
  for (int j = 0; j <= S; ++j)
#pragma unroll
    for (int r = 0; r < RP; ++r) ring[j][r][0] = ring[j][r][1] = ring[j][r][2] = 0.0f;
#pragma unroll
  for (int r = 0; r < RP; ++r) {
#pragma unroll
    for (int k = 0; k <= S; ++k) divr[r][k] = 0.0f;
    vzr[r][0] = vzr[r][1] = vzr[r][2] = 0.0f;
  }
  __syncthreads();

  const int t_begin = za - L;
  const int t_end = zb - 1 + L + dl;

  // Raw inputs of plane tt for this thread's positions, loaded one clock ahead.
  float pre_v[RP], pre_a[RP], pre_b[RP], pre_c[RP];
  auto fetch = [&](int tt) {
    const bool t_in = tt >= 0 && tt < D;
    const bool zint = tt > 0 && tt < D - 1;
#pragma unroll
    for (int r = 0; r < RP; ++r) {
      pre_a[r] = pre_b[r] = pre_c[r] = pre_v[r] = 0.0f;
      if (!(t_in && indom[r])) continue;
      const size_t i = (size_t)gxy[r] + plane * (size_t)tt;
      if (DIVV) {
        pre_a[r] = __ldg(a.vfin.c[0] + i);
        pre_b[r] = __ldg(a.vfin.c[1] + i);
        pre_c[r] = __ldg(a.vfin.c[2] + i);
      } else if (S >= 1) {
        pre_a[r] = __ldg(a.div_in + i);
      }
      if (Fr::stage0) {
        if (IN == IN_BUF) {
          pre_v[r] = __ldg(a.p_in + i);
        } else if (zint && xyint[r]) {
          const float ps = prolong_sample(a.mid, a.mid_p, gxr[r], gyr[r], tt);
          pre_v[r] = (IN == IN_BUF_PROLONG) ? __ldg(a.p_in + i) + ps : 0.0f + ps;
        }
      }
    }
  };
  fetch(t_begin);

  for (int t = t_begin; t <= t_end; ++t) {
    const int b = t & 1;

    // ---- consume the prefetched plane t
    if (DIVV) {
#pragma unroll
      for (int r = 0; r < RP; ++r) {
        if (valid[r]) {
          vxs[b * P + pidx[r]] = pre_a[r];
          vys[b * P + pidx[r]] = pre_b[r];
        }
        vzr[r][0] = vzr[r][1];
        vzr[r][1] = vzr[r][2];
        vzr[r][2] = pre_c[r];
      }
    } else {
#pragma unroll
      for (int r = 0; r < RP; ++r) {
#pragma unroll
        for (int k = S; k > 0; --k) divr[r][k] = divr[r][k - 1];
        divr[r][0] = pre_a[r];
      }
    }
    if (Fr::stage0) {
#pragma unroll
      for (int r = 0; r < RP; ++r) {
        ring[0][r][0] = ring[0][r][1];
        ring[0][r][1] = ring[0][r][2];
        ring[0][r][2] = pre_v[r];
        if (valid[r] && Fr::pub_last >= 0) pub(0, b)[pidx[r]] = pre_v[r];
      }
    }
    // ---- issue the loads of plane t + 1; they complete while this clock computes
    if (t < t_end) fetch(t + 1);

    // ---- divergence at plane t - 1 (in block)
    if (DIVV) {
      const int q = t - 1;
      const int qb = q & 1;
      const bool qint = q > 0 && q < D - 1;
      const int slot = ((q % 3) + 3) % 3;
#pragma unroll
      for (int r = 0; r < RP; ++r) {
        float d = 0.0f;
        if (qint && xyint[r] && dist[r] >= 1) {
          const int c = pidx[r];
          const float* vx = vxs + qb * P;
          const float* vy = vys + qb * P;
          const float ddx = vx[c + 1] - vx[c - 1];
          const float ddy = vy[c + EX] - vy[c - EX];
          const float ddz = vzr[r][2] - vzr[r][0];
          d = (ddx + ddy + ddz) * 0.5f;
        }
#pragma unroll
        for (int k = S; k > 0; --k) divr[r][k] = divr[r][k - 1];
        divr[r][0] = d;
        if (valid[r]) dvs[slot * P + pidx[r]] = d;
        if (q >= za && q < zb && dist[r] >= H && indom[r]) a.div_out[(size_t)gxy[r] + plane * (size_t)q] = d;
      }
      // restriction of fine planes q-2, q-1 (published at clocks t-2, t-1)
      const int q1 = q - 1;
      if (a.restrict_mid && q1 >= za && q1 < zb && (q1 & 1) == 1 && tid < (TX / 2) * (TY / 2)) {
        const int mx_ = (gx0 + H) / 2 + (tid % (TX / 2)), my_ = (gy0 + H) / 2 + (tid / (TX / 2)), mz_ = q1 / 2;
        if (mx_ < (int)a.mid.w && my_ < (int)a.mid.h && mz_ < (int)a.mid.d) {
          float out = 0.0f;
          if (!(mx_ == 0 || my_ == 0 || mz_ == 0 || mx_ == (int)a.mid.w - 1 || my_ == (int)a.mid.h - 1 || mz_ == (int)a.mid.d - 1)) {
            const float* d0 = dvs + (((q1 - 1) % 3 + 3) % 3) * P;
            const float* d1 = dvs + ((q1 % 3 + 3) % 3) * P;
            const int c = (2 * mx_ - gx0) + (2 * my_ - gy0) * EX;
            float sum = 0.0f;
            sum += d0[c];
            sum += d0[c + 1];
            sum += d0[c + EX];
            sum += d0[c + EX + 1];
            sum += d1[c];
            sum += d1[c + 1];
            sum += d1[c + EX];
            sum += d1[c + EX + 1];
            out = sum * 0.125f;
          }
          a.mid_div[flat(a.mid, (uint32_t)mx_, (uint32_t)my_, (uint32_t)mz_)] = out;
        }
      }
    }

    // ---- sweeps: stage j at plane q_j = t - dl - j
#pragma unroll
    for (int j = 1; j <= S; ++j) {
      const int q = t - dl - j;
      const bool qint = q > 0 && q < D - 1;
      const float* xy = (j - 1 >= Fr::first) ? pub(j - 1, (q & 1)) : nullptr;
#pragma unroll
      for (int r = 0; r < RP; ++r) {
        float v = 0.0f;
        if (qint && xyint[r] && dist[r] >= j) {
          const float dd = divr[r][j];
          if (j == 1 && !Fr::stage0) {
            v = div6(0.0f - dd);
          } else {
            const int c = pidx[r];
            const float s = xy[c + 1] + xy[c - 1] + xy[c + EX] + xy[c - EX] + ring[j - 1][r][2] + ring[j - 1][r][0];
            v = div6(s - dd);
          }
        }
        ring[j][r][0] = ring[j][r][1];
        ring[j][r][1] = ring[j][r][2];
        ring[j][r][2] = v;
        if (j <= Fr::pub_last && valid[r]) pub(j, q & 1)[pidx[r]] = v;
      }
    }

    // ---- last stage to global, projection
    {
      const int q = t - dl - S;
      if (q >= za && q < zb) {
#pragma unroll
        for (int r = 0; r < RP; ++r)
          if (dist[r] >= H && indom[r]) a.p_out[(size_t)gxy[r] + plane * (size_t)q] = ring[S][r][2];
      }
    }
    if (PROJ) {
      const int q = t - dl - S - 1;
      if (q >= za && q < zb) {
        const bool qint = q > 0 && q < D - 1;
        const float* xy = pub(S, q & 1);
#pragma unroll
        for (int r = 0; r < RP; ++r) {
          if (dist[r] >= H && indom[r]) {
            const size_t i = (size_t)gxy[r] + plane * (size_t)q;
            float ox = 0.f, oy = 0.f, oz = 0.f;
            if (qint && xyint[r]) {
              const int c = pidx[r];
              const float gx = (xy[c + 1] - xy[c - 1]) * 0.5f;
              const float gy = (xy[c + EX] - xy[c - EX]) * 0.5f;
              const float gz = (ring[S][r][2] - ring[S][r][0]) * 0.5f;
              ox = __ldg(a.vfin.c[0] + i) - gx;
              oy = __ldg(a.vfin.c[1] + i) - gy;
              oz = __ldg(a.vfin.c[2] + i) - gz;
            }
            a.vcur.c[0][i] = ox;
            a.vcur.c[1][i] = oy;
            a.vcur.c[2][i] = oz;
            if (a.write_vmag) a.vmag[i] = length3(ox, oy, oz);
          }
        }
      }
    }
    __syncthreads();
  }
}

template <int S, int IN, bool DIVV, bool PROJ>
cudaError_t launch_z(cudaStream_t s, const ZArgs& a) {
  using Fr = Frame<S, IN, DIVV, PROJ>;
  const size_t smem = (size_t)Fr::floats * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(k_zjacobi<S, IN, DIVV, PROJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const dim3 grid((a.dm.w + TX - 1) / TX, (a.dm.h + TY - 1) / TY, (a.dm.d + a.zchunk - 1) / a.zchunk);
  k_zjacobi<S, IN, DIVV, PROJ><<<grid, dim3(TX, TY), smem, s>>>(a);
  return cudaGetLastError();
}

template <int IN, bool DIVV, bool PROJ>
cudaError_t launch_s(cudaStream_t s, int sweeps, const ZArgs& a) {
  switch (sweeps) {
    case 0: return launch_z<0, IN, DIVV, PROJ>(s, a);
    case 1: return launch_z<1, IN, DIVV, PROJ>(s, a);
    case 2: return launch_z<2, IN, DIVV, PROJ>(s, a);
    case 3: return launch_z<3, IN, DIVV, PROJ>(s, a);
    default: return launch_z<4, IN, DIVV, PROJ>(s, a);
  }
}

// ---------------------------------------------------------------------------
// Lean per-voxel kernels (one thread per voxel, blocks of 32 x 4 x 2).
// ---------------------------------------------------------------------------

// Divergence (compute-divergence.wgsl.ts:22-42) with, pointwise, the first
// Jacobi sweep from the cleared buffer, (0 - div) / 6, and the fine->mid
// restriction (pressure-restriction.wgsl.ts:27-50) of each 2x2x2 group of the
// block through shared memory. The restriction needs every fine dimension >= 16.
__global__ void __launch_bounds__(256) k_div_first(Dims dm, VelField v, float* __restrict__ div, float* __restrict__ p1, Dims mid,
                                                   float* __restrict__ mid_div, int restrict_mid) {
  __shared__ float sd[2][4][32];
  const uint32_t x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 4 + threadIdx.y, z = blockIdx.z * 2 + threadIdx.z;
  const bool in = x < dm.w && y < dm.h && z < dm.d;
  float d = 0.0f;
  if (in) {
    const uint32_t i = flat(dm, x, y, z);
    if (!is_boundary(dm, x, y, z)) {
      const uint32_t sy = dm.w, sz = dm.w * dm.h;
      const float ddx = __ldg(v.c[0] + i + 1) - __ldg(v.c[0] + i - 1);
      const float ddy = __ldg(v.c[1] + i + sy) - __ldg(v.c[1] + i - sy);
      const float ddz = __ldg(v.c[2] + i + sz) - __ldg(v.c[2] + i - sz);
      d = (ddx + ddy + ddz) * 0.5f;
      if (p1) p1[i] = div6(0.0f - d);
    } else if (p1) {
      p1[i] = 0.0f;
    }
    div[i] = d;
  }
  if (!restrict_mid) return;
  sd[threadIdx.z][threadIdx.y][threadIdx.x] = d;
  __syncthreads();
  if (threadIdx.z == 0 && (threadIdx.y & 1) == 0 && (threadIdx.x & 1) == 0) {
    const uint32_t mx_ = x >> 1, my_ = y >> 1, mz_ = z >> 1;
    if (mx_ < mid.w && my_ < mid.h && mz_ < mid.d) {
      float out = 0.0f;
      if (!(mx_ == 0 || my_ == 0 || mz_ == 0 || mx_ == mid.w - 1 || my_ == mid.h - 1 || mz_ == mid.d - 1)) {
        const int tx = threadIdx.x, ty = threadIdx.y;
        float sum = 0.0f;
        sum += sd[0][ty][tx];
        sum += sd[0][ty][tx + 1];
        sum += sd[0][ty + 1][tx];
        sum += sd[0][ty + 1][tx + 1];
        sum += sd[1][ty][tx];
        sum += sd[1][ty][tx + 1];
        sum += sd[1][ty + 1][tx];
        sum += sd[1][ty + 1][tx + 1];
        out = sum * 0.125f;
      }
      mid_div[flat(mid, mx_, my_, mz_)] = out;
    }
  }
}

// k_div_first with four x per thread marching runs of planes (widths divisible
// by 4, even heights and depths; runs of even length starting on even planes).
// Per plane a thread loads one float4 of vx (the x neighbours by warp shuffle,
// the row ends load theirs), two of vy (rows y - 1 and y + 1) and one of vz
// (plane z + 1; planes z - 1 and z are held from the earlier planes), issuing
// the next plane's loads before it computes the current one. The restriction
// adds each 2x2x2 group in k_div_first's order: the even row's warp sums plane
// 2m (its row, then the odd row's from shared memory) and carries the partial
// sum to plane 2m + 1. Every value is computed with the same operations in the
// same order, so the results are the same bits.
__global__ void __launch_bounds__(256, 4) k_div_march(Dims dm, VelField v, float* __restrict__ div, float* __restrict__ p1, Dims mid,
                                                      float* __restrict__ mid_div, int restrict_mid, int run) {
  __shared__ float4 srow[2][8][32];  // this plane's divergence rows of the block, double-buffered by plane parity
  const uint32_t lane = threadIdx.x, ty = threadIdx.y;
  const uint32_t x0 = blockIdx.x * 128 + 4 * lane, y = blockIdx.y * 8 + ty;
  const int zb = (int)blockIdx.z * run, ze = min(zb + run, (int)dm.d);
  if (zb >= ze) return;  // whole block
  const int D = (int)dm.d;
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const bool yin = y < dm.h;
  const bool xin = x0 < dm.w;  // dm.w % 4 == 0: x0 + 3 < dm.w too
  const uint32_t base = (xin ? x0 : dm.w - 4) + dm.w * (yin ? y : dm.h - 1);
  const bool yint = yin && y > 0 && y < dm.h - 1;
  const bool int0 = x0 > 0, int3 = x0 + 3 < dm.w - 1;  // x0 + 1 and x0 + 2 are interior in x
  const bool left_end = lane == 0 && x0 > 0, right_end = lane == 31 && x0 + 4 < dm.w;
  const float4* __restrict__ vx4 = reinterpret_cast<const float4*>(v.c[0]);
  const float4* __restrict__ vy4 = reinterpret_cast<const float4*>(v.c[1]);
  const float4* __restrict__ vz4 = reinterpret_cast<const float4*>(v.c[2]);
  const float* __restrict__ vx = v.c[0];
  float4* __restrict__ div4 = reinterpret_cast<float4*>(div);
  float4* __restrict__ p14 = reinterpret_cast<float4*>(p1);
  const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  // vz row at a plane (zero outside the grid and on boundary rows, which never use it)
  auto vzrow = [&](int z) { return (yint && z >= 0 && z < D) ? __ldg(vz4 + ((base + sz * (uint32_t)z) >> 2)) : zero4; };
  float4 vzm = vzrow(zb - 1), vzc = vzrow(zb), vzp = vzrow(zb + 1);
  float4 X = zero4, YP = zero4, YM = zero4;
  float XL = 0.0f, XR = 0.0f;
  {
    const uint32_t i = base + sz * (uint32_t)zb;
    if (yint) {
      X = __ldg(vx4 + (i >> 2));
      YP = __ldg(vy4 + ((i + sy) >> 2));
      YM = __ldg(vy4 + ((i - sy) >> 2));
      if (left_end) XL = __ldg(vx + i - 1);
      if (right_end) XR = __ldg(vx + i + 4);
    }
  }
  float part0 = 0.0f, part1 = 0.0f;  // restriction sums of mid x = x0/2 and x0/2 + 1 (even rows)
  for (int z = zb; z < ze; ++z) {
    // next plane's loads (clamped in range on the last plane, values then unused)
    const int zn = min(z + 1, D - 1);
    const uint32_t in = base + sz * (uint32_t)zn;
    float4 nX = zero4, nYP = zero4, nYM = zero4;
    float nXL = 0.0f, nXR = 0.0f;
    if (yint) {
      nX = __ldg(vx4 + (in >> 2));
      nYP = __ldg(vy4 + ((in + sy) >> 2));
      nYM = __ldg(vy4 + ((in - sy) >> 2));
      if (left_end) nXL = __ldg(vx + in - 1);
      if (right_end) nXR = __ldg(vx + in + 4);
    }
    const float4 nvz = vzrow(z + 2);
    float left = __shfl_up_sync(0xffffffffu, X.w, 1);     // vx at x0 - 1
    float right = __shfl_down_sync(0xffffffffu, X.x, 1);  // vx at x0 + 4
    if (left_end) left = XL;
    if (right_end) right = XR;
    float4 d = zero4;
    const bool plane_int = yint && z > 0 && z < D - 1;
    if (plane_int) {
      if (int0) d.x = ((X.y - left) + (YP.x - YM.x) + (vzp.x - vzm.x)) * 0.5f;
      d.y = ((X.z - X.x) + (YP.y - YM.y) + (vzp.y - vzm.y)) * 0.5f;
      d.z = ((X.w - X.y) + (YP.z - YM.z) + (vzp.z - vzm.z)) * 0.5f;
      if (int3) d.w = ((right - X.z) + (YP.w - YM.w) + (vzp.w - vzm.w)) * 0.5f;
    }
    const uint32_t i = base + sz * (uint32_t)z;
    if (yin && xin) {
      div4[i >> 2] = d;
      if (p1) {
        float4 q = zero4;
        if (plane_int) {
          if (int0) q.x = div6(0.0f - d.x);
          q.y = div6(0.0f - d.y);
          q.z = div6(0.0f - d.z);
          if (int3) q.w = div6(0.0f - d.w);
        }
        p14[i >> 2] = q;
      }
    }
    if (restrict_mid) {
      const int b = z & 1;
      srow[b][ty][lane] = d;
      __syncthreads();
      if ((ty & 1) == 0) {
        const float4 o = srow[b][ty + 1][lane];  // row y + 1 (zero beyond the grid)
        if (b == 0) {
          part0 = 0.0f;
          part1 = 0.0f;
        }
        part0 += d.x;
        part0 += d.y;
        part0 += o.x;
        part0 += o.y;
        part1 += d.z;
        part1 += d.w;
        part1 += o.z;
        part1 += o.w;
        if (b == 1 && xin && yin) {
          const uint32_t my_ = y >> 1, mz_ = (uint32_t)z >> 1;
          for (int h = 0; h < 2; ++h) {
            const uint32_t mx_ = (x0 >> 1) + (uint32_t)h;
            if (mx_ < mid.w && my_ < mid.h && mz_ < mid.d) {
              const bool mb = mx_ == 0 || my_ == 0 || mz_ == 0 || mx_ == mid.w - 1 || my_ == mid.h - 1 || mz_ == mid.d - 1;
              mid_div[flat(mid, mx_, my_, mz_)] = mb ? 0.0f : (h ? part1 : part0) * 0.125f;
            }
          }
        }
      }
    }
    vzm = vzc;
    vzc = vzp;
    vzp = nvz;
    X = nX;
    YP = nYP;
    YM = nYM;
    XL = nXL;
    XR = nXR;
  }
}

// One Jacobi sweep (pressure-jacobi.wgsl.ts:15-36). With `mid_p`, the result
// then gets the prolongation added (pressure-prolongation.wgsl.ts:36-43: the
// boundary stays 0, the interior becomes p + sample), as when the reference
// prolongs into the buffer this sweep wrote. With `src` NULL the input is the
// cleared buffer.
//
// A thread computes a column of ZB voxels along z, reusing the z neighbours in
// registers; all loads of the column are independent, which keeps enough bytes
// in flight per SM to stream HBM.
// A warp holds 32 consecutive x of one row. The x neighbours come from the
// coalesced centre row by shuffles (the two row ends load their outer
// neighbour), the z neighbours from the column in registers; every load of the
// column is issued before the arithmetic. The sum keeps the reference order
// +x, -x, +y, -y, +z, -z.
template <int ZB>
__global__ void __launch_bounds__(256) k_sweep(Dims dm, const float* __restrict__ div, const float* __restrict__ src, float* __restrict__ dst,
                                               Dims mid, const float* __restrict__ mid_p) {
  const uint32_t lane = threadIdx.x;
  const uint32_t x = blockIdx.x * 32 + lane, y = blockIdx.y * 8 + threadIdx.y, z0 = blockIdx.z * ZB;
  if (y >= dm.h) return;  // whole warp
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const bool xin = x < dm.w;
  const uint32_t base = (xin ? x : dm.w - 1) + dm.w * y;
  const bool yint = y > 0 && y < dm.h - 1;
  const bool xint = x > 0 && x < dm.w - 1;
  const int nz = min(ZB, (int)dm.d - (int)z0);
  if (!yint) {
    if (xin)
      for (int k = 0; k < nz; ++k) dst[base + sz * (z0 + k)] = 0.0f;
    return;
  }
  float c[ZB + 2], yp[ZB], ym[ZB], dv[ZB], xe[ZB];
  const bool left_end = lane == 0 && x > 0, right_end = (lane == 31 || x == dm.w - 1) && x + 1 < dm.w;
#pragma unroll
  for (int k = 0; k < ZB + 2; ++k) {
    const int z = (int)z0 + k - 1;
    c[k] = (src && z >= 0 && z < (int)dm.d) ? __ldg(src + base + sz * (uint32_t)z) : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < ZB; ++k) {
    const uint32_t z = min(z0 + k, dm.d - 1);
    const uint32_t i = base + sz * z;
    dv[k] = __ldg(div + i);
    yp[k] = src ? __ldg(src + i + sy) : 0.0f;
    ym[k] = src ? __ldg(src + i - sy) : 0.0f;
    xe[k] = 0.0f;
    if (src && left_end) xe[k] = __ldg(src + i - 1);
    if (src && right_end) xe[k] = __ldg(src + i + 1);
  }
#pragma unroll
  for (int k = 0; k < ZB; ++k) {
    const float cm = c[k + 1];
    float xr = __shfl_down_sync(0xffffffffu, cm, 1);
    float xl = __shfl_up_sync(0xffffffffu, cm, 1);
    if (right_end) xr = xe[k];
    if (left_end) xl = xe[k];
    const uint32_t z = z0 + k;
    if (k >= nz || !xin) continue;
    float v = 0.0f;
    if (xint && z > 0 && z < dm.d - 1) {
      if (src) {
        const float s = xr + xl + yp[k] + ym[k] + c[k + 2] + c[k];
        v = div6(s - dv[k]);
      } else {
        v = div6(0.0f - dv[k]);
      }
      if (mid_p) v = v + prolong_sample(mid, mid_p, (int)x, (int)y, (int)z);
    }
    dst[base + sz * z] = v;
  }
}

// k_sweep with two consecutive x per thread (even widths): a warp covers 64 x,
// the column loads are float2, and one shuffle per voxel brings the outer x
// neighbour of each pair from the next lane. Each voxel's sum, division and
// prolongation are those of k_sweep, in the same order, so the results are the
// same bits.
template <int ZB>
__global__ void __launch_bounds__(256) k_sweep_v2(Dims dm, const float* __restrict__ div, const float* __restrict__ src, float* __restrict__ dst,
                                                  Dims mid, const float* __restrict__ mid_p) {
  const uint32_t lane = threadIdx.x;
  const uint32_t x0 = blockIdx.x * 64 + 2 * lane, y = blockIdx.y * 8 + threadIdx.y, z0 = blockIdx.z * ZB;
  if (y >= dm.h) return;  // whole warp
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const bool xin = x0 < dm.w;  // dm.w is even: x0 + 1 < dm.w too
  const uint32_t base = (xin ? x0 : dm.w - 2) + dm.w * y;
  const bool yint = y > 0 && y < dm.h - 1;
  const int nz = min(ZB, (int)dm.d - (int)z0);
  const float2* __restrict__ src2 = reinterpret_cast<const float2*>(src);
  const float2* __restrict__ div2 = reinterpret_cast<const float2*>(div);
  float2* __restrict__ dst2 = reinterpret_cast<float2*>(dst);
  if (!yint) {
    if (xin)
      for (int k = 0; k < nz; ++k) dst2[(base + sz * (z0 + k)) >> 1] = make_float2(0.0f, 0.0f);
    return;
  }
  const bool int0 = x0 > 0 && x0 < dm.w - 1, int1 = x0 + 1 < dm.w - 1;
  const bool left_end = lane == 0 && x0 > 0, right_end = lane == 31 && x0 + 2 < dm.w;
  float2 c[ZB + 2], yp[ZB], ym[ZB], dv[ZB];
  float xl_e[ZB], xr_e[ZB];
#pragma unroll
  for (int k = 0; k < ZB + 2; ++k) {
    const int z = (int)z0 + k - 1;
    c[k] = (src && z >= 0 && z < (int)dm.d) ? __ldg(src2 + ((base + sz * (uint32_t)z) >> 1)) : make_float2(0.0f, 0.0f);
  }
#pragma unroll
  for (int k = 0; k < ZB; ++k) {
    const uint32_t z = min(z0 + k, dm.d - 1);
    const uint32_t i = base + sz * z;
    dv[k] = __ldg(div2 + (i >> 1));
    yp[k] = src ? __ldg(src2 + ((i + sy) >> 1)) : make_float2(0.0f, 0.0f);
    ym[k] = src ? __ldg(src2 + ((i - sy) >> 1)) : make_float2(0.0f, 0.0f);
    xl_e[k] = (src && left_end) ? __ldg(src + i - 1) : 0.0f;
    xr_e[k] = (src && right_end) ? __ldg(src + i + 2) : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < ZB; ++k) {
    const float2 cm = c[k + 1];
    float left = __shfl_up_sync(0xffffffffu, cm.y, 1);     // x0 - 1
    float right = __shfl_down_sync(0xffffffffu, cm.x, 1);  // x0 + 2
    if (left_end) left = xl_e[k];
    if (right_end) right = xr_e[k];
    const uint32_t z = z0 + k;
    if (k >= nz || !xin) continue;
    const bool zint = z > 0 && z < dm.d - 1;
    float v0 = 0.0f, v1 = 0.0f;
    if (zint && int0) {
      v0 = src ? div6(cm.y + left + yp[k].x + ym[k].x + c[k + 2].x + c[k].x - dv[k].x) : div6(0.0f - dv[k].x);
      if (mid_p) v0 = v0 + prolong_sample(mid, mid_p, (int)x0, (int)y, (int)z);
    }
    if (zint && int1) {
      v1 = src ? div6(right + cm.x + yp[k].y + ym[k].y + c[k + 2].y + c[k].y - dv[k].y) : div6(0.0f - dv[k].y);
      if (mid_p) v1 = v1 + prolong_sample(mid, mid_p, (int)x0 + 1, (int)y, (int)z);
    }
    dst2[(base + sz * z) >> 1] = make_float2(v0, v1);
  }
}

// k_sweep with four consecutive x per thread (widths divisible by 4): a warp
// covers 128 x, the column loads are float4, and one shuffle each way per voxel
// row brings the outer x neighbours from the adjacent lanes. Each voxel's sum,
// division and prolongation are those of k_sweep, in the same order, so the
// results are the same bits.
template <int ZB>
__global__ void __launch_bounds__(256) k_sweep_v4(Dims dm, const float* __restrict__ div, const float* __restrict__ src, float* __restrict__ dst,
                                                  Dims mid, const float* __restrict__ mid_p) {
  const uint32_t lane = threadIdx.x;
  const uint32_t x0 = blockIdx.x * 128 + 4 * lane, y = blockIdx.y * 8 + threadIdx.y, z0 = blockIdx.z * ZB;
  if (y >= dm.h) return;  // whole warp
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const bool xin = x0 < dm.w;  // dm.w % 4 == 0: x0 + 3 < dm.w too
  const uint32_t base = (xin ? x0 : dm.w - 4) + dm.w * y;
  const bool yint = y > 0 && y < dm.h - 1;
  const int nz = min(ZB, (int)dm.d - (int)z0);
  const float4* __restrict__ src4 = reinterpret_cast<const float4*>(src);
  const float4* __restrict__ div4 = reinterpret_cast<const float4*>(div);
  float4* __restrict__ dst4 = reinterpret_cast<float4*>(dst);
  if (!yint) {
    if (xin)
      for (int k = 0; k < nz; ++k) dst4[(base + sz * (z0 + k)) >> 2] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    return;
  }
  const bool int0 = x0 > 0, int3 = x0 + 3 < dm.w - 1;  // x0 + 1 and x0 + 2 are always interior
  const bool left_end = lane == 0 && x0 > 0, right_end = lane == 31 && x0 + 4 < dm.w;
  float4 c[ZB + 2], yp[ZB], ym[ZB], dv[ZB];
  float xl_e[ZB], xr_e[ZB];
  const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
  for (int k = 0; k < ZB + 2; ++k) {
    const int z = (int)z0 + k - 1;
    c[k] = (src && z >= 0 && z < (int)dm.d) ? __ldg(src4 + ((base + sz * (uint32_t)z) >> 2)) : zero4;
  }
#pragma unroll
  for (int k = 0; k < ZB; ++k) {
    const uint32_t z = min(z0 + k, dm.d - 1);
    const uint32_t i = base + sz * z;
    dv[k] = __ldg(div4 + (i >> 2));
    yp[k] = src ? __ldg(src4 + ((i + sy) >> 2)) : zero4;
    ym[k] = src ? __ldg(src4 + ((i - sy) >> 2)) : zero4;
    xl_e[k] = (src && left_end) ? __ldg(src + i - 1) : 0.0f;
    xr_e[k] = (src && right_end) ? __ldg(src + i + 4) : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < ZB; ++k) {
    const float4 cm = c[k + 1];
    float left = __shfl_up_sync(0xffffffffu, cm.w, 1);     // x0 - 1
    float right = __shfl_down_sync(0xffffffffu, cm.x, 1);  // x0 + 4
    if (left_end) left = xl_e[k];
    if (right_end) right = xr_e[k];
    const uint32_t z = z0 + k;
    if (k >= nz || !xin) continue;
    float4 v = zero4;
    if (z > 0 && z < dm.d - 1) {
      if (src) {
        if (int0) v.x = div6(cm.y + left + yp[k].x + ym[k].x + c[k + 2].x + c[k].x - dv[k].x);
        v.y = div6(cm.z + cm.x + yp[k].y + ym[k].y + c[k + 2].y + c[k].y - dv[k].y);
        v.z = div6(cm.w + cm.y + yp[k].z + ym[k].z + c[k + 2].z + c[k].z - dv[k].z);
        if (int3) v.w = div6(right + cm.z + yp[k].w + ym[k].w + c[k + 2].w + c[k].w - dv[k].w);
      } else {
        if (int0) v.x = div6(0.0f - dv[k].x);
        v.y = div6(0.0f - dv[k].y);
        v.z = div6(0.0f - dv[k].z);
        if (int3) v.w = div6(0.0f - dv[k].w);
      }
      if (mid_p) {
        if (int0) v.x = v.x + prolong_sample(mid, mid_p, (int)x0, (int)y, (int)z);
        v.y = v.y + prolong_sample(mid, mid_p, (int)x0 + 1, (int)y, (int)z);
        v.z = v.z + prolong_sample(mid, mid_p, (int)x0 + 2, (int)y, (int)z);
        if (int3) v.w = v.w + prolong_sample(mid, mid_p, (int)x0 + 3, (int)y, (int)z);
      }
    }
    dst4[(base + sz * z) >> 2] = v;
  }
}

// k_sweep_v4 marching in z: a thread owns four x of one row and walks a run of
// `run` planes, holding the rows at z - 1, z and z + 1 in registers and issuing
// the loads of plane z + 1 before it computes plane z, so a warp always has one
// plane of loads in flight. The host sizes the runs so the grid is one wave of
// resident blocks. Each voxel's sum and division are those of k_sweep, in the
// same order, so the results are the same bits. The sweep with the fused
// prolongation has its own marching kernel, k_sweep_march_prolong, which also
// shares the prolongation's mid-level corners between voxels.
__global__ void __launch_bounds__(256, 4) k_sweep_march(Dims dm, const float* __restrict__ div, const float* __restrict__ src,
                                                        float* __restrict__ dst, int run) {
  const uint32_t lane = threadIdx.x;
  const uint32_t x0 = blockIdx.x * 128 + 4 * lane, y = blockIdx.y * 8 + threadIdx.y;
  const int zb = (int)blockIdx.z * run, ze = min(zb + run, (int)dm.d);
  if (y >= dm.h || zb >= ze) return;  // whole warp
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const bool xin = x0 < dm.w;  // dm.w % 4 == 0: x0 + 3 < dm.w too
  const uint32_t base = (xin ? x0 : dm.w - 4) + dm.w * y;
  const bool yint = y > 0 && y < dm.h - 1;
  const float4* __restrict__ src4 = reinterpret_cast<const float4*>(src);
  const float4* __restrict__ div4 = reinterpret_cast<const float4*>(div);
  float4* __restrict__ dst4 = reinterpret_cast<float4*>(dst);
  const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (!yint) {
    if (xin)
      for (int z = zb; z < ze; ++z) dst4[(base + sz * (uint32_t)z) >> 2] = zero4;
    return;
  }
  const bool int0 = x0 > 0, int3 = x0 + 3 < dm.w - 1;  // x0 + 1 and x0 + 2 are always interior
  const bool left_end = lane == 0 && x0 > 0, right_end = lane == 31 && x0 + 4 < dm.w;
  const int D = (int)dm.d;
  // Rows of the source at a plane, zero outside the grid (only the interior
  // planes 1..D-2 read them, and those reach 0..D-1).
  auto crow = [&](int z) { return (src && z >= 0 && z < D) ? __ldg(src4 + ((base + sz * (uint32_t)z) >> 2)) : zero4; };
  float4 cm = crow(zb - 1), c0 = crow(zb), cp = crow(zb + 1);
  // Plane zb's own rows; every later plane's are loaded one iteration ahead.
  const uint32_t i = base + sz * (uint32_t)zb;
  float4 dv = __ldg(div4 + (i >> 2));
  float4 yp = src ? __ldg(src4 + ((i + sy) >> 2)) : zero4;
  float4 ym = src ? __ldg(src4 + ((i - sy) >> 2)) : zero4;
  float xle = (src && left_end) ? __ldg(src + i - 1) : 0.0f;
  float xre = (src && right_end) ? __ldg(src + i + 4) : 0.0f;
  for (int z = zb; z < ze; ++z) {
    // Loads for plane z + 1 (its z + 1 row is plane z + 2), clamped in range on
    // the last plane, whose values are then never used.
    const int zn = min(z + 1, D - 1);
    const uint32_t in = base + sz * (uint32_t)zn;
    const float4 n_c = crow(z + 2);
    const float4 n_dv = __ldg(div4 + (in >> 2));
    const float4 n_yp = src ? __ldg(src4 + ((in + sy) >> 2)) : zero4;
    const float4 n_ym = src ? __ldg(src4 + ((in - sy) >> 2)) : zero4;
    const float n_xle = (src && left_end) ? __ldg(src + in - 1) : 0.0f;
    const float n_xre = (src && right_end) ? __ldg(src + in + 4) : 0.0f;
    float left = __shfl_up_sync(0xffffffffu, c0.w, 1);     // x0 - 1
    float right = __shfl_down_sync(0xffffffffu, c0.x, 1);  // x0 + 4
    if (left_end) left = xle;
    if (right_end) right = xre;
    if (xin) {
      float4 v = zero4;
      if (z > 0 && z < D - 1) {
        if (src) {
          if (int0) v.x = div6(c0.y + left + yp.x + ym.x + cp.x + cm.x - dv.x);
          v.y = div6(c0.z + c0.x + yp.y + ym.y + cp.y + cm.y - dv.y);
          v.z = div6(c0.w + c0.y + yp.z + ym.z + cp.z + cm.z - dv.z);
          if (int3) v.w = div6(right + c0.z + yp.w + ym.w + cp.w + cm.w - dv.w);
        } else {
          if (int0) v.x = div6(0.0f - dv.x);
          v.y = div6(0.0f - dv.y);
          v.z = div6(0.0f - dv.z);
          if (int3) v.w = div6(0.0f - dv.w);
        }
      }
      dst4[(base + sz * (uint32_t)z) >> 2] = v;
    }
    cm = c0;
    c0 = cp;
    cp = n_c;
    dv = n_dv;
    yp = n_yp;
    ym = n_ym;
    xle = n_xle;
    xre = n_xre;
  }
}

// k_sweep_march with the prolongation of mid_p added (the first fine post-sweep),
// for even fine grids with widths divisible by 4 whose mid level is exactly half
// their size. There, at an interior fine voxel, prolong_sample's position
// ((c + 0.5) * 0.5 - 0.5 per axis) needs no clamp, its corners are mid cells
// (c - 1) >> 1 and one more, and its weights are exactly 0.75 for even c and
// 0.25 for odd c. A thread's four x then read mid columns x0/2 - 1 .. x0/2 + 2 of
// two mid rows, and consecutive fine planes share mid planes: the kernel holds
// the two mid planes of the current fine plane (8 values each: a float2 load
// per row, the outer columns by warp shuffle) and loads the next one, from L2,
// when fine z reaches it. Each sample is tri_interp's mix of the same corner values with the
// same weights in the same order, so the results are the same bits.
__global__ void __launch_bounds__(256, 3) k_sweep_march_prolong(Dims dm, const float* __restrict__ div, const float* __restrict__ src,
                                                                float* __restrict__ dst, Dims mid, const float* __restrict__ mid_p, int run) {
  const uint32_t lane = threadIdx.x;
  const uint32_t x0 = blockIdx.x * 128 + 4 * lane, y = blockIdx.y * 8 + threadIdx.y;
  const int zb = (int)blockIdx.z * run, ze = min(zb + run, (int)dm.d);
  if (y >= dm.h || zb >= ze) return;  // whole warp
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const bool xin = x0 < dm.w;  // dm.w % 4 == 0: x0 + 3 < dm.w too
  const uint32_t xb = xin ? x0 : dm.w - 4;
  const uint32_t base = xb + dm.w * y;
  const bool yint = y > 0 && y < dm.h - 1;
  const float4* __restrict__ src4 = reinterpret_cast<const float4*>(src);
  const float4* __restrict__ div4 = reinterpret_cast<const float4*>(div);
  float4* __restrict__ dst4 = reinterpret_cast<float4*>(dst);
  const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (!yint) {
    if (xin)
      for (int z = zb; z < ze; ++z) dst4[(base + sz * (uint32_t)z) >> 2] = zero4;
    return;
  }
  const bool int0 = x0 > 0, int3 = x0 + 3 < dm.w - 1;  // x0 + 1 and x0 + 2 are always interior
  const bool left_end = lane == 0 && x0 > 0, right_end = lane == 31 && x0 + 4 < dm.w;
  const int D = (int)dm.d;
  // mid rows and row weight of this fine row (interior, so unclamped)
  const uint32_t mc = xb >> 1;  // even; the thread's mid columns are mc - 1 .. mc + 2
  const uint32_t mby = (y - 1u) >> 1, muy = mby + 1u;
  const float fy = (y & 1u) ? 0.25f : 0.75f;
  const float2* __restrict__ mid2 = reinterpret_cast<const float2*>(mid_p);
  // Raw loads of one mid plane: the float2 (mc, mc + 1) of each row, and at the
  // row ends of the warp the outer column the shuffle cannot bring.
  struct Raw {
    float2 r0, r1;
    float l0, l1, q0, q1;
  };
  auto mid_raw = [&](int pz) {
    Raw o;
    const uint32_t pc = (uint32_t)max(0, min(pz, (int)mid.d - 1));
    const uint32_t i0 = mc + mid.w * (mby + mid.h * pc), i1 = mc + mid.w * (muy + mid.h * pc);
    o.r0 = __ldg(mid2 + (i0 >> 1));
    o.r1 = __ldg(mid2 + (i1 >> 1));
    o.l0 = left_end ? __ldg(mid_p + i0 - 1) : 0.0f;
    o.l1 = left_end ? __ldg(mid_p + i1 - 1) : 0.0f;
    o.q0 = right_end ? __ldg(mid_p + i0 + 2) : 0.0f;
    o.q1 = right_end ? __ldg(mid_p + i1 + 2) : 0.0f;
    return o;
  };
  // The 8 values of a mid plane: [row][column mc - 1 + k]
  struct Plane {
    float v[2][4];
  };
  auto expand = [&](const Raw& r) {
    Plane p;
    float a = __shfl_up_sync(0xffffffffu, r.r0.y, 1), b = __shfl_down_sync(0xffffffffu, r.r0.x, 1);
    float c = __shfl_up_sync(0xffffffffu, r.r1.y, 1), d = __shfl_down_sync(0xffffffffu, r.r1.x, 1);
    if (left_end) {
      a = r.l0;
      c = r.l1;
    }
    if (right_end) {
      b = r.q0;
      d = r.q1;
    }
    p.v[0][0] = a;
    p.v[0][1] = r.r0.x;
    p.v[0][2] = r.r0.y;
    p.v[0][3] = b;
    p.v[1][0] = c;
    p.v[1][1] = r.r1.x;
    p.v[1][2] = r.r1.y;
    p.v[1][3] = d;
    return p;
  };
  // tri_interp over mid columns (k, k + 1) of planes A (z corner b) and B (u)
  auto sample = [&](const Plane& A, const Plane& B, int k, float fx, float fz) {
    const float x00 = mixv(A.v[0][k], A.v[0][k + 1], fx);
    const float x10 = mixv(A.v[1][k], A.v[1][k + 1], fx);
    const float x01 = mixv(B.v[0][k], B.v[0][k + 1], fx);
    const float x11 = mixv(B.v[1][k], B.v[1][k + 1], fx);
    return mixv(mixv(x00, x10, fy), mixv(x01, x11, fy), fz);
  };
  int cbz = (zb - 1) >> 1;  // the mid plane held in A (B holds cbz + 1)
  Plane A = expand(mid_raw(cbz)), B = expand(mid_raw(cbz + 1));

  auto crow = [&](int z) { return (src && z >= 0 && z < D) ? __ldg(src4 + ((base + sz * (uint32_t)z) >> 2)) : zero4; };
  float4 cm = crow(zb - 1), c0 = crow(zb), cp = crow(zb + 1);
  const uint32_t i = base + sz * (uint32_t)zb;
  float4 dv = __ldg(div4 + (i >> 2));
  float4 yp = src ? __ldg(src4 + ((i + sy) >> 2)) : zero4;
  float4 ym = src ? __ldg(src4 + ((i - sy) >> 2)) : zero4;
  float xle = (src && left_end) ? __ldg(src + i - 1) : 0.0f;
  float xre = (src && right_end) ? __ldg(src + i + 4) : 0.0f;
  for (int z = zb; z < ze; ++z) {
    const int bz = (z - 1) >> 1;
    if (bz != cbz) {  // warp-uniform: fine z moved on to the next mid plane pair (an L2 hit)
      A = B;
      cbz = bz;
      B = expand(mid_raw(cbz + 1));
    }
    const int zn = min(z + 1, D - 1);
    const uint32_t in = base + sz * (uint32_t)zn;
    const float4 n_c = crow(z + 2);
    const float4 n_dv = __ldg(div4 + (in >> 2));
    const float4 n_yp = src ? __ldg(src4 + ((in + sy) >> 2)) : zero4;
    const float4 n_ym = src ? __ldg(src4 + ((in - sy) >> 2)) : zero4;
    const float n_xle = (src && left_end) ? __ldg(src + in - 1) : 0.0f;
    const float n_xre = (src && right_end) ? __ldg(src + in + 4) : 0.0f;
    float left = __shfl_up_sync(0xffffffffu, c0.w, 1);     // x0 - 1
    float right = __shfl_down_sync(0xffffffffu, c0.x, 1);  // x0 + 4
    if (left_end) left = xle;
    if (right_end) right = xre;
    if (xin) {
      float4 v = zero4;
      if (z > 0 && z < D - 1) {
        if (src) {
          if (int0) v.x = div6(c0.y + left + yp.x + ym.x + cp.x + cm.x - dv.x);
          v.y = div6(c0.z + c0.x + yp.y + ym.y + cp.y + cm.y - dv.y);
          v.z = div6(c0.w + c0.y + yp.z + ym.z + cp.z + cm.z - dv.z);
          if (int3) v.w = div6(right + c0.z + yp.w + ym.w + cp.w + cm.w - dv.w);
        } else {
          if (int0) v.x = div6(0.0f - dv.x);
          v.y = div6(0.0f - dv.y);
          v.z = div6(0.0f - dv.z);
          if (int3) v.w = div6(0.0f - dv.w);
        }
        const float fz = (z & 1) ? 0.25f : 0.75f;
        if (int0) v.x = v.x + sample(A, B, 0, 0.75f, fz);
        v.y = v.y + sample(A, B, 1, 0.25f, fz);
        v.z = v.z + sample(A, B, 1, 0.75f, fz);
        if (int3) v.w = v.w + sample(A, B, 2, 0.25f, fz);
      }
      dst4[(base + sz * (uint32_t)z) >> 2] = v;
    }
    cm = c0;
    c0 = cp;
    cp = n_c;
    dv = n_dv;
    yp = n_yp;
    ym = n_ym;
    xle = n_xle;
    xre = n_xre;
  }
}

// The cleared buffer plus the prolongation (finePre = 0): boundary 0, interior 0 + sample.
__global__ void __launch_bounds__(256) k_prolong_zero(Dims dm, float* __restrict__ dst, Dims mid, const float* __restrict__ mid_p) {
  const uint32_t x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 4 + threadIdx.y, z = blockIdx.z * 2 + threadIdx.z;
  if (x >= dm.w || y >= dm.h || z >= dm.d) return;
  const uint32_t i = flat(dm, x, y, z);
  dst[i] = is_boundary(dm, x, y, z) ? 0.0f : 0.0f + prolong_sample(mid, mid_p, (int)x, (int)y, (int)z);
}

inline dim3 lean_grid(Dims d) { return dim3((d.w + 31) / 32, (d.h + 3) / 4, (d.d + 1) / 2); }

// ---------------------------------------------------------------------------
// The mid and coarse levels of PressureSolvePass.solve (:73-82) in one
// cooperative launch: mid pre-smoothing, restriction to coarse, coarse
// smoothing, prolongation into mid pressureA and mid post-smoothing, separated
// by grid-wide barriers. The levels are small enough to stay in L2, so the
// launch-per-sweep cost of the reference schedule dominates without this.
// ---------------------------------------------------------------------------
struct MgArgs {
  Dims mid, coarse;
  float* mdiv;
  float* mp[2];
  float* cdiv;
  float* cp[2];
  int mid_pre, coarse_n, mid_post;
  unsigned* bar;  // [0] arrivals, [1] generation, [2] error flag
};

// Grid barrier with a bounded wait: after 2^24 polls of at least 64 ns (about a
// second; a correct barrier takes microseconds) the waiting block records an
// error and every block leaves the kernel.
FX_DEV bool grid_sync(unsigned* bar) {
  // bar[0]: arrivals, bar[32]: generation, bar[64]: error flag (separate 128-byte lines)
  __syncthreads();
  __shared__ int failed;
  if (threadIdx.x == 0) {
    failed = 0;
    volatile unsigned* vgen = bar + 32;
    volatile unsigned* verr = bar + 64;
    const unsigned gen = *vgen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u);
    if (arrived == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 32, 1u);
    } else {
      unsigned polls = 0;
      while (*vgen == gen) {
        __nanosleep(64);
        if (++polls > (1u << 24) || *verr) {
          atomicExch(bar + 64, 1u);
          failed = 1;
          break;
        }
      }
    }
    __threadfence();
  }
  __syncthreads();
  return failed == 0 && *((volatile unsigned*)bar + 64) == 0;
}

// Grid-stride walk over a level's voxels keeping (x, y, z) by carry instead of
// dividing each linear index by the dimensions.
struct Walk {
  uint32_t i, x, y, z, step, sx, sy, sz;
  FX_DEV Walk(const Dims& d) {
    i = blockIdx.x * blockDim.x + threadIdx.x;
    step = gridDim.x * blockDim.x;
    x = i % d.w;
    y = (i / d.w) % d.h;
    z = i / (d.w * d.h);
    sx = step % d.w;
    sy = (step / d.w) % d.h;
    sz = step / (d.w * d.h);
  }
  FX_DEV void next(const Dims& d) {
    i += step;
    x += sx;
    uint32_t cy = 0;
    if (x >= d.w) {
      x -= d.w;
      cy = 1;
    }
    y += sy + cy;
    uint32_t cz = 0;
    if (y >= d.h) {
      y -= d.h;
      cz = 1;
    }
    z += sz + cz;
  }
};

// A warp owns chunks of 32*MG_RUN consecutive voxels, lane-interleaved (so the
// accesses stay coalesced); each lane loads its MG_RUN voxels' operands before
// computing, which keeps MG_RUN independent loads in flight per thread.
constexpr int MG_RUN = 8;

FX_DEV void mg_sweep(const Dims& d, const float* __restrict__ div, const float* __restrict__ src, float* __restrict__ dst) {
  const uint32_t n = d.w * d.h * d.d;
  const uint32_t sy = d.w, sz = d.w * d.h;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t chunk = 32u * MG_RUN;
  for (uint32_t c0 = warp * chunk; c0 < n; c0 += nwarps * chunk) {
    uint32_t i0 = c0 + lane;
    uint32_t x = i0 % d.w, y = (i0 / d.w) % d.h, z = i0 / sz;
    float nb[MG_RUN][6], dv[MG_RUN];
    bool live[MG_RUN], interior[MG_RUN];
    uint32_t idx[MG_RUN];
#pragma unroll
    for (int k = 0; k < MG_RUN; ++k) {
      const uint32_t i = i0 + 32u * k;
      idx[k] = i;
      live[k] = i < n;
      interior[k] = live[k] && !is_boundary(d, x, y, z);
      if (interior[k]) {
        nb[k][0] = src[i + 1];
        nb[k][1] = src[i - 1];
        nb[k][2] = src[i + sy];
        nb[k][3] = src[i - sy];
        nb[k][4] = src[i + sz];
        nb[k][5] = src[i - sz];
        dv[k] = div[i];
      }
      // advance (x, y, z) by 32 voxels
      x += 32u;
      while (x >= d.w) {
        x -= d.w;
        if (++y >= d.h) {
          y = 0;
          ++z;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < MG_RUN; ++k) {
      if (!live[k]) continue;
      float v = 0.0f;
      if (interior[k]) {
        const float s = nb[k][0] + nb[k][1] + nb[k][2] + nb[k][3] + nb[k][4] + nb[k][5];
        v = div6(s - dv[k]);
      }
      dst[idx[k]] = v;
    }
  }
}

__global__ void __launch_bounds__(512) k_mg_lower(MgArgs a) {
  int m = 0;
  for (int k = 0; k < a.mid_pre; ++k, m ^= 1) {
    mg_sweep(a.mid, a.mdiv, a.mp[m], a.mp[m ^ 1]);
    if (!grid_sync(a.bar)) return;
  }
  const int mid_pre = m;
  {  // restriction mid -> coarse (pressure-restriction.wgsl.ts:27-50)
    const Dims& t = a.coarse;
    const Dims& sdm = a.mid;
    const uint32_t n = t.w * t.h * t.d;
    for (Walk w(t); w.i < n; w.next(t)) {
      const uint32_t i = w.i, x = w.x, y = w.y, z = w.z;
      if (x == 0u || y == 0u || z == 0u || x == t.w - 1u || y == t.h - 1u || z == t.d - 1u) {
        a.cdiv[i] = 0.0f;
        continue;
      }
      float sum = 0.0f;
      for (uint32_t dz = 0; dz < 2u; ++dz)
        for (uint32_t dy = 0; dy < 2u; ++dy)
          for (uint32_t dx = 0; dx < 2u; ++dx) {
            const uint32_t sx = min(2u * x + dx, sdm.w - 1u), sy = min(2u * y + dy, sdm.h - 1u), sz = min(2u * z + dz, sdm.d - 1u);
            sum += a.mdiv[flat(sdm, sx, sy, sz)];
          }
      a.cdiv[i] = sum * 0.125f;
    }
    if (!grid_sync(a.bar)) return;
  }
  int c = 0;
  for (int k = 0; k < a.coarse_n; ++k, c ^= 1) {
    mg_sweep(a.coarse, a.cdiv, a.cp[c], a.cp[c ^ 1]);
    if (!grid_sync(a.bar)) return;
  }
  {  // prolongation coarse -> mid pressureA (pressure-prolongation.wgsl.ts:29-44)
    const Dims& t = a.mid;
    const uint32_t n = t.w * t.h * t.d;
    for (Walk w(t); w.i < n; w.next(t)) {
      const uint32_t i = w.i, x = w.x, y = w.y, z = w.z;
      if (x == 0u || y == 0u || z == 0u || x == t.w - 1u || y == t.h - 1u || z == t.d - 1u) {
        a.mp[0][i] = 0.0f;
        continue;
      }
      const float px = ((float)x + 0.5f) * 0.5f - 0.5f;
      const float py = ((float)y + 0.5f) * 0.5f - 0.5f;
      const float pz = ((float)z + 0.5f) * 0.5f - 0.5f;
      a.mp[0][i] += tri_interp(a.cp[c], tri_corners(a.coarse, px, py, pz));
    }
    if (!grid_sync(a.bar)) return;
  }
  m = mid_pre;
  for (int k = 0; k < a.mid_post; ++k, m ^= 1) {
    mg_sweep(a.mid, a.mdiv, a.mp[m], a.mp[m ^ 1]);
    if (k + 1 < a.mid_post && !grid_sync(a.bar)) return;
  }
}

__global__ void k_div6_check(uint32_t hi_base, unsigned long long* bad) {
  const uint32_t u = hi_base + blockIdx.x * blockDim.x + threadIdx.x;
  const float x = __uint_as_float(u);
  if (x != x) return;
  const float a = div6(x), b = x / 6.0f;
  if (__float_as_uint(a) != __float_as_uint(b)) atomicAdd(bad, 1ull);
}

}  // namespace

cudaError_t zpass_launch(cudaStream_t s, const ZPass& p) {
  ZArgs a{};
  a.dm = p.dm;
  a.mid = p.mid;
  a.zchunk = p.zchunk > 0 ? p.zchunk : 64;
  a.p_in = p.p_in;
  a.div_in = p.div_in;
  a.div_out = p.div_out;
  a.mid_div = p.mid_div;
  a.mid_p = p.mid_p;
  a.p_out = p.p_out;
  a.vfin = p.vfin;
  a.vcur = p.vcur;
  a.vmag = p.vmag;
  a.write_vmag = p.write_vmag;
  a.restrict_mid = p.restrict_mid;
  const int S = std::min(p.sweeps, 4);
  if (p.div_from_velocity) {
    if (p.input != ZIN_ZERO || p.project || S < 1) return cudaErrorInvalidValue;
    return launch_s<IN_ZERO, true, false>(s, S, a);
  }
  switch (p.input) {
    case ZIN_BUF:
      return p.project ? launch_s<IN_BUF, false, true>(s, S, a) : launch_s<IN_BUF, false, false>(s, S, a);
    case ZIN_BUF_PROLONG:
      return p.project ? launch_s<IN_BUF_PROLONG, false, true>(s, S, a) : launch_s<IN_BUF_PROLONG, false, false>(s, S, a);
    case ZIN_ZERO_PROLONG:
      return p.project ? launch_s<IN_ZERO_PROLONG, false, true>(s, S, a) : launch_s<IN_ZERO_PROLONG, false, false>(s, S, a);
    default:
      return cudaErrorInvalidValue;
  }
}


int zpass_max_sweeps() {
  static const int k = env_int("FENIX_ZPASS_SWEEPS", 4, 1, 4);
  return k;
}

int zpass_zchunk() {
  static const int z = env_int("FENIX_ZPASS_ZCHUNK", 64, 8, 4096) & ~1;
  return z;
}

// k_div_march where the grid allows it (FENIX_DIV_MARCH=0 keeps k_div_first):
// widths divisible by 4, even heights and depths. Runs of an even number of
// planes such that the row tiles times the runs fill the resident blocks once.
cudaError_t lean_div_first(cudaStream_t s, Dims dm, VelField v, float* div, float* p1, Dims mid, float* mid_div, bool restrict_mid) {
  static const int march = env_int("FENIX_DIV_MARCH", 1, 0, 1);
  if (march && dm.w % 4 == 0 && dm.w >= 8 && dm.h % 2 == 0 && dm.d % 2 == 0) {
    static int slots[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    int n = (dev >= 0 && dev < 64) ? slots[dev] : 0;
    if (n <= 0) {
      int per_sm = 0, sms = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_div_march, 256, 0);
      if (e != cudaSuccess) return e;
      e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return e;
      n = std::max(1, per_sm) * std::max(1, sms);
      if (dev >= 0 && dev < 64) slots[dev] = n;
    }
    const int run = march_plan_pairs(dm, n);
    const dim3 g((dm.w + 127) / 128, (dm.h + 7) / 8, (dm.d + run - 1) / run);
    k_div_march<<<g, dim3(32, 8, 1), 0, s>>>(dm, v, div, p1, mid, mid_div, restrict_mid ? 1 : 0, run);
    return cudaGetLastError();
  }
  k_div_first<<<lean_grid(dm), dim3(32, 4, 2), 0, s>>>(dm, v, div, p1, mid, mid_div, restrict_mid ? 1 : 0);
  return cudaGetLastError();
}

bool sweep_variant_valid(int variant, Dims dm) {
  if (variant < 0 || variant >= kSweepVariants) return false;
  if (variant >= SWEEP_VEC4_Z2) return dm.w % 4 == 0 && dm.w >= 8;
  return variant < SWEEP_VEC_Z2 || (dm.w % 2 == 0 && dm.w >= 4);
}

int march_plan_one_wave(Dims dm, int slots) {
  const int tiles = (int)(((dm.w + 127) / 128) * ((dm.h + 7) / 8));
  const int runs = std::max(1, std::min((int)dm.d, std::max(slots, 1) / std::max(tiles, 1)));
  return ((int)dm.d + runs - 1) / runs;
}

int march_plan_pairs(Dims dm, int slots) {
  const int tiles = (int)(((dm.w + 127) / 128) * ((dm.h + 7) / 8));
  const int pairs = std::max(1, (int)dm.d / 2);
  const int runs = std::max(1, std::min(pairs, std::max(slots, 1) / std::max(tiles, 1)));
  return 2 * ((pairs + runs - 1) / runs);
}

int march_plan_waves(Dims dm, int tx, int ty, int slots) {
  const long n = std::max(slots, 1);
  const long tiles = (long)((dm.w + tx - 1) / tx) * (long)((dm.h + ty - 1) / ty);
  int best = 1;
  double best_eff = -1.0;
  for (int r = 1; r <= std::max(1, (int)dm.d / 8); ++r) {
    const int len = ((int)dm.d + r - 1) / r;
    const int runs = ((int)dm.d + len - 1) / len;
    const long blocks = tiles * runs;
    const long waves = (blocks + n - 1) / n;
    const double eff = (double)blocks / (double)(waves * n);
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = len;
    }
  }
  return best;
}

static cudaError_t march_run(Dims dm, int* run);

// The variant used when none was chosen: four x per thread marching in z where
// the width allows and a thread marches at least 8 planes (the 256^3 level of
// plume_256, 39.8 against 49.8 us per sweep), else four x per thread at z-depth
// 2 where the width allows (on the 128^3 and 64^3 levels the marching kernel
// gets 4 and 1 planes per thread and ties with it), else two x, else one.
// FENIX_SWEEP_VEC (0, 1, 2) caps the x per thread at 1, 2 or 4, and 2 also
// leaves out the marching kernel.
int sweep_variant_default(Dims dm) {
  static const int zb = env_int("FENIX_SWEEP_ZB", 4, 1, 8);
  static const int vec = env_int("FENIX_SWEEP_VEC", 3, 0, 3);
  static const int vzb = env_int("FENIX_SWEEP_VEC_ZB", 2, 2, 4);
  int run = 0;
  if (vec >= 3 && sweep_variant_valid(SWEEP_VEC4_MARCH, dm) && march_run(dm, &run) == cudaSuccess && run >= 8) return SWEEP_VEC4_MARCH;
  if (vec >= 2 && sweep_variant_valid(SWEEP_VEC4_Z2, dm)) return vzb <= 2 ? SWEEP_VEC4_Z2 : SWEEP_VEC4_Z4;
  if (vec >= 1 && sweep_variant_valid(SWEEP_VEC_Z2, dm)) return vzb <= 2 ? SWEEP_VEC_Z2 : SWEEP_VEC_Z4;
  return zb <= 2 ? SWEEP_Z2 : (zb <= 4 ? SWEEP_Z4 : SWEEP_Z8);
}

// Resident blocks of k_sweep_march on the current device (SMs x blocks per SM),
// looked up once per device.
static cudaError_t march_slots(int* slots) {
  static int cached[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < 64 && cached[dev] > 0) {
    *slots = cached[dev];
    return cudaSuccess;
  }
  int per_sm = 0, sms = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_march, 256, 0);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  *slots = std::max(1, per_sm) * std::max(1, sms);
  if (dev >= 0 && dev < 64) cached[dev] = *slots;
  return cudaSuccess;
}

// Planes per thread of k_sweep_march on a level: runs of planes such that the
// row tiles times the runs fill the resident slots once.
static cudaError_t march_run(Dims dm, int* run) {
  int slots = 0;
  const cudaError_t e = march_slots(&slots);
  if (e != cudaSuccess) return e;
  *run = march_plan_one_wave(dm, slots);
  return cudaSuccess;
}

// march_run for another marching kernel of 256-thread blocks over 128 x 8 row
// tiles (its own resident blocks, looked up once per device).
template <typename K>
static cudaError_t march_run_of(K kernel, Dims dm, int* run) {
  static int cached[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int slots = (dev >= 0 && dev < 64) ? cached[dev] : 0;
  if (slots <= 0) {
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    slots = std::max(1, per_sm) * std::max(1, sms);
    if (dev >= 0 && dev < 64) cached[dev] = slots;
  }
  *run = march_plan_one_wave(dm, slots);
  return cudaSuccess;
}

cudaError_t lean_sweep_variant(cudaStream_t s, int variant, Dims dm, const float* div, const float* src, float* dst, Dims mid,
                               const float* mid_p) {
  if (!sweep_variant_valid(variant, dm)) variant = sweep_variant_default(dm);
  auto grid = [&](int x_per_block, int z) { return dim3((dm.w + x_per_block - 1) / x_per_block, (dm.h + 7) / 8, (dm.d + z - 1) / z); };
  const dim3 block(32, 8, 1);
  switch (variant) {
    case SWEEP_Z2: k_sweep<2><<<grid(32, 2), block, 0, s>>>(dm, div, src, dst, mid, mid_p); break;
    case SWEEP_Z4: k_sweep<4><<<grid(32, 4), block, 0, s>>>(dm, div, src, dst, mid, mid_p); break;
    case SWEEP_Z8: k_sweep<8><<<grid(32, 8), block, 0, s>>>(dm, div, src, dst, mid, mid_p); break;
    case SWEEP_VEC_Z2: k_sweep_v2<2><<<grid(64, 2), block, 0, s>>>(dm, div, src, dst, mid, mid_p); break;
    case SWEEP_VEC_Z4: k_sweep_v2<4><<<grid(64, 4), block, 0, s>>>(dm, div, src, dst, mid, mid_p); break;
    case SWEEP_VEC4_Z2: k_sweep_v4<2><<<grid(128, 2), block, 0, s>>>(dm, div, src, dst, mid, mid_p); break;
    case SWEEP_VEC4_Z4: k_sweep_v4<4><<<grid(128, 4), block, 0, s>>>(dm, div, src, dst, mid, mid_p); break;
    case SWEEP_VEC4_Z1: k_sweep_v4<1><<<grid(128, 1), block, 0, s>>>(dm, div, src, dst, mid, mid_p); break;
    default: {
      int run = 0;
      const cudaError_t e = march_run(dm, &run);
      if (e != cudaSuccess) return e;
      // FENIX_PROLONG_MARCH=0 keeps k_sweep_v4<2> for the sweep with the prolongation
      static const bool prolong_march = env_int("FENIX_PROLONG_MARCH", 1, 0, 1) == 1;
      int prun = 0;
      const bool pm_ok = mid_p && dm.h % 2 == 0 && dm.d % 2 == 0 && mid.w * 2 == dm.w && mid.h * 2 == dm.h && mid.d * 2 == dm.d;
      if (pm_ok && prolong_march && march_run_of(k_sweep_march_prolong, dm, &prun) == cudaSuccess) {
        const dim3 g((dm.w + 127) / 128, (dm.h + 7) / 8, (dm.d + prun - 1) / prun);
        k_sweep_march_prolong<<<g, block, 0, s>>>(dm, div, src, dst, mid, mid_p, prun);
      } else if (mid_p) {
        k_sweep_v4<2><<<grid(128, 2), block, 0, s>>>(dm, div, src, dst, mid, mid_p);
      } else {
        const dim3 g((dm.w + 127) / 128, (dm.h + 7) / 8, (dm.d + run - 1) / run);
        k_sweep_march<<<g, block, 0, s>>>(dm, div, src, dst, run);
      }
      break;
    }
  }
  return cudaGetLastError();
}

cudaError_t lean_sweep(cudaStream_t s, Dims dm, const float* div, const float* src, float* dst, Dims mid, const float* mid_p) {
  return lean_sweep_variant(s, -1, dm, div, src, dst, mid, mid_p);
}

cudaError_t lean_prolong_zero(cudaStream_t s, Dims dm, float* dst, Dims mid, const float* mid_p) {
  k_prolong_zero<<<lean_grid(dm), dim3(32, 4, 2), 0, s>>>(dm, dst, mid, mid_p);
  return cudaGetLastError();
}

cudaError_t mg_lower_launch(cudaStream_t s, const LevelBuf& mid, const LevelBuf& coarse, int mid_pre, int coarse_n, int mid_post,
                            unsigned* bar, int* mid_result) {
  static int grid = 0;
  static int grid_dev = -1;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (grid == 0 || grid_dev != dev) {
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mg_lower, 512, 0);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    grid = std::max(1, std::min(per_sm, 2) * sms);
    grid_dev = dev;
  }
  MgArgs a;
  a.mid = mid.dm;
  a.coarse = coarse.dm;
  a.mdiv = mid.div;
  a.mp[0] = mid.p[0];
  a.mp[1] = mid.p[1];
  a.cdiv = coarse.div;
  a.cp[0] = coarse.p[0];
  a.cp[1] = coarse.p[1];
  a.mid_pre = mid_pre;
  a.coarse_n = coarse_n;
  a.mid_post = mid_post;
  a.bar = bar;
  *mid_result = (mid_pre & 1) ^ (mid_post & 1);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(512);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  e = cudaLaunchKernelEx(&cfg, k_mg_lower, a);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

int multigrid_plan() {
  static const int p = env_int("FENIX_MG_PLAN", 0, 0, 1);
  return p;
}

int pressure_plan() {
  static const int p = env_int("FENIX_PRESSURE_PLAN", 0, 0, 1);
  return p;
}

cudaError_t div6_exhaustive_check(unsigned long long* host_bad) {
  unsigned long long* d = nullptr;
  cudaError_t e = cudaMalloc(&d, sizeof(unsigned long long));
  if (e != cudaSuccess) return e;
  cudaMemset(d, 0, sizeof(unsigned long long));
  // 2^32 inputs in 256 launches of 2^24 (65536 blocks of 256 threads)
  for (uint32_t k = 0; k < 256; ++k) k_div6_check<<<65536, 256>>>(k << 24, d);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(host_bad, d, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return e;
}

}  // namespace fx
