// Sparse mode of the fused path (an extension; part of fx_fused.cu, included
// inside its anonymous namespace).
//
// The reference runs velocity advection, curl, confinement, divergence, the
// fine pressure sweeps and the projection over the whole grid
// (runtime/createCombustionVolumeSimulation.ts:270-296) while only a sixth of
// its bricks hold smoke. Sparse mode runs them on a set of bricks and keeps them
// zero outside it:
//  - velocity advection computes in the bricks flagged in the current set
//    (compute-active-bricks.wgsl.ts), 0 elsewhere;
//  - once the next set's flags exist, U = current | next flags; curl, |curl|,
//    confinement, divergence, every fine sweep, the fine prolongation and the
//    projection compute as the reference inside U and give 0 outside it.
// Scalar passes, injection, the mid and coarse levels and the restriction are
// the reference's. The oracle has the same mode (Sim::sparse), and each voxel
// computed here is the parity kernels' arithmetic in their order, so the two
// agree bit for bit.
//
// Fields keep their dense layout: a gather or stencil that leaves the set reads
// the zeros stored there, with no indirection. Per-brick "may be non-zero" bits
// of each buffer family tell which bricks outside the set still hold values of
// an earlier step; the lists the kernels walk are the set plus those bricks.
// An entry holds the brick's coordinates (10 bits each: x, then y, then z; at
// most 1024 bricks per axis) with bit 31 set where the brick is computed and
// clear where it is only zeroed, so no kernel divides to locate its brick.
constexpr uint32_t kSpCompute = 0x80000000u;
constexpr uint32_t kSpMaxBricksPerAxis = 1024;

FX_DEV uint32_t sp_pack(uint3 bc, uint32_t b, bool comp) {
  const uint32_t bx = b % bc.x, by = (b / bc.x) % bc.y, bz = b / (bc.x * bc.y);
  return bx | (by << 10) | (bz << 20) | (comp ? kSpCompute : 0u);
}
FX_DEV BrickCtx sp_ctx(const Dims& dm, uint32_t e) {
  BrickCtx c;
  c.bx = e & 1023u;
  c.by = (e >> 10) & 1023u;
  c.bz = (e >> 20) & 1023u;
  c.x0 = c.bx * 8u;
  c.y0 = c.by * 8u;
  c.z0 = c.bz * 8u;
  c.cx = min(c.x0 + 4u, dm.w - 1u);
  c.cy = min(c.y0 + 4u, dm.h - 1u);
  c.cz = min(c.z0 + 4u, dm.d - 1u);
  return c;
}
FX_DEV uint32_t sp_brick_index(uint3 bc, const BrickCtx& c) { return c.bx + bc.x * (c.by + bc.y * c.bz); }

// Buffer families with their own non-zero bits (FusedWork::nz_sp).
enum SpFamily { SP_VSCR = 0, SP_CURL = 1, SP_PRESSURE = 2, SP_VCUR = 3, kSpFamilies = 4 };

// Builds up to three lists over the bricks. For list k: a brick is computed when
// flags_a or flags_b (nullable) flags it, and listed when computed or when
// nz[k] marks it; nz[k] then marks exactly the computed bricks. extra (nullable)
// also receives the computed marks. Lists of families that are not due (null)
// are skipped, and their bits are left alone.
struct SpLists {
  uint32_t* list[3];
  uint32_t* count[3];
  uint8_t* nz[3];
};

__global__ void __launch_bounds__(256) k_sp_lists(uint3 bc, uint32_t nb, const uint32_t* __restrict__ flags_a,
                                                  const uint32_t* __restrict__ flags_b, SpLists L, uint8_t* __restrict__ extra) {
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31u;
  const bool live = b < nb;
  const bool comp = live && (__ldg(flags_a + b) != 0u || (flags_b && __ldg(flags_b + b) != 0u));
  if (live && extra) extra[b] = comp ? 1 : 0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (!L.list[k]) continue;  // uniform
    const bool take = comp || (live && L.nz[k][b] != 0);
    const unsigned ballot = __ballot_sync(0xffffffffu, take);
    uint32_t base = 0;
    if (lane == 0 && ballot) base = atomicAdd(L.count[k], (uint32_t)__popc(ballot));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (take) L.list[k][base + __popc(ballot & ((1u << lane) - 1u))] = sp_pack(bc, b, comp);
    if (live) L.nz[k][b] = comp ? 1 : 0;
  }
}

// Marks the bricks of a host-built list (the injection list) in nz.
__global__ void k_sp_mark(const uint32_t* __restrict__ list, const uint32_t* __restrict__ count, uint8_t* __restrict__ nz) {
  const uint32_t n = *count;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) nz[list[i]] = 1;
}

// The prolongation term of pressure-prolongation.wgsl.ts:42-43 at fine voxel (x, y, z).
FX_DEV float prolong_sample_at(const Dims& mid, const float* __restrict__ mp, int x, int y, int z) {
  const float px = ((float)x + 0.5f) * 0.5f - 0.5f;
  const float py = ((float)y + 0.5f) * 0.5f - 0.5f;
  const float pz = ((float)z + 0.5f) * 0.5f - 0.5f;
  return tri_interp(mp, tri_corners(mid, px, py, pz));
}

// Thread -> voxel of a 256-thread brick block: x = t & 7, y = (t >> 3) & 7 and
// z = t >> 6, plus 4 for the second voxel.
struct SpVoxel {
  uint32_t x, y, z, i;
  bool inside;
};
FX_DEV SpVoxel sp_voxel(const Dims& dm, const BrickCtx& c, int j) {
  SpVoxel v;
  v.x = c.x0 + (threadIdx.x & 7u);
  v.y = c.y0 + ((threadIdx.x >> 3) & 7u);
  v.z = c.z0 + ((threadIdx.x + kBrickThreads * j) >> 6);
  v.inside = v.x < dm.w && v.y < dm.h && v.z < dm.d;
  v.i = v.inside ? flat(dm, v.x, v.y, v.z) : 0u;
  return v;
}

// Column walk of the sparse kernels below: a block of 256 threads takes four list
// entries at a time, and thread t takes the (x, y) column (t & 7, (t >> 3) & 7) of
// entry 4 * block + (t >> 6) and its 8 z, so a brick's decoding and tests serve 8
// voxels and z neighbours stay in registers. A warp holds four rows of one brick.
constexpr uint32_t kSpColBricks = 4;

// advect-velocity-semilagrangian.wgsl.ts:23-41 in computed bricks, over
// vCurrent clamped to +-80/dx on read (advect_velocity_column<true>'s
// arithmetic); 0 in zeroed bricks. The next voxel's velocity is loaded before
// the current voxel's 24 gathers are issued.
__global__ void __launch_bounds__(kBrickThreads) k_sp_advect_velocity(Dims dm, uint3 bc, const Params* __restrict__ Pp, VelField src,
                                                                      VelField dst, const uint32_t* __restrict__ list,
                                                                      const uint32_t* __restrict__ count) {
  const float dt = Pp->dt;
  const float lim = speed_limit(*Pp);
  const float damp = 1.0f - dt * 0.025f;
  const uint32_t n = *count;
  const uint32_t lx = threadIdx.x & 7u, ly = (threadIdx.x >> 3) & 7u;
  const uint32_t sz = dm.w * dm.h;
  for (uint32_t li = blockIdx.x * kSpColBricks + (threadIdx.x >> 6); li < n; li += gridDim.x * kSpColBricks) {
    const uint32_t e = list[li];
    const BrickCtx c = sp_ctx(dm, e);
    const uint32_t x = c.x0 + lx, y = c.y0 + ly;
    if (x >= dm.w || y >= dm.h) continue;
    const uint32_t ze = min(c.z0 + 8u, dm.d);
    uint32_t i = x + dm.w * (y + dm.h * c.z0);
    const bool xyint = (e & kSpCompute) != 0u && x > 0u && y > 0u && x < dm.w - 1u && y < dm.h - 1u;
    if (!xyint) {
      for (uint32_t z = c.z0; z < ze; ++z, i += sz) {
        dst.c[0][i] = 0.0f;
        dst.c[1][i] = 0.0f;
        dst.c[2][i] = 0.0f;
      }
      continue;
    }
    float ax = __ldg(src.c[0] + i), ay = __ldg(src.c[1] + i), az = __ldg(src.c[2] + i);
    for (uint32_t z = c.z0; z < ze; ++z, i += sz) {
      const uint32_t in = z + 1u < ze ? i + sz : i;
      const float nx = __ldg(src.c[0] + in), ny = __ldg(src.c[1] + in), nz = __ldg(src.c[2] + in);
      float ox = 0.f, oy = 0.f, oz = 0.f;
      if (z > 0u && z < dm.d - 1u) {
        const float cx = (float)x + 0.5f, cy = (float)y + 0.5f, cz = (float)z + 0.5f;
        const float v0x = clampv(ax, -lim, lim), v0y = clampv(ay, -lim, lim), v0z = clampv(az, -lim, lim);
        const float bx = cx - v0x * dt, by = cy - v0y * dt, bz = cz - v0z * dt;
        const Tri c1 = tri_corners(dm, bx - 0.5f, by - 0.5f, bz - 0.5f);
        ox = tri_interp_clamped(src.c[0], c1, lim) * damp;
        oy = tri_interp_clamped(src.c[1], c1, lim) * damp;
        oz = tri_interp_clamped(src.c[2], c1, lim) * damp;
      }
      dst.c[0][i] = ox;
      dst.c[1][i] = oy;
      dst.c[2][i] = oz;
      ax = nx;
      ay = ny;
      az = nz;
    }
  }
}

// compute-vorticity.wgsl.ts:23-50: |w| (w itself with debug fields) in computed
// bricks, 0 in zeroed bricks and on the boundary.
__global__ void __launch_bounds__(kBrickThreads) k_sp_vorticity(Dims dm, uint3 bc, VelField v, float* __restrict__ wmag, VelField w,
                                                                int write_w, const uint32_t* __restrict__ list,
                                                                const uint32_t* __restrict__ count) {
  const uint32_t n = *count;
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  for (uint32_t li = blockIdx.x; li < n; li += gridDim.x) {
    const uint32_t e = list[li];
    const bool comp = (e & kSpCompute) != 0u;
    const BrickCtx c = sp_ctx(dm, e);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const SpVoxel q = sp_voxel(dm, c, j);
      if (!q.inside) continue;
      float cx = 0.f, cy = 0.f, cz = 0.f;
      const bool live = comp && !is_boundary(dm, q.x, q.y, q.z);
      if (live) curl_at(v, q.i, sy, sz, cx, cy, cz);
      wmag[q.i] = live ? length3(cx, cy, cz) : 0.0f;
      if (write_w) {
        w.c[0][q.i] = cx;
        w.c[1][q.i] = cy;
        w.c[2][q.i] = cz;
      }
    }
  }
}

// apply-vorticity-confinement.wgsl.ts:30-66 in computed bricks (k_confinement's
// arithmetic, out = vScratch + F dt clamped); the boundary passes vScratch
// through, and zeroed bricks get 0 (vScratch is 0 there). Column walk: the z
// neighbours of |w|, vx and vy (the gradient's and the curl's z terms) stay in
// registers; each voxel's values and operations are k_confinement's.
template <typename S, bool FMAG>
__global__ void __launch_bounds__(kBrickThreads) k_sp_confinement(Dims dm, uint3 bc, const Params* __restrict__ Pp, VelField v,
                                                                  const float* __restrict__ wmag, SSet<S> set, const uint8_t* __restrict__ nz,
                                                                  VelField out, float* __restrict__ fmag, const uint32_t* __restrict__ list,
                                                                  const uint32_t* __restrict__ count) {
  const Params P = *Pp;
  const uint32_t n = *count;
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const uint32_t lx = threadIdx.x & 7u, ly = (threadIdx.x >> 3) & 7u;
  for (uint32_t li = blockIdx.x * kSpColBricks + (threadIdx.x >> 6); li < n; li += gridDim.x * kSpColBricks) {
    const uint32_t e = list[li];
    const BrickCtx c = sp_ctx(dm, e);
    const uint32_t x = c.x0 + lx, y = c.y0 + ly;
    if (x >= dm.w || y >= dm.h) continue;
    const uint32_t ze = min(c.z0 + 8u, dm.d);
    uint32_t i = x + dm.w * (y + dm.h * c.z0);
    if (!(e & kSpCompute)) {
      for (uint32_t z = c.z0; z < ze; ++z, i += sz) {
        out.c[0][i] = 0.0f;
        out.c[1][i] = 0.0f;
        out.c[2][i] = 0.0f;
        if (FMAG) fmag[i] = 0.0f;
      }
      continue;
    }
    const bool xyint = x > 0u && y > 0u && x < dm.w - 1u && y < dm.h - 1u;
    if (!xyint) {  // boundary column: vScratch passes through
      for (uint32_t z = c.z0; z < ze; ++z, i += sz) {
        out.c[0][i] = __ldg(v.c[0] + i);
        out.c[1][i] = __ldg(v.c[1] + i);
        out.c[2][i] = __ldg(v.c[2] + i);
        if (FMAG) fmag[i] = 0.0f;
      }
      continue;
    }
    const bool scal = __ldg(nz + sp_brick_index(bc, c)) != 0;
    // planes z - 1, z, z + 1 of |w|, vx and vy (reads at z - 1 < 0 or z + 1 >= d are never used)
    auto at = [&](const float* f, uint32_t z) { return z < dm.d ? __ldg(f + x + dm.w * (y + dm.h * z)) : 0.0f; };
    float wm = c.z0 > 0u ? at(wmag, c.z0 - 1u) : 0.0f, w0 = at(wmag, c.z0);
    float xm = c.z0 > 0u ? at(v.c[0], c.z0 - 1u) : 0.0f, x0 = at(v.c[0], c.z0);
    float ym = c.z0 > 0u ? at(v.c[1], c.z0 - 1u) : 0.0f, y0 = at(v.c[1], c.z0);
    for (uint32_t z = c.z0; z < ze; ++z, i += sz) {
      const float wp = at(wmag, z + 1u), xp = at(v.c[0], z + 1u), yp = at(v.c[1], z + 1u);
      float vx = x0, vy = y0, vz = __ldg(v.c[2] + i);
      if (z == 0u || z == dm.d - 1u) {
        out.c[0][i] = vx;
        out.c[1][i] = vy;
        out.c[2][i] = vz;
        if (FMAG) fmag[i] = 0.0f;
      } else {
        const float gx = (__ldg(wmag + i + 1u) - __ldg(wmag + i - 1u)) * 0.5f;
        const float gy = (__ldg(wmag + i + sy) - __ldg(wmag + i - sy)) * 0.5f;
        const float gz = (wp - wm) * 0.5f;
        // curl_at with the z terms from the column
        const float wx = ((__ldg(v.c[2] + i + sy) - __ldg(v.c[2] + i - sy)) - (yp - ym)) * 0.5f;
        const float wy = ((xp - xm) - (__ldg(v.c[2] + i + 1u) - __ldg(v.c[2] + i - 1u))) * 0.5f;
        const float wz = ((__ldg(v.c[1] + i + 1u) - __ldg(v.c[1] + i - 1u)) - (__ldg(v.c[0] + i + sy) - __ldg(v.c[0] + i - sy))) * 0.5f;
        float d = 0.f, t = 0.f, r = 0.f;
        if (scal) {
          d = ldS(set.f[0], i);
          t = ldS(set.f[1], i);
          r = ldS(set.f[3], i);
        }
        if (FMAG) {
          fmag[i] = confinement_voxel(P, gx, gy, gz, wx, wy, wz, w0, d, t, r, vx, vy, vz);
        } else {
          confinement_voxel_v(P, gx, gy, gz, wx, wy, wz, w0, d, t, r, vx, vy, vz);
        }
        out.c[0][i] = vx;
        out.c[1][i] = vy;
        out.c[2][i] = vz;
      }
      wm = w0;
      w0 = wp;
      xm = x0;
      x0 = xp;
      ym = y0;
      y0 = yp;
    }
  }
}

// compute-divergence.wgsl.ts:22-42 in computed bricks (0 in zeroed bricks and on
// the boundary), with the first Jacobi sweep from the cleared buffer,
// (0 - div) / 6, when p1 is given, and the restriction of the brick's
// divergence into the mid cells it covers (pressure-restriction.wgsl.ts:27-50:
// the mean of the clamped 2x2x2 children, 0 on the mid boundary). Every mid cell
// m lies in fine brick m >> 2 (the mid level is at most half the fine one, or 4
// cells on a grid under 8), and so do its clamped children.
__global__ void __launch_bounds__(kBrickThreads) k_sp_div_first(Dims dm, uint3 bc, VelField v, float* __restrict__ div, float* __restrict__ p1,
                                                                Dims mid, float* __restrict__ mid_div, const uint32_t* __restrict__ list,
                                                                const uint32_t* __restrict__ count) {
  __shared__ float sd[512];
  const uint32_t n = *count;
  for (uint32_t li = blockIdx.x; li < n; li += gridDim.x) {
    const uint32_t e = list[li];
    const bool comp = (e & kSpCompute) != 0u;
    const BrickCtx c = sp_ctx(dm, e);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const SpVoxel q = sp_voxel(dm, c, j);
      float dv = 0.0f;
      if (q.inside) {
        const bool live = comp && !is_boundary(dm, q.x, q.y, q.z);
        if (live) {
          const Nbr nb = neighbours(dm, q.x, q.y, q.z, q.i);
          const float ddx = __ldg(v.c[0] + nb.xp) - __ldg(v.c[0] + nb.xm);
          const float ddy = __ldg(v.c[1] + nb.yp) - __ldg(v.c[1] + nb.ym);
          const float ddz = __ldg(v.c[2] + nb.zp) - __ldg(v.c[2] + nb.zm);
          dv = (ddx + ddy + ddz) * 0.5f;
        }
        div[q.i] = dv;
        if (p1) p1[q.i] = live ? div6(0.0f - dv) : 0.0f;
      }
      sd[threadIdx.x + kBrickThreads * j] = dv;
    }
    __syncthreads();
    if (threadIdx.x < 64u) {
      const uint32_t mx = c.bx * 4u + (threadIdx.x & 3u), my = c.by * 4u + ((threadIdx.x >> 2) & 3u), mz = c.bz * 4u + (threadIdx.x >> 4);
      if (mx < mid.w && my < mid.h && mz < mid.d) {
        float out = 0.0f;
        if (mx != 0u && my != 0u && mz != 0u && mx != mid.w - 1u && my != mid.h - 1u && mz != mid.d - 1u) {
          float sum = 0.0f;
          for (uint32_t dz = 0; dz < 2u; ++dz)
            for (uint32_t dy = 0; dy < 2u; ++dy)
              for (uint32_t dx = 0; dx < 2u; ++dx) {
                const uint32_t fx = min(2u * mx + dx, dm.w - 1u) - c.x0, fy = min(2u * my + dy, dm.h - 1u) - c.y0,
                               fz = min(2u * mz + dz, dm.d - 1u) - c.z0;
                sum += sd[fx + 8u * (fy + 8u * fz)];
              }
          out = sum * 0.125f;
        }
        mid_div[flat(mid, mx, my, mz)] = out;
      }
    }
    __syncthreads();
  }
}

// One fine Jacobi sweep (pressure-jacobi.wgsl.ts:15-36) in computed bricks, 0 in
// zeroed bricks and on the boundary. src NULL is the cleared buffer. With mid_p,
// the prolongation of the mid level is added to each interior result
// (pressure-prolongation.wgsl.ts:36-43, as k_sweep does); with `only_prolong`,
// the result is 0 + the prolongation (the cleared buffer prolonged into).
__global__ void __launch_bounds__(kBrickThreads) k_sp_sweep(Dims dm, uint3 bc, const float* __restrict__ div, const float* __restrict__ src,
                                                            float* __restrict__ dst, Dims mid, const float* __restrict__ mid_p, int only_prolong,
                                                            const uint32_t* __restrict__ list, const uint32_t* __restrict__ count) {
  const uint32_t n = *count;
  for (uint32_t li = blockIdx.x; li < n; li += gridDim.x) {
    const uint32_t e = list[li];
    const bool comp = (e & kSpCompute) != 0u;
    const BrickCtx c = sp_ctx(dm, e);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const SpVoxel q = sp_voxel(dm, c, j);
      if (!q.inside) continue;
      float out = 0.0f;
      if (comp && !is_boundary(dm, q.x, q.y, q.z)) {
        if (only_prolong) {
          out = 0.0f + prolong_sample_at(mid, mid_p, (int)q.x, (int)q.y, (int)q.z);
        } else {
          const uint32_t sy = dm.w, sz = dm.w * dm.h, i = q.i;
          float s = 0.0f;
          if (src) s = __ldg(src + i + 1u) + __ldg(src + i - 1u) + __ldg(src + i + sy) + __ldg(src + i - sy) + __ldg(src + i + sz) + __ldg(src + i - sz);
          out = div6((src ? s : 0.0f) - __ldg(div + i));
          if (mid_p) out = out + prolong_sample_at(mid, mid_p, (int)q.x, (int)q.y, (int)q.z);
        }
      }
      dst[q.i] = out;
    }
  }
}

// project-velocity.wgsl.ts:21-43 in computed bricks (vCurrent = vScratch - the
// central pressure gradient), 0 in zeroed bricks and on the boundary.
__global__ void __launch_bounds__(kBrickThreads) k_sp_project(Dims dm, uint3 bc, VelField vs, const float* __restrict__ p, VelField vd,
                                                              const uint32_t* __restrict__ list, const uint32_t* __restrict__ count) {
  const uint32_t n = *count;
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  for (uint32_t li = blockIdx.x; li < n; li += gridDim.x) {
    const uint32_t e = list[li];
    const bool comp = (e & kSpCompute) != 0u;
    const BrickCtx c = sp_ctx(dm, e);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const SpVoxel q = sp_voxel(dm, c, j);
      if (!q.inside) continue;
      float ox = 0.f, oy = 0.f, oz = 0.f;
      if (comp && !is_boundary(dm, q.x, q.y, q.z)) {
        const uint32_t i = q.i;
        const float gx = (__ldg(p + i + 1u) - __ldg(p + i - 1u)) * 0.5f;
        const float gy = (__ldg(p + i + sy) - __ldg(p + i - sy)) * 0.5f;
        const float gz = (__ldg(p + i + sz) - __ldg(p + i - sz)) * 0.5f;
        ox = __ldg(vs.c[0] + i) - gx;
        oy = __ldg(vs.c[1] + i) - gy;
        oz = __ldg(vs.c[2] + i) - gz;
      }
      vd.c[0][q.i] = ox;
      vd.c[1][q.i] = oy;
      vd.c[2][q.i] = oz;
    }
  }
}

// |v| (compute-debug-fields.wgsl.ts:18-25) over the whole grid.
__global__ void __launch_bounds__(256) k_sp_velocity_magnitude(Dims dm, VelField v, float* __restrict__ out) {
  const uint32_t n = dm.w * dm.h * dm.d;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = length3(__ldg(v.c[0] + i), __ldg(v.c[1] + i), __ldg(v.c[2] + i));
}

// ------------------------------------------------------------------ TMA staging
// The sparse fine sweep with each brick's source tile staged in shared memory by
// the tensor-memory accelerator: one 3-D tile load of 16 x 10 x 10 floats (the
// brick, its one-voxel halo in y and z, and x from x0 - 4 so the tile starts on
// a 16-byte boundary) and one of the brick's 8 x 8 x 8 divergence, completing on
// an mbarrier. A block walks its list entries with two stages: the loads of the
// next entry are in flight while the current one is computed. Loads outside the
// grid read 0 (they only reach the halo of boundary voxels, which are not
// computed). The tensor maps cover this GPU's own buffers; no multicast.
constexpr int kSpTileFloats = 16 * 10 * 10;
constexpr int kSpDivFloats = 8 * 8 * 8;
constexpr uint32_t kSpStageBytes = (kSpTileFloats + kSpDivFloats) * 4;

FX_DEV uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

FX_DEV void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

FX_DEV void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

FX_DEV bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

FX_DEV uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for the phase `parity` of *bar for at most limit_ns; false on timeout.
FX_DEV bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_test(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_test(bar, parity))
    if (global_ns() - t0 > limit_ns) return false;
  return true;
}

FX_DEV void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

// k_sp_sweep (src given) from TMA-staged tiles; the same operations in the same
// order, so the same bits. A block of 128 threads takes a brick at a time; a
// thread owns one (x, y) of it and four consecutive z, so the brick's decoding,
// tests and index arithmetic are shared by four voxels and the z neighbours of
// its column are read once. Three stages: the loads of the next two entries are
// in flight while one is computed. `wait_ns` bounds every wait on a tile: when one
// runs out the block sets *err, waits (bounded again) for its loads in flight and
// returns. `extra_tx` adds to the bytes a stage expects and is 0 except in the
// test of that timeout path, where the stage then never completes.
constexpr int kSpSweepThreads = 128;
constexpr int kSpStages = 3;

__global__ void __launch_bounds__(kSpSweepThreads) k_sp_sweep_tma(const __grid_constant__ CUtensorMap src_map,
                                                                  const __grid_constant__ CUtensorMap div_map, Dims dm, uint3 bc,
                                                                  float* __restrict__ dst, Dims mid, const float* __restrict__ mid_p,
                                                                  const uint32_t* __restrict__ list, const uint32_t* __restrict__ count,
                                                                  uint32_t* __restrict__ err, uint64_t wait_ns, uint32_t extra_tx) {
  __shared__ __align__(128) float tile[kSpStages][kSpTileFloats + kSpDivFloats];
  __shared__ __align__(8) uint64_t bar[kSpStages];
  const uint32_t n = *count;
  if (threadIdx.x == 0) {
    for (int k = 0; k < kSpStages; ++k) mbar_init(&bar[k], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // Thread 0 starts the loads of list entry li into `stage` (computed entries only).
  auto issue = [&](uint32_t li, int stage) {
    const uint32_t e = list[li];
    if (!(e & kSpCompute)) return false;
    const BrickCtx c = sp_ctx(dm, e);
    mbar_arrive_expect_tx(&bar[stage], kSpStageBytes + extra_tx);
    tma_load_3d(&tile[stage][0], &src_map, (int)c.x0 - 4, (int)c.y0 - 1, (int)c.z0 - 1, &bar[stage]);
    tma_load_3d(&tile[stage][kSpTileFloats], &div_map, (int)c.x0, (int)c.y0, (int)c.z0, &bar[stage]);
    return true;
  };
  // bit k of `issued`: stage k has loads in flight; bit k of `parity`: the phase it waits for
  uint32_t issued = 0u, parity = 0u;
  if (threadIdx.x == 0)
    for (int k = 0; k < kSpStages - 1; ++k) {
      const uint32_t li = blockIdx.x + (uint32_t)k * gridDim.x;
      if (li < n && issue(li, k)) issued |= 1u << k;
    }
  const uint32_t lx = threadIdx.x & 7u, ly = (threadIdx.x >> 3) & 7u, lz0 = (threadIdx.x >> 6) * 4u;
  const uint32_t sz = dm.w * dm.h;
  int stage = 0;
  for (uint32_t li = blockIdx.x; li < n; li += gridDim.x) {
    // keep kSpStages - 1 entries ahead in flight (that stage was read two iterations ago)
    const uint32_t ahead = li + (uint32_t)(kSpStages - 1) * gridDim.x;
    const int ast = (stage + kSpStages - 1) % kSpStages;
    if (threadIdx.x == 0 && ahead < n && issue(ahead, ast)) issued |= 1u << ast;
    const uint32_t e = list[li];
    const bool comp = (e & kSpCompute) != 0u;
    const BrickCtx c = sp_ctx(dm, e);
    if (comp) {
      const uint32_t ph = (parity >> stage) & 1u;
      const bool ok = mbar_wait_bounded(&bar[stage], ph, wait_ns);
      if (__syncthreads_or(ok ? 0 : 1)) {
        // A tile never arrived: record it, let the loads in flight land, leave.
        if (threadIdx.x == 0) {
          atomicOr(err, 1u);
          for (int k = 0; k < kSpStages; ++k)
            if (issued & (1u << k)) mbar_wait_bounded(&bar[k], (parity >> k) & 1u, wait_ns);
        }
        __syncthreads();
        return;
      }
      parity ^= 1u << stage;
      issued &= ~(1u << stage);
    }
    const uint32_t x = c.x0 + lx, y = c.y0 + ly;
    if (x < dm.w && y < dm.h) {
      const bool xyint = comp && x > 0u && y > 0u && x < dm.w - 1u && y < dm.h - 1u;
      const float* T = tile[stage];
      const float* Dv = tile[stage] + kSpTileFloats;
      const uint32_t col = (lx + 4u) + 16u * (ly + 1u);  // tile index of (x, y) at tile plane 0
      const uint32_t base = x + dm.w * y;
      float zc[6];
      if (xyint) {
#pragma unroll
        for (int k = 0; k < 6; ++k) zc[k] = T[col + 160u * (lz0 + (uint32_t)k)];  // planes lz0 - 1 .. lz0 + 4
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const uint32_t lz = lz0 + (uint32_t)k, z = c.z0 + lz;
        if (z >= dm.d) break;
        float out = 0.0f;
        if (xyint && z > 0u && z < dm.d - 1u) {
          const uint32_t t = col + 160u * (lz + 1u);
          const float s = T[t + 1u] + T[t - 1u] + T[t + 16u] + T[t - 16u] + zc[k + 2] + zc[k];
          out = div6(s - Dv[lx + 8u * (ly + 8u * lz)]);
          if (mid_p) out = out + prolong_sample_at(mid, mid_p, (int)x, (int)y, (int)z);
        }
        dst[base + sz * z] = out;
      }
    }
    __syncthreads();  // the stage is read; a later iteration may reload it
    stage = (stage + 1) % kSpStages;
  }
}

// Host: the tensor-map encoder of the driver (cuTensorMapEncodeTiled), reached
// through the runtime so the library needs no link to libcuda.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                                   const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
      return (EncodeTiledFn) nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// A 3-D tensor map over a dense float field of dm (x fastest) with a bx x by x bz
// box; false where the layout does not allow one (widths not divisible by 4).
bool field_tensor_map(CUtensorMap* m, const float* base, Dims dm, uint32_t bx, uint32_t by, uint32_t bz) {
  const EncodeTiledFn enc = encode_tiled();
  if (!enc || dm.w % 4u != 0u || (reinterpret_cast<uintptr_t>(base) & 15u) != 0u) return false;
  const cuuint64_t dims[3] = {dm.w, dm.h, dm.d};
  const cuuint64_t strides[2] = {(cuuint64_t)dm.w * 4u, (cuuint64_t)dm.w * dm.h * 4u};
  const cuuint32_t box[3] = {bx, by, bz};
  const cuuint32_t es[3] = {1u, 1u, 1u};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
