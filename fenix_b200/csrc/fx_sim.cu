// The simulation object behind the C ABI of include/fenix_cuda.h: buffer
// ownership, the reference's per-step schedule
// (runtime/createCombustionVolumeSimulation.ts:230-305), its parameter and
// quality handling, and the multilevel pressure schedule
// (runtime/passes/PressureSolvePass.ts:62-158).
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <map>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include <cuda_fp16.h>

#include "../../include/fenix_cuda.h"
#include "fx_adjoint.h"
#include "fx_fused.h"
#include "fx_kernels.h"
#include "fx_pressure.h"

using namespace fx;

namespace {

thread_local std::string g_last_error;

constexpr int kParamSlots = 32;

// Per-kernel CUDA-event timing on the simulation's stream (FX_INSTR_KERNEL_TIMES).
struct KernelTimer {
  bool on = false;
  struct Pending {
    const char* name;
    cudaEvent_t a, b;
  };
  std::vector<cudaEvent_t> pool;
  std::vector<Pending> pending;
  std::map<std::string, std::pair<uint32_t, double>> acc;
  const char* open_name = nullptr;
  cudaEvent_t open_a = nullptr;

  cudaEvent_t take() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
  }
  void begin(cudaStream_t s, const char* name) {
    if (!on) return;
    open_name = name;
    open_a = take();
    cudaEventRecord(open_a, s);
  }
  void end(cudaStream_t s) {
    if (!on || !open_name) return;
    cudaEvent_t b = take();
    cudaEventRecord(b, s);
    pending.push_back({open_name, open_a, b});
    open_name = nullptr;
  }
  void drain() {
    for (auto& p : pending) {
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, p.a, p.b);
      auto& e = acc[p.name];
      e.first += 1;
      e.second += ms;
      pool.push_back(p.a);
      pool.push_back(p.b);
    }
    pending.clear();
  }
  void release() {
    drain();
    for (auto e : pool) cudaEventDestroy(e);
    pool.clear();
  }
};

}  // namespace

struct fx_sim {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  Dims dm{};
  uint32_t n = 0;
  uint3 bricks{};
  uint32_t nb = 0;
  int kernels = FX_KERNELS_FUSED;
  uint32_t opt_flags = 0;
  bool half = false;  // FX_OPT_SCALARS_F16: the scalar sets are binary16 buffers
  bool sparse = false;  // FX_OPT_SPARSE / fx_sim_set_sparse
  bool half_nearest = false;  // FX_OPT_F16_ROUND_NEAREST
  fx_solver_settings solver{};
  uint32_t last_cycle_launches = 0;  // kernels per V-cycle in the latest step
  int sweep_variant[3] = {-1, -1, -1};  // sweep kernel per pressure level, chosen by fx_sim_autotune
  uint8_t brick_ctas[kBrickKernels] = {};  // CTAs per SM of the brick kernels (0 = default), fx_sim_autotune_bricks
  int last_solver_mode = 0;

  // device memory
  void* arena = nullptr;
  size_t arena_bytes = 0;
  ScalarSet sets[3]{};  // [0], [1]: the reference's two sets; [2]: scratch (snapshot / advected)
  VelField vcur{}, vscr{}, vscr2{}, vort{};
  float* vort_mag = nullptr;
  float* conf_mag = nullptr;
  float* vel_mag = nullptr;
  uint32_t* flags[2]{};
  LevelBuf lv[3]{};
  LevelBuf xlv[3]{};  // V-cycle levels 3..5
  Params* d_params = nullptr;
  FusedWork fw{};

  // sources
  float* d_sources = nullptr;
  uint32_t src_cap = 0;   // in sources
  uint32_t src_count = 0; // as given (0 -> one zero "phantom" source on device)
  float* h_src_stage = nullptr;
  uint32_t h_src_cap = 0;
  cudaEvent_t src_event = nullptr;
  std::vector<float> host_sources;  // packed copy, used for the injection bounds

  // pinned parameter ring
  Params* h_params = nullptr;
  cudaEvent_t param_events[kParamSlots]{};
  uint64_t param_counter = 0;

  // reference host state (createCombustionVolumeSimulation.ts:180-204)
  int cur = 0;
  int64_t step_index = 0;
  bool initialized = false;
  double start_s = 0, last_elapsed_s = 0;
  int last_p = 0;
  bool debug_requested = false;
  int advect_mode = FX_ADVECT_MACCORMACK;
  fx_quality quality{};
  int qi[7]{};  // clamped integers of `quality`
  fx_runtime_params rp{};
  uint32_t last_kernel_count = 0;
  bool last_step_graph = false;
  uint32_t instr = 0;
  KernelTimer timer;
  unsigned long long* d_active_acc = nullptr;  // [0] brick-steps, [1] voxel-steps
  // In the fused path the final velocity of the step may live in vscr2.
  VelField* final_vscr = nullptr;

  std::string err;
};

namespace fx {

int device_sm_count() {
  static int cache[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 1;
  if (cache[dev] <= 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) return 1;
    cache[dev] = n;
  }
  return cache[dev];
}

namespace {
// 0: off; n > 0: the n-th allocation from now on fails.
std::atomic<int> g_alloc_countdown{0};

bool injected_allocation_failure() {
  int c = g_alloc_countdown.load();
  while (c > 0)
    if (g_alloc_countdown.compare_exchange_weak(c, c - 1)) return c == 1;
  return false;
}
}  // namespace

cudaError_t device_alloc(void** ptr, size_t bytes) {
  if (injected_allocation_failure()) {
    *ptr = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(ptr, bytes);
}

cudaError_t host_alloc(void** ptr, size_t bytes) {
  if (injected_allocation_failure()) {
    *ptr = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMallocHost(ptr, bytes);
}

}  // namespace fx

namespace {

fx_status fail(fx_sim* s, fx_status code, const std::string& msg) {
  if (s) {
    if (s->err.empty()) s->err = msg;
  } else {
    g_last_error = msg;
  }
  return code;
}

#define FX_CUDA(sim, call)                                                                  \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return fail((sim), e_ == cudaErrorMemoryAllocation ? FX_ERR_OUT_OF_MEMORY : FX_ERR_CUDA, \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                      \
  } while (0)

// clampInteger of types.ts:26-28 with JavaScript Math.round (half toward +inf).
double js_round(double v) {
  const double f = std::floor(v);
  return (v - f >= 0.5) ? f + 1.0 : f;
}
int clamp_integer(double v, int lo, int hi) { return (int)std::max<double>(lo, std::min<double>(hi, js_round(v))); }

void apply_quality_clamps(fx_sim* s) {
  const fx_quality& q = s->quality;
  s->qi[0] = clamp_integer(q.pressure_interval, 1, 16);
  s->qi[1] = clamp_integer(q.vorticity_interval, 1, 16);
  s->qi[2] = clamp_integer(q.fine_pre_iterations, 0, 32);
  s->qi[3] = clamp_integer(q.fine_post_iterations, 0, 32);
  s->qi[4] = clamp_integer(q.mid_pre_iterations, 0, 32);
  s->qi[5] = clamp_integer(q.mid_post_iterations, 0, 32);
  s->qi[6] = clamp_integer(q.coarse_iterations, 0, 64);
  // Store the clamped values back, as createSimulationQualitySettings returns them.
  s->quality.pressure_interval = s->qi[0];
  s->quality.vorticity_interval = s->qi[1];
  s->quality.fine_pre_iterations = s->qi[2];
  s->quality.fine_post_iterations = s->qi[3];
  s->quality.mid_pre_iterations = s->qi[4];
  s->quality.mid_post_iterations = s->qi[5];
  s->quality.coarse_iterations = s->qi[6];
}

bool merge_quality(fx_quality& dst, const fx_quality& src, uint32_t mask) {
  const double* sv = &src.pressure_interval;
  double* dv = &dst.pressure_interval;
  for (int k = 0; k < 7; ++k)
    if (mask & (1u << k)) {
      if (std::isnan(sv[k])) return false;
      dv[k] = sv[k];
    }
  return true;
}

void merge_params(fx_runtime_params& d, const fx_runtime_params& s, uint32_t m) {
  if (m & FX_PARAM_WIND) std::memcpy(d.wind, s.wind, sizeof d.wind);
  if (m & FX_PARAM_WIND_STRENGTH) d.wind_strength = s.wind_strength;
  if (m & FX_PARAM_GRAVITY) std::memcpy(d.gravity, s.gravity, sizeof d.gravity);
  if (m & FX_PARAM_GRAVITY_STRENGTH) d.gravity_strength = s.gravity_strength;
  if (m & FX_PARAM_BUOYANCY) d.buoyancy = s.buoyancy;
  if (m & FX_PARAM_VORTICITY_STRENGTH) d.vorticity_strength = s.vorticity_strength;
  if (m & FX_PARAM_VORTICITY_CONSTANT_MASK) d.vorticity_constant_mask = s.vorticity_constant_mask;
  if (m & FX_PARAM_VORTICITY_VELOCITY_MASK) d.vorticity_velocity_mask = s.vorticity_velocity_mask;
  if (m & FX_PARAM_VORTICITY_HEAT_MASK) d.vorticity_heat_mask = s.vorticity_heat_mask;
  if (m & FX_PARAM_VORTICITY_DENSITY_MASK) d.vorticity_density_mask = s.vorticity_density_mask;
  if (m & FX_PARAM_WORLD_SIZE) d.world_size = s.world_size;
}

Dims halve(Dims a) {
  return Dims{std::max<uint32_t>(4, a.w / 2), std::max<uint32_t>(4, a.h / 2), std::max<uint32_t>(4, a.d / 2)};
}

size_t count_of(Dims d) { return (size_t)d.w * d.h * d.d; }

fx_status zero_state(fx_sim* s) {
  // doReset (createCombustionVolumeSimulation.ts:213-225) clears everything the
  // step reads; clearing the whole arena is a superset.
  FX_CUDA(s, cudaMemsetAsync(s->arena, 0, s->arena_bytes, s->stream));
  return FX_OK;
}

fx_status upload_sources(fx_sim* s) {
  // SourceInjectionPass.ts:13-23,71-83: a buffer of max(bytes, 128); with no
  // sources the kernels see one all-zero entry.
  const uint32_t dev_count = std::max<uint32_t>(s->src_count, 1);
  if (dev_count > s->src_cap) {
    FX_CUDA(s, cudaStreamSynchronize(s->stream));
    if (s->d_sources) FX_CUDA(s, cudaFree(s->d_sources));
    s->d_sources = nullptr;
    const uint32_t cap = std::max<uint32_t>(dev_count, 2 * s->src_cap);
    FX_CUDA(s, device_alloc((void**)&s->d_sources, (size_t)cap * 32 * sizeof(float)));
    s->src_cap = cap;
  }
  if (dev_count > s->h_src_cap) {
    FX_CUDA(s, cudaEventSynchronize(s->src_event));
    if (s->h_src_stage) FX_CUDA(s, cudaFreeHost(s->h_src_stage));
    s->h_src_stage = nullptr;
    FX_CUDA(s, host_alloc((void**)&s->h_src_stage, (size_t)dev_count * 32 * sizeof(float)));
    s->h_src_cap = dev_count;
  }
  FX_CUDA(s, cudaEventSynchronize(s->src_event));
  if (s->src_count == 0) std::memset(s->h_src_stage, 0, 32 * sizeof(float));
  else std::memcpy(s->h_src_stage, s->host_sources.data(), (size_t)s->src_count * 32 * sizeof(float));
  FX_CUDA(s, cudaMemcpyAsync(s->d_sources, s->h_src_stage, (size_t)dev_count * 32 * sizeof(float), cudaMemcpyHostToDevice, s->stream));
  FX_CUDA(s, cudaEventRecord(s->src_event, s->stream));
  return FX_OK;
}

// Fills the 80-byte uniform exactly as createCombustionVolumeSimulation.ts:237-266
// does: doubles computed on the host, then rounded to f32.
Params make_params(const fx_sim* s, double elapsed, double step_s) {
  const double effective = std::min(step_s, 1.0 / 15.0);
  const double local_time = elapsed - s->start_s;
  const double prev_local = s->last_elapsed_s - s->start_s;
  const double dx = s->rp.world_size / (double)std::max(s->dm.w, s->dm.d);
  Params P;
  P.time = (float)local_time;
  P.dt = (float)effective;
  P.prev_time = (float)prev_local;
  P.scalar_set = (float)s->cur;
  for (int k = 0; k < 3; ++k) P.wind[k] = (float)s->rp.wind[k];
  P.wind[3] = (float)s->rp.wind_strength;
  for (int k = 0; k < 3; ++k) P.gravity[k] = (float)s->rp.gravity[k];
  P.gravity[3] = (float)s->rp.gravity_strength;
  P.buoyancy = (float)s->rp.buoyancy;
  P.vorticity_strength = (float)s->rp.vorticity_strength;
  P.dx = (float)dx;
  P.world_size = (float)s->rp.world_size;
  P.vmask[0] = (float)s->rp.vorticity_constant_mask;
  P.vmask[1] = (float)s->rp.vorticity_velocity_mask;
  P.vmask[2] = (float)s->rp.vorticity_heat_mask;
  P.vmask[3] = (float)s->rp.vorticity_density_mask;
  P.step_index = (uint32_t)s->step_index;
  P.half_round = (s->half && !s->half_nearest) ? 1u : 0u;
  return P;
}

// PressureSolvePass.smooth (:129-143) for the plain path.
int plain_smooth(fx_sim* s, LevelBuf& L, int iters, int start, uint32_t& launches, const char* name) {
  int active = start;
  for (int k = 0; k < iters; ++k) {
    s->timer.begin(s->stream, name);
    plain_jacobi(s->stream, L.dm, L.div, L.p[active], L.p[active ^ 1]);
    s->timer.end(s->stream);
    active ^= 1;
    ++launches;
  }
  return active;
}

#define FX_TIMED(sim, name, call)            \
  do {                                       \
    (sim)->timer.begin((sim)->stream, name); \
    call;                                    \
    (sim)->timer.end((sim)->stream);         \
  } while (0)

// Additions to a plain step used by the differentiable rollout: the inflow
// patch (applied after inject-velocity), and copies of the intermediate fields
// its adjoint reads (a null pointer skips a copy).
VCycleConfig vcycle_config(const fx_sim* s, bool plain) {
  VCycleConfig c{};
  c.levels = s->solver.levels;
  c.pre = s->solver.pre_sweeps;
  c.post = s->solver.post_sweeps;
  c.coarse = s->solver.coarse_sweeps;
  c.max_cycles = s->solver.max_cycles;
  c.omega = (float)s->solver.omega;
  c.omega_one = s->solver.omega == 1.0;
  c.tol = s->solver.tolerance;
  c.warm = s->solver.warm_start != 0;
  c.plain = plain;
  return c;
}

struct PlainHooks {
  const float* inflow = nullptr;
  InflowPatch patch{};
  float* t1 = nullptr;  // temperature after inject-scalar
  float* r1 = nullptr;  // reaction after inject-scalar
  VelField v1{};        // velocity after inject-velocity and the inflow
  VelField a{};         // velocity after advect-velocity
  VelField b{};         // velocity after buoyancy
};

fx_status copy_vel(fx_sim* s, VelField dst, VelField src) {
  if (!dst.c[0]) return FX_OK;
  for (int c = 0; c < 3; ++c)
    FX_CUDA(s, cudaMemcpyAsync(dst.c[c], src.c[c], (size_t)s->n * sizeof(float), cudaMemcpyDeviceToDevice, s->stream));
  return FX_OK;
}

// The plain FP32 step: one kernel per reference dispatch, in the reference order.
fx_status step_plain(fx_sim* s, bool vort_on, bool pressure_on, bool debug_on, const PlainHooks* hk = nullptr) {
  cudaStream_t st = s->stream;
  const int cur = s->cur, next = cur ^ 1;
  const uint32_t nsrc = std::max<uint32_t>(s->src_count, 1);
  uint32_t launches = 0;
  FX_TIMED(s, "plain_inject_scalar", plain_inject_scalar(st, s->dm, s->d_params, s->d_sources, nsrc, s->sets[cur]));
  FX_TIMED(s, "plain_inject_velocity", plain_inject_velocity(st, s->dm, s->d_params, s->d_sources, nsrc, s->vcur));
  if (hk) {
    if (hk->inflow) plain_inflow(st, s->dm, hk->patch, hk->inflow, s->vcur);
    if (hk->t1) FX_CUDA(s, cudaMemcpyAsync(hk->t1, s->sets[cur].f[1], (size_t)s->n * sizeof(float), cudaMemcpyDeviceToDevice, st));
    if (hk->r1) FX_CUDA(s, cudaMemcpyAsync(hk->r1, s->sets[cur].f[3], (size_t)s->n * sizeof(float), cudaMemcpyDeviceToDevice, st));
    if (copy_vel(s, hk->v1, s->vcur) != FX_OK) return FX_ERR_CUDA;
  }
  FX_TIMED(s, "plain_inject_igniter", plain_inject_igniter(st, s->dm, s->d_params, s->d_sources, nsrc, s->sets[cur]));
  FX_CUDA(s, cudaMemsetAsync(s->flags[cur], 0, s->nb * sizeof(uint32_t), st));
  FX_TIMED(s, "plain_active_bricks", plain_active_bricks(st, s->dm, s->bricks, s->sets[cur], s->flags[cur]));
  FX_TIMED(s, "plain_advect_velocity", plain_advect_velocity(st, s->dm, s->d_params, s->vcur, s->vscr));
  if (hk && copy_vel(s, hk->a, s->vscr) != FX_OK) return FX_ERR_CUDA;
  FX_TIMED(s, "plain_advect_scalars", plain_advect_scalars(st, s->dm, s->bricks, s->d_params, s->advect_mode, s->sets[cur], s->vscr, s->flags[cur], s->sets[next]));
  FX_CUDA(s, cudaMemsetAsync(s->flags[next], 0, s->nb * sizeof(uint32_t), st));
  FX_TIMED(s, "plain_active_bricks", plain_active_bricks(st, s->dm, s->bricks, s->sets[next], s->flags[next]));
  launches += 7;
  // Combustion reads a snapshot of the set so that every neighbour read sees the
  // state before the pass (see the note at plain k_combustion).
  for (int f = 0; f < 4; ++f)
    FX_CUDA(s, cudaMemcpyAsync(s->sets[2].f[f], s->sets[next].f[f], (size_t)s->n * sizeof(float), cudaMemcpyDeviceToDevice, st));
  FX_TIMED(s, "plain_combustion", plain_combustion(st, s->dm, s->bricks, s->d_params, s->sets[2], s->flags[next], s->sets[next]));
  FX_TIMED(s, "plain_buoyancy", plain_buoyancy(st, s->dm, s->bricks, s->d_params, s->sets[next], s->flags[next], s->vscr));
  launches += 2;
  if (hk && copy_vel(s, hk->b, s->vscr) != FX_OK) return FX_ERR_CUDA;
  if (vort_on) {
    FX_TIMED(s, "plain_vorticity", plain_vorticity(st, s->dm, s->vscr, s->vort, s->vort_mag));
    FX_TIMED(s, "plain_confinement", plain_confinement(st, s->dm, s->d_params, s->vort, s->vort_mag, s->sets[next], s->vscr, s->conf_mag));
    launches += 2;
  }
  const bool vcycle = pressure_on && s->solver.mode == FX_SOLVER_VCYCLE;
  if (vcycle) {
    // The V-cycle extension with its one-voxel kernels, from the previous
    // step's pressure; the host reads the continue flag after every cycle.
    FX_TIMED(s, "plain_divergence", plain_divergence(st, s->dm, s->vscr, s->lv[0].div));
    ++launches;
    VCycleLevels L;
    for (int k = 0; k < 3; ++k) {
      L.lv[k] = s->lv[k];
      L.lv[3 + k] = s->xlv[k];
    }
    const VCycleConfig c = vcycle_config(s, true);
    const int start = s->last_p;
    FX_CUDA(s, vcycle_prologue(st, L, c, start, s->fw.solver, 0));
    launches += 3;
    for (int k = 0; k < c.max_cycles; ++k) {
      FX_CUDA(s, cudaMemcpyAsync(s->fw.host_cont, &s->fw.solver->cont, sizeof(int), cudaMemcpyDeviceToHost, st));
      FX_CUDA(s, cudaStreamSynchronize(st));
      if (!*s->fw.host_cont) break;
      uint32_t body = 0;
      s->timer.begin(st, "plain_vcycle");
      FX_CUDA(s, vcycle_body(st, L, c, start, s->fw.solver, 0, &body));
      s->timer.end(st);
      launches += body;
    }
  } else if (pressure_on) {
    for (auto& L : s->lv) FX_CUDA(s, cudaMemsetAsync(L.p[0], 0, count_of(L.dm) * sizeof(float), st));
    FX_TIMED(s, "plain_divergence", plain_divergence(st, s->dm, s->vscr, s->lv[0].div));
    ++launches;
    const int* q = s->qi;
    const int fine_pre = plain_smooth(s, s->lv[0], q[2], 0, launches, "plain_jacobi_fine");
    FX_TIMED(s, "plain_restrict", plain_restrict(st, s->lv[0].dm, s->lv[1].dm, s->lv[0].div, s->lv[1].div));
    const int mid_pre = plain_smooth(s, s->lv[1], q[4], 0, launches, "plain_jacobi_mid");
    FX_TIMED(s, "plain_restrict", plain_restrict(st, s->lv[1].dm, s->lv[2].dm, s->lv[1].div, s->lv[2].div));
    const int coarse = plain_smooth(s, s->lv[2], q[6], 0, launches, "plain_jacobi_coarse");
    FX_TIMED(s, "plain_prolong", plain_prolong(st, s->lv[2].dm, s->lv[1].dm, s->lv[2].p[coarse], s->lv[1].p[0]));
    const int mid = plain_smooth(s, s->lv[1], q[5], mid_pre, launches, "plain_jacobi_mid");
    FX_TIMED(s, "plain_prolong", plain_prolong(st, s->lv[1].dm, s->lv[0].dm, s->lv[1].p[mid], s->lv[0].p[0]));
    s->last_p = plain_smooth(s, s->lv[0], q[3], fine_pre, launches, "plain_jacobi_fine");
    launches += 4;
  }
  FX_TIMED(s, "plain_project", plain_project(st, s->dm, s->vscr, s->lv[0].p[s->last_p], s->vcur));
  ++launches;
  if (vcycle) {
    FX_CUDA(s, max_divergence(st, s->dm, s->vcur, s->fw.solver));
    ++launches;
  }
  if (debug_on) {
    FX_TIMED(s, "plain_velocity_magnitude", plain_velocity_magnitude(st, s->dm, s->vcur, s->vel_mag));
    ++launches;
  }
  s->final_vscr = &s->vscr;
  s->last_kernel_count = launches;
  FX_CUDA(s, cudaGetLastError());
  return FX_OK;
}

bool is_scalar_field(int id) { return id >= FX_FIELD_DENSITY && id <= FX_FIELD_PREV_REACTION; }

// Pointer of a field for read/write, with its element count.
bool field_ref(fx_sim* s, int id, void** ptr, size_t* count) {
  const int prev = s->cur ^ 1;
  *count = s->n;
  switch (id) {
    case FX_FIELD_DENSITY: case FX_FIELD_TEMPERATURE: case FX_FIELD_FUEL: case FX_FIELD_REACTION:
      *ptr = s->sets[s->cur].f[id - FX_FIELD_DENSITY]; return true;
    case FX_FIELD_PREV_DENSITY: case FX_FIELD_PREV_TEMPERATURE: case FX_FIELD_PREV_FUEL: case FX_FIELD_PREV_REACTION:
      *ptr = s->sets[prev].f[id - FX_FIELD_PREV_DENSITY]; return true;
    case FX_FIELD_VELOCITY_X: case FX_FIELD_VELOCITY_Y: case FX_FIELD_VELOCITY_Z:
      *ptr = s->vcur.c[id - FX_FIELD_VELOCITY_X]; return true;
    case FX_FIELD_VELOCITY_SCRATCH_X: case FX_FIELD_VELOCITY_SCRATCH_Y: case FX_FIELD_VELOCITY_SCRATCH_Z:
      *ptr = s->final_vscr->c[id - FX_FIELD_VELOCITY_SCRATCH_X]; return true;
    case FX_FIELD_VORTICITY_X: case FX_FIELD_VORTICITY_Y: case FX_FIELD_VORTICITY_Z:
      *ptr = s->vort.c[id - FX_FIELD_VORTICITY_X]; return true;
    case FX_FIELD_VORTICITY_MAGNITUDE: *ptr = s->vort_mag; return true;
    case FX_FIELD_CONFINEMENT_MAGNITUDE: *ptr = s->conf_mag; return true;
    case FX_FIELD_VELOCITY_MAGNITUDE: *ptr = s->vel_mag; return true;
    case FX_FIELD_BRICK_FLAGS: *ptr = s->flags[s->cur]; *count = s->nb; return true;
    case FX_FIELD_PREV_BRICK_FLAGS: *ptr = s->flags[prev]; *count = s->nb; return true;
    case FX_FIELD_FINE_DIVERGENCE: case FX_FIELD_FINE_PRESSURE_A: case FX_FIELD_FINE_PRESSURE_B:
    case FX_FIELD_MID_DIVERGENCE: case FX_FIELD_MID_PRESSURE_A: case FX_FIELD_MID_PRESSURE_B:
    case FX_FIELD_COARSE_DIVERGENCE: case FX_FIELD_COARSE_PRESSURE_A: case FX_FIELD_COARSE_PRESSURE_B: {
      const int l = (id - FX_FIELD_FINE_DIVERGENCE) / 3, k = (id - FX_FIELD_FINE_DIVERGENCE) % 3;
      *count = count_of(s->lv[l].dm);
      *ptr = k == 0 ? s->lv[l].div : s->lv[l].p[k - 1];
      return true;
    }
    case FX_FIELD_PRESSURE: *ptr = s->lv[0].p[s->last_p]; return true;
    default: return false;
  }
}

// The host side of a step around its device work, shared by fx_sim_step and the
// batch step: step_begin latches the parameters (createCombustionVolumeSimulation.ts:
// 236-266) into the device uniform and describes the fused step; step_finish
// records the result and advances the host state (:293-305).
struct StepPlan {
  bool vort_on = false, pressure_on = false, debug_on = false;
  FusedStep fs{};
};

fx_status step_begin(fx_sim* s, double elapsed, double step_s, StepPlan& sp) {
  if (!s->initialized) {
    s->initialized = true;
    s->start_s = elapsed;
    s->last_elapsed_s = elapsed;
  }
  const Params P = make_params(s, elapsed, step_s);
  const int slot = (int)(s->param_counter % kParamSlots);
  FX_CUDA(s, cudaEventSynchronize(s->param_events[slot]));
  s->h_params[slot] = P;
  FX_CUDA(s, cudaMemcpyAsync(s->d_params, &s->h_params[slot], sizeof(Params), cudaMemcpyHostToDevice, s->stream));
  FX_CUDA(s, cudaEventRecord(s->param_events[slot], s->stream));
  ++s->param_counter;

  sp.vort_on = s->step_index % s->qi[1] == 0;
  sp.pressure_on = s->step_index % s->qi[0] == 0;
  sp.debug_on = s->n < 1800000u || s->debug_requested;
  if (s->kernels != FX_KERNELS_FUSED) return FX_OK;
  FusedStep& fs = sp.fs;
  fs.stream = s->stream;
  fs.dm = s->dm;
  fs.bricks = s->bricks;
  fs.params = s->d_params;
  fs.host_params = P;
  fs.sources = s->d_sources;
  fs.nsrc = std::max<uint32_t>(s->src_count, 1);
  fs.host_sources = s->src_count ? s->host_sources.data() : nullptr;
  fs.host_nsrc = s->src_count;
  fs.advect_mode = s->advect_mode;
  fs.cur_index = s->cur;
  fs.cur = s->sets[s->cur];
  fs.next = s->sets[s->cur ^ 1];
  fs.scratch = s->sets[2];
  fs.half_storage = s->half;
  fs.flags_cur = s->flags[s->cur];
  fs.flags_next = s->flags[s->cur ^ 1];
  fs.vcur = s->vcur;
  fs.vscr = s->vscr;
  fs.vscr2 = s->vscr2;
  fs.vort = s->vort;
  fs.vort_mag = s->vort_mag;
  fs.conf_mag = s->conf_mag;
  fs.vel_mag = s->vel_mag;
  for (int l = 0; l < 3; ++l) fs.lv[l] = s->lv[l];
  for (int l = 0; l < 3; ++l) fs.xlv[l] = s->xlv[l];
  for (int k = 0; k < 7; ++k) fs.q[k] = s->qi[k];
  for (int l = 0; l < 3; ++l) fs.sweep_variant[l] = s->sweep_variant[l];
  for (int k = 0; k < kBrickKernels; ++k) fs.brick_ctas[k] = s->brick_ctas[k];
  fs.solver_mode = s->solver.mode;
  fs.vc = vcycle_config(s, false);
  fs.solver_norms = (s->instr & FX_INSTR_SOLVER_NORMS) != 0;
  fs.vort_on = sp.vort_on;
  fs.pressure_on = sp.pressure_on;
  fs.debug_on = sp.debug_on;
  fs.debug_fields = (s->opt_flags & FX_OPT_DEBUG_FIELDS) != 0;
  fs.sparse = s->sparse;
  fs.last_p = s->last_p;
  return FX_OK;
}

fx_status step_finish(fx_sim* s, fx_status st, const FusedResult* fr, const StepPlan& sp, double elapsed) {
  if (st != FX_OK) return st;
  if (fr) {
    s->last_p = fr->last_p;
    s->final_vscr = fr->final_vscr_is_2 ? &s->vscr2 : &s->vscr;
    s->last_kernel_count = fr->launches;
    s->last_step_graph = fr->graph;
    s->last_cycle_launches = sp.pressure_on && s->solver.mode == FX_SOLVER_VCYCLE ? fr->cycle_launches : 0;
    s->last_solver_mode = s->solver.mode;
  }
  if (s->instr & FX_INSTR_COUNT_ACTIVE) {
    // flags of the step's advected set: the render flags once the step is done
    FX_CUDA(s, fused_accumulate_active(s->stream, s->dm, s->bricks, s->flags[s->cur ^ 1], s->d_active_acc));
    s->last_kernel_count += 1;
  }
  if (sp.debug_on) s->debug_requested = false;
  s->cur ^= 1;
  s->last_elapsed_s = elapsed;
  s->step_index += 1;
  return FX_OK;
}

}  // namespace

namespace fx {
// The calling thread's fx_last_error message, for entry points outside this file.
void set_last_error(const std::string& msg) { g_last_error = msg; }

// The state a render reads: the current scalar set and brick flags (what
// getRenderBuffers returns), on the simulation's stream.
struct SimView {
  Dims dm;
  uint3 bricks;
  const void* f[4];
  const uint32_t* flags;
  bool half;
  cudaStream_t stream;
  int device;
};

bool sim_view(fx_sim* s, SimView* out) {
  if (!s || !s->err.empty()) return false;
  out->dm = s->dm;
  out->bricks = s->bricks;
  for (int k = 0; k < 4; ++k) out->f[k] = s->sets[s->cur].f[k];
  out->flags = s->flags[s->cur];
  out->half = s->half;
  out->stream = s->stream;
  out->device = s->device;
  return true;
}
}  // namespace fx

extern "C" {

int32_t fx_abi_version(void) { return FX_ABI_VERSION; }

const char* fx_last_error(void) { return g_last_error.c_str(); }

void fx_sim_options_default(fx_sim_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->struct_size = sizeof *o;
  o->width = 128;
  o->height = 256;
  o->depth = 128;
  o->scalar_advection_mode = FX_ADVECT_MACCORMACK;
  o->runtime_mask = 0;
  o->runtime.gravity[1] = -1.0;
  o->runtime.gravity_strength = 0.45;
  o->runtime.buoyancy = 3.6;
  o->runtime.vorticity_strength = 2.15;
  o->runtime.vorticity_constant_mask = 1.0;
  o->runtime.vorticity_velocity_mask = 0.4;
  o->runtime.vorticity_heat_mask = 0.8;
  o->runtime.vorticity_density_mask = 0.35;
  o->runtime.world_size = 10.0;
  o->quality_mask = 0;
  o->quality.pressure_interval = 1;
  o->quality.vorticity_interval = 1;
  o->quality.fine_pre_iterations = 2;
  o->quality.fine_post_iterations = 3;
  o->quality.mid_pre_iterations = 2;
  o->quality.mid_post_iterations = 3;
  o->quality.coarse_iterations = 10;
  o->device = 0;
  o->kernels = FX_KERNELS_FUSED;
  o->flags = 0;
  o->stream = nullptr;
}

fx_status fx_sim_create(const fx_sim_options* opt_in, fx_sim** out) {
  g_last_error.clear();
  if (!out) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_create: out is NULL");
  *out = nullptr;
  fx_sim_options opt;
  fx_sim_options_default(&opt);
  if (opt_in) {
    if (opt_in->struct_size != sizeof(fx_sim_options))
      return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_create: struct_size does not match this library's fx_sim_options");
    opt = *opt_in;
  }
  uint32_t w = opt.width ? opt.width : 128, h = opt.height ? opt.height : 256, d = opt.depth ? opt.depth : 128;
  if (w < 2 || h < 2 || d < 2) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_create: every dimension must be >= 2");
  if ((double)w * h * d >= 4294967296.0) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_create: grid must hold fewer than 2^32 voxels");
  if (opt.scalar_advection_mode != FX_ADVECT_SEMI_LAGRANGIAN && opt.scalar_advection_mode != FX_ADVECT_MACCORMACK)
    return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_create: unknown scalar_advection_mode");
  if (opt.kernels != FX_KERNELS_FUSED && opt.kernels != FX_KERNELS_PLAIN)
    return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_create: unknown kernels path");
  if ((opt.flags & FX_OPT_SCALARS_F16) && opt.kernels != FX_KERNELS_FUSED)
    return fail(nullptr, FX_ERR_UNSUPPORTED, "fx_sim_create: FP16 scalar storage needs the fused kernels");
  if ((opt.flags & FX_OPT_SPARSE) && opt.kernels != FX_KERNELS_FUSED)
    return fail(nullptr, FX_ERR_UNSUPPORTED, "fx_sim_create: sparse mode needs the fused kernels");
  if ((opt.flags & FX_OPT_SPARSE) && (opt.width > 8192u || opt.height > 8192u || opt.depth > 8192u))
    return fail(nullptr, FX_ERR_UNSUPPORTED, "fx_sim_create: sparse mode supports at most 8192 voxels (1024 bricks) per axis");

  fx_sim* s = new (std::nothrow) fx_sim;
  if (!s) return fail(nullptr, FX_ERR_OUT_OF_MEMORY, "fx_sim_create: host allocation failed");
  auto bail = [&](fx_status code) {
    g_last_error = s->err;
    fx_sim_destroy(s);
    return code;
  };
  s->device = opt.device;
  s->kernels = opt.kernels;
  s->opt_flags = opt.flags;
  s->half = (opt.flags & FX_OPT_SCALARS_F16) != 0;
  s->sparse = (opt.flags & FX_OPT_SPARSE) != 0;
  s->half_nearest = (opt.flags & FX_OPT_F16_ROUND_NEAREST) != 0;
  s->dm = Dims{w, h, d};
  s->n = w * h * d;
  s->bricks = make_uint3((w + 7) / 8, (h + 7) / 8, (d + 7) / 8);
  s->nb = s->bricks.x * s->bricks.y * s->bricks.z;
  s->advect_mode = opt.scalar_advection_mode;
  fx_sim_options defaults;
  fx_sim_options_default(&defaults);
  s->rp = defaults.runtime;
  merge_params(s->rp, opt.runtime, opt.runtime_mask);
  s->quality = defaults.quality;
  if (!merge_quality(s->quality, opt.quality, opt.quality_mask)) {
    s->err = "fx_sim_create: NaN quality setting";
    return bail(FX_ERR_INVALID_ARGUMENT);
  }
  apply_quality_clamps(s);

  fx_status st;
  if (cudaSetDevice(s->device) != cudaSuccess) {
    s->err = "fx_sim_create: cudaSetDevice failed (no CUDA device?)";
    return bail(FX_ERR_CUDA);
  }
  if (opt.stream) {
    s->stream = (cudaStream_t)opt.stream;
  } else {
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) {
      s->err = "fx_sim_create: cudaStreamCreate failed";
      return bail(FX_ERR_CUDA);
    }
    s->own_stream = true;
  }
  s->lv[0].dm = s->dm;
  s->lv[1].dm = halve(s->lv[0].dm);
  s->lv[2].dm = halve(s->lv[1].dm);
  s->xlv[0].dm = halve(s->lv[2].dm);
  s->xlv[1].dm = halve(s->xlv[0].dm);
  s->xlv[2].dm = halve(s->xlv[1].dm);
  fx_solver_settings_default(&s->solver);

  // One arena; every buffer starts on a 256-byte boundary.
  const size_t n = s->n;
  size_t off = 0;
  auto carve = [&](size_t bytes) {
    const size_t o = off;
    off += (bytes + 255) & ~(size_t)255;
    return o;
  };
  size_t o_sets[3][4], o_vcur[3], o_vscr[3], o_vscr2[3], o_vort[3], o_wmag, o_fmag, o_vmag, o_flags[2], o_lv[3][3], o_xlv[3][3], o_params;
  for (auto& set : o_sets)
    for (auto& f : set) f = carve(n * (s->half ? 2 : 4));
  for (int c = 0; c < 3; ++c) {
    o_vcur[c] = carve(n * 4);
    o_vscr[c] = carve(n * 4);
    o_vscr2[c] = carve(n * 4);
    o_vort[c] = carve(n * 4);
  }
  o_wmag = carve(n * 4);
  o_fmag = carve(n * 4);
  o_vmag = carve(n * 4);
  o_flags[0] = carve((size_t)s->nb * 4);
  o_flags[1] = carve((size_t)s->nb * 4);
  for (int l = 0; l < 3; ++l)
    for (int k = 0; k < 3; ++k) o_lv[l][k] = carve(count_of(s->lv[l].dm) * 4);
  for (int l = 0; l < 3; ++l)
    for (int k = 0; k < 3; ++k) o_xlv[l][k] = carve(count_of(s->xlv[l].dm) * 4);
  o_params = carve(sizeof(Params));
  const size_t o_acc = carve(2 * sizeof(unsigned long long));
  const size_t o_fused = off;
  off += fused_work_bytes(s->dm, s->bricks, s->half ? 8 : 16);
  s->arena_bytes = off;
  {
    cudaError_t e = device_alloc(&s->arena, s->arena_bytes);
    if (e != cudaSuccess) {
      s->err = std::string("fx_sim_create: cudaMalloc of the field arena failed: ") + cudaGetErrorString(e);
      return bail(e == cudaErrorMemoryAllocation ? FX_ERR_OUT_OF_MEMORY : FX_ERR_CUDA);
    }
  }
  char* base = (char*)s->arena;
  for (int k = 0; k < 3; ++k)
    for (int f = 0; f < 4; ++f) s->sets[k].f[f] = (float*)(base + o_sets[k][f]);
  for (int c = 0; c < 3; ++c) {
    s->vcur.c[c] = (float*)(base + o_vcur[c]);
    s->vscr.c[c] = (float*)(base + o_vscr[c]);
    s->vscr2.c[c] = (float*)(base + o_vscr2[c]);
    s->vort.c[c] = (float*)(base + o_vort[c]);
  }
  s->vort_mag = (float*)(base + o_wmag);
  s->conf_mag = (float*)(base + o_fmag);
  s->vel_mag = (float*)(base + o_vmag);
  s->flags[0] = (uint32_t*)(base + o_flags[0]);
  s->flags[1] = (uint32_t*)(base + o_flags[1]);
  for (int l = 0; l < 3; ++l) {
    s->lv[l].div = (float*)(base + o_lv[l][0]);
    s->lv[l].p[0] = (float*)(base + o_lv[l][1]);
    s->lv[l].p[1] = (float*)(base + o_lv[l][2]);
    s->xlv[l].div = (float*)(base + o_xlv[l][0]);
    s->xlv[l].p[0] = (float*)(base + o_xlv[l][1]);
    s->xlv[l].p[1] = (float*)(base + o_xlv[l][2]);
  }
  s->d_params = (Params*)(base + o_params);
  s->d_active_acc = (unsigned long long*)(base + o_acc);
  fused_work_carve(s->fw, base + o_fused, s->dm, s->bricks, s->half ? 8 : 16);
  s->fw.use_graphs = (s->opt_flags & FX_OPT_NO_GRAPHS) == 0;
  s->final_vscr = &s->vscr;

  if (host_alloc((void**)&s->h_params, kParamSlots * sizeof(Params)) != cudaSuccess) {
    s->err = "fx_sim_create: cudaMallocHost failed";
    return bail(FX_ERR_OUT_OF_MEMORY);
  }
  for (auto& ev : s->param_events)
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
      s->err = "fx_sim_create: cudaEventCreate failed";
      return bail(FX_ERR_CUDA);
    }
  if (cudaEventCreateWithFlags(&s->src_event, cudaEventDisableTiming) != cudaSuccess) {
    s->err = "fx_sim_create: cudaEventCreate failed";
    return bail(FX_ERR_CUDA);
  }
  if ((st = zero_state(s)) != FX_OK) return bail(st);
  if ((st = upload_sources(s)) != FX_OK) return bail(st);
  if ((st = fused_init(s->fw, s->stream)) != FX_OK) {
    s->err = "fx_sim_create: fused path initialisation failed";
    return bail(st);
  }
  if (cudaStreamSynchronize(s->stream) != cudaSuccess) {
    s->err = "fx_sim_create: initial clear failed";
    return bail(FX_ERR_CUDA);
  }
  *out = s;
  return FX_OK;
}

void fx_sim_destroy(fx_sim* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  fused_release(s->fw);
  s->timer.release();
  if (s->arena) cudaFree(s->arena);
  if (s->d_sources) cudaFree(s->d_sources);
  if (s->h_src_stage) cudaFreeHost(s->h_src_stage);
  if (s->h_params) cudaFreeHost(s->h_params);
  for (auto& ev : s->param_events)
    if (ev) cudaEventDestroy(ev);
  if (s->src_event) cudaEventDestroy(s->src_event);
  if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

fx_status fx_sim_step(fx_sim* s, double elapsed, double step_s) {
  if (!s) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_step: NULL handle");
  if (!s->err.empty()) return FX_ERR_STATE;
  FX_CUDA(s, cudaSetDevice(s->device));
  StepPlan sp;
  fx_status st = step_begin(s, elapsed, step_s, sp);
  if (st != FX_OK) return st;
  if (s->kernels == FX_KERNELS_PLAIN) return step_finish(s, step_plain(s, sp.vort_on, sp.pressure_on, sp.debug_on), nullptr, sp, elapsed);
  FusedResult fr;
  st = fused_step(s->fw, sp.fs, fr);
  if (st != FX_OK) fail(s, st, "fx_sim_step: fused step failed: " + fr.error);
  return step_finish(s, st, &fr, sp, elapsed);
}

fx_status fx_sim_get_render_buffers(fx_sim* s, fx_render_buffers* o) {
  if (!s || !o) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_get_render_buffers: NULL argument");
  std::memset(o, 0, sizeof *o);
  const ScalarSet& set = s->sets[s->cur];
  o->density = (uint64_t)(uintptr_t)set.f[0];
  o->temperature = (uint64_t)(uintptr_t)set.f[1];
  o->fuel = (uint64_t)(uintptr_t)set.f[2];
  o->reaction = (uint64_t)(uintptr_t)set.f[3];
  o->active_brick_flags = (uint64_t)(uintptr_t)s->flags[s->cur];
  o->active_brick_info[0] = s->bricks.x;
  o->active_brick_info[1] = s->bricks.y;
  o->active_brick_info[2] = s->bricks.z;
  o->active_brick_info[3] = s->nb;
  o->active_brick_info[4] = 8;
  o->width = s->dm.w;
  o->height = s->dm.h;
  o->depth = s->dm.d;
  o->dtype = s->half ? FX_DTYPE_F16 : FX_DTYPE_F32;
  return FX_OK;
}

fx_status fx_sim_get_debug_buffers(fx_sim* s, fx_debug_buffers* o) {
  if (!s || !o) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_get_debug_buffers: NULL argument");
  fx_status st = fx_sim_get_render_buffers(s, &o->render);
  if (st != FX_OK) return st;
  s->debug_requested = true;
  o->velocity_magnitude = (uint64_t)(uintptr_t)s->vel_mag;
  o->divergence = (uint64_t)(uintptr_t)s->lv[0].div;
  o->pressure = (uint64_t)(uintptr_t)s->lv[0].p[s->last_p];
  o->vorticity_magnitude = (uint64_t)(uintptr_t)s->vort_mag;
  o->confinement_force_magnitude = (uint64_t)(uintptr_t)s->conf_mag;
  return FX_OK;
}

fx_status fx_sim_get_scalar_advection_mode(fx_sim* s, int32_t* mode) {
  if (!s || !mode) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_get_scalar_advection_mode: NULL argument");
  *mode = s->advect_mode;
  return FX_OK;
}

fx_status fx_sim_set_scalar_advection_mode(fx_sim* s, int32_t mode) {
  if (!s) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_set_scalar_advection_mode: NULL handle");
  if (mode != FX_ADVECT_SEMI_LAGRANGIAN && mode != FX_ADVECT_MACCORMACK)
    return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_set_scalar_advection_mode: unknown mode");
  s->advect_mode = mode;
  return FX_OK;
}

fx_status fx_sim_get_runtime_params(fx_sim* s, fx_runtime_params* o) {
  if (!s || !o) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_get_runtime_params: NULL argument");
  *o = s->rp;
  return FX_OK;
}

fx_status fx_sim_set_runtime_params(fx_sim* s, const fx_runtime_params* p, uint32_t mask) {
  if (!s || (!p && mask)) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_set_runtime_params: NULL argument");
  if (mask & ~FX_PARAM_ALL) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_set_runtime_params: unknown mask bits");
  if (p) merge_params(s->rp, *p, mask);
  return FX_OK;
}

fx_status fx_sim_get_quality(fx_sim* s, fx_quality* o) {
  if (!s || !o) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_get_quality: NULL argument");
  *o = s->quality;
  return FX_OK;
}

fx_status fx_sim_set_quality(fx_sim* s, const fx_quality* q, uint32_t mask) {
  if (!s || (!q && mask)) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_set_quality: NULL argument");
  if (mask & ~FX_QUALITY_ALL) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_set_quality: unknown mask bits");
  fx_quality merged = s->quality;
  if (q && !merge_quality(merged, *q, mask)) return FX_ERR_INVALID_ARGUMENT;
  s->quality = merged;
  apply_quality_clamps(s);
  return FX_OK;
}

fx_status fx_sim_update_sources(fx_sim* s, const float* packed, uint32_t count) {
  if (!s || (count && !packed)) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_update_sources: NULL argument");
  if (!s->err.empty()) return FX_ERR_STATE;
  FX_CUDA(s, cudaSetDevice(s->device));
  s->host_sources.assign(packed, packed + (size_t)count * 32);
  s->src_count = count;
  return upload_sources(s);
}

fx_status fx_sim_reset(fx_sim* s) {
  if (!s) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_reset: NULL handle");
  if (!s->err.empty()) return FX_ERR_STATE;
  FX_CUDA(s, cudaSetDevice(s->device));
  // doReset(lastElapsedSeconds), createCombustionVolumeSimulation.ts:206-226,381-383
  s->cur = 0;
  s->step_index = 0;
  s->last_p = 0;
  s->initialized = false;
  s->start_s = s->last_elapsed_s;
  fx_status st = zero_state(s);
  if (st != FX_OK) return st;
  return fused_reset(s->fw, s->stream);
}

fx_status fx_sim_get_resolution(fx_sim* s, uint32_t* w, uint32_t* h, uint32_t* d) {
  if (!s || !w || !h || !d) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_get_resolution: NULL argument");
  *w = s->dm.w;
  *h = s->dm.h;
  *d = s->dm.d;
  return FX_OK;
}

fx_status fx_sim_field_size(fx_sim* s, int32_t id, size_t* bytes) {
  if (!s || !bytes) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_field_size: NULL argument");
  void* p;
  size_t count;
  if (!field_ref(s, id, &p, &count)) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_field_size: unknown field id");
  *bytes = count * 4;
  return FX_OK;
}

fx_status fx_sim_read_field(fx_sim* s, int32_t id, void* dst, size_t bytes) {
  if (!s || !dst) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_read_field: NULL argument");
  void* p;
  size_t count;
  if (!field_ref(s, id, &p, &count)) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_read_field: unknown field id");
  if (bytes != count * 4) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_read_field: byte count does not match the field");
  FX_CUDA(s, cudaSetDevice(s->device));
  FX_CUDA(s, cudaStreamSynchronize(s->stream));
  if (s->half && is_scalar_field(id)) {
    // binary16 on the device, f32 at the ABI (exact widening)
    std::vector<__half> tmp(count);
    FX_CUDA(s, cudaMemcpy(tmp.data(), p, count * sizeof(__half), cudaMemcpyDeviceToHost));
    float* out = static_cast<float*>(dst);
    for (size_t i = 0; i < count; ++i) out[i] = __half2float(tmp[i]);
    return FX_OK;
  }
  FX_CUDA(s, cudaMemcpy(dst, p, bytes, cudaMemcpyDeviceToHost));
  return FX_OK;
}

fx_status fx_sim_write_field(fx_sim* s, int32_t id, const void* src, size_t bytes) {
  if (!s || !src) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_write_field: NULL argument");
  void* p;
  size_t count;
  if (!field_ref(s, id, &p, &count)) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_write_field: unknown field id");
  if (bytes != count * 4) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_write_field: byte count does not match the field");
  FX_CUDA(s, cudaSetDevice(s->device));
  FX_CUDA(s, cudaStreamSynchronize(s->stream));
  if (s->half && is_scalar_field(id)) {
    // f32 at the ABI, rounded to the nearest binary16 (ties to even) on the device
    std::vector<__half> tmp(count);
    const float* in = static_cast<const float*>(src);
    for (size_t i = 0; i < count; ++i) tmp[i] = __float2half_rn(in[i]);
    FX_CUDA(s, cudaMemcpy(p, tmp.data(), count * sizeof(__half), cudaMemcpyHostToDevice));
  } else {
    FX_CUDA(s, cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice));
  }
  // A scratch velocity written here is what the next read returns.
  return fused_invalidate(s->fw, s->stream);
}

namespace {

// The saved state's layout: this header, then the current scalar set as stored
// (4 fields of n elements of scalar_bytes each), the velocity (3 f32 fields),
// the fine pressure of the latest solve (n f32) and the brick flags of the
// current and the other set (2 x nb u32), each part starting on 16 bytes.
struct StateHeader {
  uint32_t magic;
  uint32_t version;
  uint32_t w, h, d;
  uint32_t scalar_bytes;
  int32_t cur, last_p;
  int64_t step_index;
  double start_s, last_elapsed_s;
  uint32_t initialized, reserved;
};
constexpr uint32_t kStateMagic = 0x54535846u;  // "FXST"
constexpr uint32_t kStateVersion = 1;

size_t align16(size_t b) { return (b + 15) & ~size_t(15); }

struct StateLayout {
  size_t scalar, vel, pressure, flags, total;
};

StateLayout state_layout(const fx_sim* s) {
  StateLayout L;
  const size_t es = s->half ? sizeof(__half) : sizeof(float);
  L.scalar = align16(sizeof(StateHeader));
  L.vel = L.scalar + 4 * align16(s->n * es);
  L.pressure = L.vel + 3 * align16(s->n * sizeof(float));
  L.flags = L.pressure + align16(s->n * sizeof(float));
  L.total = L.flags + 2 * align16(s->nb * sizeof(uint32_t));
  return L;
}

}  // namespace

fx_status fx_sim_state_bytes(fx_sim* s, uint64_t* bytes) {
  if (!s || !bytes) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_state_bytes: NULL argument");
  *bytes = state_layout(s).total;
  return FX_OK;
}

fx_status fx_sim_save_state(fx_sim* s, void* dst, uint64_t bytes) {
  if (!s || !dst) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_save_state: NULL argument");
  if (!s->err.empty()) return FX_ERR_STATE;
  const StateLayout L = state_layout(s);
  if (bytes != L.total) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_save_state: byte count does not match fx_sim_state_bytes");
  FX_CUDA(s, cudaSetDevice(s->device));
  StateHeader h{};
  h.magic = kStateMagic;
  h.version = kStateVersion;
  h.w = s->dm.w, h.h = s->dm.h, h.d = s->dm.d;
  h.scalar_bytes = s->half ? 2 : 4;
  h.cur = s->cur, h.last_p = s->last_p;
  h.step_index = s->step_index;
  h.start_s = s->start_s, h.last_elapsed_s = s->last_elapsed_s;
  h.initialized = s->initialized ? 1u : 0u;
  char* o = static_cast<char*>(dst);
  const size_t sb = s->n * (size_t)h.scalar_bytes, fb = s->n * sizeof(float), gb = s->nb * sizeof(uint32_t);
  FX_CUDA(s, cudaStreamSynchronize(s->stream));
  FX_CUDA(s, cudaMemcpy(o, &h, sizeof h, cudaMemcpyDefault));
  for (int k = 0; k < 4; ++k)
    FX_CUDA(s, cudaMemcpyAsync(o + L.scalar + k * align16(sb), s->sets[s->cur].f[k], sb, cudaMemcpyDefault, s->stream));
  for (int k = 0; k < 3; ++k)
    FX_CUDA(s, cudaMemcpyAsync(o + L.vel + k * align16(fb), s->vcur.c[k], fb, cudaMemcpyDefault, s->stream));
  FX_CUDA(s, cudaMemcpyAsync(o + L.pressure, s->lv[0].p[s->last_p], fb, cudaMemcpyDefault, s->stream));
  for (int k = 0; k < 2; ++k)
    FX_CUDA(s, cudaMemcpyAsync(o + L.flags + k * align16(gb), s->flags[s->cur ^ k], gb, cudaMemcpyDefault, s->stream));
  FX_CUDA(s, cudaStreamSynchronize(s->stream));
  return FX_OK;
}

fx_status fx_sim_load_state(fx_sim* s, const void* src, uint64_t bytes) {
  if (!s || !src) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_load_state: NULL argument");
  if (!s->err.empty()) return FX_ERR_STATE;
  const StateLayout L = state_layout(s);
  if (bytes != L.total) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_load_state: byte count does not match fx_sim_state_bytes");
  FX_CUDA(s, cudaSetDevice(s->device));
  StateHeader h{};
  FX_CUDA(s, cudaMemcpy(&h, src, sizeof h, cudaMemcpyDefault));
  if (h.magic != kStateMagic || h.version != kStateVersion)
    return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_load_state: not a saved state of this version");
  if (h.w != s->dm.w || h.h != s->dm.h || h.d != s->dm.d || h.scalar_bytes != (s->half ? 2u : 4u))
    return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_load_state: the state has another resolution or scalar storage");
  if ((h.cur != 0 && h.cur != 1) || (h.last_p != 0 && h.last_p != 1) || h.step_index < 0)
    return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_load_state: corrupt header");
  // doReset's clears (a superset), then the saved parts
  fx_status st = zero_state(s);
  if (st != FX_OK) return st;
  if ((st = fused_reset(s->fw, s->stream)) != FX_OK) return st;
  s->cur = h.cur;
  s->last_p = h.last_p;
  s->step_index = h.step_index;
  s->start_s = h.start_s;
  s->last_elapsed_s = h.last_elapsed_s;
  s->initialized = h.initialized != 0;
  const char* in = static_cast<const char*>(src);
  const size_t sb = s->n * (size_t)h.scalar_bytes, fb = s->n * sizeof(float), gb = s->nb * sizeof(uint32_t);
  for (int k = 0; k < 4; ++k)
    FX_CUDA(s, cudaMemcpyAsync(s->sets[s->cur].f[k], in + L.scalar + k * align16(sb), sb, cudaMemcpyDefault, s->stream));
  for (int k = 0; k < 3; ++k)
    FX_CUDA(s, cudaMemcpyAsync(s->vcur.c[k], in + L.vel + k * align16(fb), fb, cudaMemcpyDefault, s->stream));
  FX_CUDA(s, cudaMemcpyAsync(s->lv[0].p[s->last_p], in + L.pressure, fb, cudaMemcpyDefault, s->stream));
  for (int k = 0; k < 2; ++k)
    FX_CUDA(s, cudaMemcpyAsync(s->flags[s->cur ^ k], in + L.flags + k * align16(gb), gb, cudaMemcpyDefault, s->stream));
  if ((st = fused_invalidate(s->fw, s->stream)) != FX_OK) return st;
  FX_CUDA(s, cudaStreamSynchronize(s->stream));
  return FX_OK;
}

fx_status fx_sim_synchronize(fx_sim* s) {
  if (!s) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_synchronize: NULL handle");
  FX_CUDA(s, cudaSetDevice(s->device));
  FX_CUDA(s, cudaStreamSynchronize(s->stream));
  if (fused_check_device_error(s->fw, s->stream) == FX_ERR_TIMEOUT)
    return fail(s, FX_ERR_TIMEOUT, "a bounded wait of the sparse sweep ran out; the results of that step are invalid");
  return FX_OK;
}

fx_status fx_sim_get_stats(fx_sim* s, fx_stats* o) {
  if (!s || !o) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_get_stats: NULL argument");
  std::memset(o, 0, sizeof *o);
  o->step_index = s->step_index;
  o->current_scalar_set = s->cur;
  o->last_pressure_buffer = s->last_p;
  o->brick_count = s->nb;
  o->kernels_per_step = s->last_kernel_count;
  o->flags = (s->last_step_graph ? FX_STATS_GRAPH : 0u) | (s->fw.use_graphs ? 0u : FX_STATS_GRAPHS_OFF);
  FX_CUDA(s, cudaSetDevice(s->device));
  if (s->last_cycle_launches) {
    // the V-cycle loop ran a device-decided number of cycles
    SolverDev d{};
    FX_CUDA(s, cudaMemcpyAsync(&d, s->fw.solver, sizeof d, cudaMemcpyDeviceToHost, s->stream));
    FX_CUDA(s, cudaStreamSynchronize(s->stream));
    o->kernels_per_step += (uint32_t)d.cycles * s->last_cycle_launches;
  }
  uint32_t active = 0;
  fx_status st = fused_count_active(s->fw, s->stream, s->flags[s->cur], s->nb, &active);
  if (st != FX_OK) return fail(s, st, "fx_sim_get_stats: counting active bricks failed");
  o->active_bricks = active;
  return FX_OK;
}

fx_status fx_sim_set_instrumentation(fx_sim* s, uint32_t flags) {
  if (!s) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_set_instrumentation: NULL handle");
  if (flags & ~(FX_INSTR_KERNEL_TIMES | FX_INSTR_COUNT_ACTIVE | FX_INSTR_SOLVER_NORMS))
    return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_set_instrumentation: unknown flags");
  if ((flags & FX_INSTR_SOLVER_NORMS) && s->kernels != FX_KERNELS_FUSED)
    return fail(s, FX_ERR_UNSUPPORTED, "fx_sim_set_instrumentation: solver statistics need the fused kernels");
  s->instr = flags;
  s->timer.on = (flags & FX_INSTR_KERNEL_TIMES) != 0;
  fused_set_timing(s->fw, s->timer.on);
  return FX_OK;
}

fx_status fx_sim_read_kernel_times(fx_sim* s, fx_kernel_time* out, uint32_t capacity, uint32_t* count) {
  if (!s || !count || (capacity && !out)) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_read_kernel_times: NULL argument");
  FX_CUDA(s, cudaSetDevice(s->device));
  FX_CUDA(s, cudaStreamSynchronize(s->stream));
  s->timer.drain();
  fused_drain_timing(s->fw, [&](const char* name, uint32_t launches, double ms) {
    auto& e = s->timer.acc[name];
    e.first += launches;
    e.second += ms;
  });
  uint32_t k = 0;
  for (auto& kv : s->timer.acc) {
    if (k < capacity) {
      std::memset(&out[k], 0, sizeof out[k]);
      std::snprintf(out[k].name, sizeof out[k].name, "%s", kv.first.c_str());
      out[k].launches = kv.second.first;
      out[k].total_ms = kv.second.second;
    }
    ++k;
  }
  *count = k;
  s->timer.acc.clear();
  return FX_OK;
}

fx_status fx_sim_read_active_counters(fx_sim* s, uint64_t* brick_steps, uint64_t* voxel_steps) {
  if (!s || !brick_steps || !voxel_steps) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_read_active_counters: NULL argument");
  FX_CUDA(s, cudaSetDevice(s->device));
  unsigned long long h[2] = {0, 0};
  FX_CUDA(s, cudaMemcpyAsync(h, s->d_active_acc, sizeof h, cudaMemcpyDeviceToHost, s->stream));
  FX_CUDA(s, cudaMemsetAsync(s->d_active_acc, 0, sizeof h, s->stream));
  FX_CUDA(s, cudaStreamSynchronize(s->stream));
  *brick_steps = h[0];
  *voxel_steps = h[1];
  return FX_OK;
}

fx_status fx_sim_get_stream(fx_sim* s, void** stream) {
  if (!s || !stream) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_get_stream: NULL argument");
  *stream = (void*)s->stream;
  return FX_OK;
}

const char* fx_sim_last_error(fx_sim* s) {
  if (!s) return g_last_error.c_str();
  return s->err.c_str();
}

// Test hook (declared in fenix_b200/csrc/fx_testing.h, not part of the public
// ABI): evaluates the pinned sin/cos on the device.
fx_status fx_test_pinned_sincos(const float* host_x, float* host_out, uint32_t n, int cosine) {
  if (n == 0) return FX_OK;
  float *dx = nullptr, *dout = nullptr;
  if (cudaMalloc(&dx, n * sizeof(float)) != cudaSuccess) return FX_ERR_OUT_OF_MEMORY;
  if (cudaMalloc(&dout, n * sizeof(float)) != cudaSuccess) {
    cudaFree(dx);
    return FX_ERR_OUT_OF_MEMORY;
  }
  fx_status st = FX_OK;
  if (cudaMemcpy(dx, host_x, n * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) st = FX_ERR_CUDA;
  if (st == FX_OK) {
    pinned_sincos_array(0, dx, dout, n, cosine);
    if (cudaMemcpy(host_out, dout, n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) st = FX_ERR_CUDA;
  }
  cudaFree(dx);
  cudaFree(dout);
  return st;
}

void fx_solver_settings_default(fx_solver_settings* o) {
  if (!o) return;
  std::memset(o, 0, sizeof *o);
  o->mode = FX_SOLVER_REFERENCE;
  o->levels = 5;
  o->pre_sweeps = 4;
  o->post_sweeps = 4;
  o->coarse_sweeps = 20;
  o->max_cycles = 30;
  o->warm_start = 1;
  o->omega = 2.0 / 3.0;
  o->tolerance = 1e-5;
}

fx_status fx_sim_set_solver(fx_sim* s, const fx_solver_settings* v) {
  if (!s || !v) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_set_solver: NULL argument");
  if (v->mode != FX_SOLVER_REFERENCE && v->mode != FX_SOLVER_VCYCLE)
    return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_set_solver: unknown mode");
  if (v->levels < 2 || v->levels > kMaxVLevels || v->pre_sweeps < 0 || v->pre_sweeps > 32 || v->post_sweeps < 0 || v->post_sweeps > 32 ||
      v->coarse_sweeps < 0 || v->coarse_sweeps > 256 || v->max_cycles < 1 || v->max_cycles > 1000)
    return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_set_solver: a count is out of range");
  if (!(v->omega > 0.0 && v->omega <= 1.0) || !(v->tolerance >= 0.0) || !std::isfinite(v->tolerance))
    return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_set_solver: omega must be in (0, 1] and tolerance finite and >= 0");
  if (v->mode == FX_SOLVER_VCYCLE && s->sparse)
    return fail(s, FX_ERR_UNSUPPORTED, "fx_sim_set_solver: sparse mode has no V-cycle form");
  s->solver = *v;
  s->solver.reserved = 0;
  return FX_OK;
}

fx_status fx_sim_get_solver(fx_sim* s, fx_solver_settings* o) {
  if (!s || !o) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_get_solver: NULL argument");
  *o = s->solver;
  return FX_OK;
}

fx_status fx_sim_set_sweep_variants(fx_sim* s, const int32_t v[3]) {
  if (!s || !v) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_set_sweep_variants: NULL argument");
  for (int l = 0; l < 3; ++l)
    if (v[l] != -1 && !sweep_variant_valid(v[l], s->lv[l].dm))
      return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_set_sweep_variants: variant " + std::to_string(v[l]) +
                                                         " does not fit level " + std::to_string(l));
  for (int l = 0; l < 3; ++l) s->sweep_variant[l] = v[l];
  return FX_OK;
}

fx_status fx_sim_get_sweep_variants(fx_sim* s, int32_t v[3]) {
  if (!s || !v) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_get_sweep_variants: NULL argument");
  for (int l = 0; l < 3; ++l) v[l] = s->sweep_variant[l] >= 0 ? s->sweep_variant[l] : sweep_variant_default(s->lv[l].dm);
  return FX_OK;
}

fx_status fx_sim_autotune(fx_sim* s, fx_autotune_report* o) {
  if (!s || !o) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_autotune: NULL argument");
  if (s->kernels != FX_KERNELS_FUSED) return fail(s, FX_ERR_UNSUPPORTED, "fx_sim_autotune: the plain kernels have nothing to tune");
  std::memset(o, 0, sizeof *o);
  FX_CUDA(s, cudaSetDevice(s->device));
  FX_CUDA(s, cudaStreamSynchronize(s->stream));
  cudaEvent_t ev[2] = {nullptr, nullptr};
  FX_CUDA(s, cudaEventCreate(&ev[0]));
  if (cudaEventCreate(&ev[1]) != cudaSuccess) {
    cudaEventDestroy(ev[0]);
    return fail(s, FX_ERR_CUDA, "fx_sim_autotune: cudaEventCreate failed");
  }
  fx_status st = FX_OK;
  for (int l = 0; l < 3 && st == FX_OK; ++l) {
    // Sweeps from the level's current iterate into the buffer that is dead
    // between steps (the non-current fine pressure; the mid and coarse buffers
    // restart from zero every solve).
    const LevelBuf& L = s->lv[l];
    const float* src = l == 0 ? L.p[s->last_p] : L.p[0];
    float* dst = l == 0 ? L.p[s->last_p ^ 1] : L.p[1];
    const int dflt = sweep_variant_default(L.dm);
    int best = dflt;
    float best_us = 0.0f;
    for (int v = 0; v < kSweepVariants && st == FX_OK; ++v) {
      if (!sweep_variant_valid(v, L.dm)) continue;
      float ms = 0.0f;
      for (int k = 0; k < 3; ++k) lean_sweep_variant(s->stream, v, L.dm, L.div, src, dst, L.dm, nullptr);
      cudaEventRecord(ev[0], s->stream);
      for (int k = 0; k < 20; ++k) lean_sweep_variant(s->stream, v, L.dm, L.div, src, dst, L.dm, nullptr);
      cudaEventRecord(ev[1], s->stream);
      if (cudaEventSynchronize(ev[1]) != cudaSuccess || cudaEventElapsedTime(&ms, ev[0], ev[1]) != cudaSuccess) {
        st = fail(s, FX_ERR_CUDA, "fx_sim_autotune: timing failed");
        break;
      }
      const float us = ms * 1000.0f / 20.0f;
      if (v == dflt) o->default_us[l] = us;
      if (best_us == 0.0f || us < best_us) {
        best_us = us;
        best = v;
      }
    }
    // A variant replaces the default only when it is at least 3 % faster:
    // closer timings of 20 sweeps are within the run-to-run noise, and on the
    // small levels such ties measured slower inside the step's graph.
    if (best != dflt && o->default_us[l] > 0.0f && best_us > 0.97f * o->default_us[l]) {
      best = dflt;
      best_us = o->default_us[l];
    }
    s->sweep_variant[l] = best;
    o->sweep_variant[l] = best;
    o->sweep_us[l] = best_us;
  }
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (st != FX_OK) return st;
  FX_CUDA(s, cudaGetLastError());
  return FX_OK;
}

static_assert(FX_BRICK_KERNELS == kBrickKernels && FX_BK_INJECT == BK_INJECT && FX_BK_ADVECT_SCALARS == BK_ADVECT_SCALARS &&
                  FX_BK_COMBUSTION == BK_COMBUSTION && FX_BK_BUOYANCY == BK_BUOYANCY &&
                  FX_BK_SPARSE_ADVECT_VELOCITY == BK_SP_ADVECT_VELOCITY && FX_BK_SPARSE_VORTICITY == BK_SP_VORTICITY &&
                  FX_BK_SPARSE_CONFINEMENT == BK_SP_CONFINEMENT && FX_BK_SPARSE_DIV_FIRST_SWEEP == BK_SP_DIV_FIRST &&
                  FX_BK_SPARSE_SWEEP == BK_SP_SWEEP && FX_BK_SPARSE_PROLONG_FINE == BK_SP_PROLONG_FINE &&
                  FX_BK_SPARSE_PROJECT == BK_SP_PROJECT,
              "the ABI's brick kernel indices follow BrickKernel");

fx_status fx_sim_set_brick_ctas(fx_sim* s, const int32_t* v) {
  if (!s || !v) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_set_brick_ctas: NULL argument");
  for (int k = 0; k < kBrickKernels; ++k)
    if (v[k] < 0 || v[k] > kBrickCtasMax)
      return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_set_brick_ctas: CTAs per SM must be 0 (default) or 1.." + std::to_string(kBrickCtasMax));
  for (int k = 0; k < kBrickKernels; ++k) s->brick_ctas[k] = (uint8_t)v[k];
  return FX_OK;
}

fx_status fx_sim_get_brick_ctas(fx_sim* s, int32_t* v) {
  if (!s || !v) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_get_brick_ctas: NULL argument");
  for (int k = 0; k < kBrickKernels; ++k) v[k] = s->brick_ctas[k];
  return FX_OK;
}

namespace {

// The timer names of each brick kernel's launches (fused_sequence's Timed labels).
const char* const kBrickKernelTimers[kBrickKernels][2] = {
    {"fused_inject", nullptr},
    {"fused_advect_scalars", nullptr},
    {"fused_combustion", nullptr},
    {"fused_buoyancy", nullptr},
    {"sparse_advect_velocity", nullptr},
    {"sparse_vorticity", nullptr},
    {"sparse_confinement", nullptr},
    {"sparse_div_first_sweep", nullptr},
    {"sparse_sweep", "sparse_sweep_prolong"},
    {"sparse_prolong_fine", nullptr},
    {"sparse_project", nullptr},
};

// A second simulation with s's settings and sources (not its state).
fx_status clone_settings(fx_sim* s, fx_sim** out) {
  fx_sim_options o;
  fx_sim_options_default(&o);
  o.width = s->dm.w, o.height = s->dm.h, o.depth = s->dm.d;
  o.scalar_advection_mode = s->advect_mode;
  o.runtime_mask = FX_PARAM_ALL;
  o.runtime = s->rp;
  o.quality_mask = FX_QUALITY_ALL;
  o.quality = s->quality;
  o.device = s->device;
  o.kernels = s->kernels;
  o.flags = s->opt_flags & ~FX_OPT_SPARSE;
  fx_sim* c = nullptr;
  fx_status st = fx_sim_create(&o, &c);
  if (st != FX_OK) return st;
  const uint32_t nsrc = (uint32_t)(s->host_sources.size() / 32);
  if ((st = fx_sim_update_sources(c, nsrc ? s->host_sources.data() : nullptr, nsrc)) == FX_OK &&
      (st = fx_sim_set_solver(c, &s->solver)) == FX_OK && (st = fx_sim_set_sparse(c, s->sparse ? 1 : 0)) == FX_OK) {
    for (int l = 0; l < 3; ++l) c->sweep_variant[l] = s->sweep_variant[l];
    c->debug_requested = s->debug_requested;
    *out = c;
    return FX_OK;
  }
  g_last_error = "fx_sim_autotune_bricks: clone: " + (c->err.empty() ? g_last_error : c->err);
  fx_sim_destroy(c);
  return st;
}

}  // namespace

fx_status fx_sim_autotune_bricks(fx_sim* s, double step_seconds, int32_t steps, fx_brick_tune_report* o) {
  if (!s || !o) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_autotune_bricks: NULL argument");
  if (!s->err.empty()) return FX_ERR_STATE;
  if (s->kernels != FX_KERNELS_FUSED) return fail(s, FX_ERR_UNSUPPORTED, "fx_sim_autotune_bricks: the plain kernels have no brick lists");
  if (!(step_seconds > 0.0) || !std::isfinite(step_seconds) || steps < 1 || steps > 64)
    return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_autotune_bricks: step_seconds must be > 0 and steps in 1..64");
  std::memset(o, 0, sizeof *o);
  FX_CUDA(s, cudaSetDevice(s->device));
  uint64_t bytes = 0;
  fx_sim_state_bytes(s, &bytes);
  void* blob = nullptr;
  FX_CUDA(s, device_alloc(&blob, bytes));
  fx_sim* c = nullptr;
  fx_status st = fx_sim_save_state(s, blob, bytes);
  if (st == FX_OK) st = clone_settings(s, &c);
  static const int kCandidates[] = {2, 4, 8, 16, 32};
  float us[5][kBrickKernels] = {};
  std::vector<fx_kernel_time> kt(128);
  for (int ci = 0; ci < 5 && st == FX_OK; ++ci) {
    for (int k = 0; k < kBrickKernels; ++k) c->brick_ctas[k] = (uint8_t)kCandidates[ci];
    // every candidate steps the same state, so every candidate does the same work
    if ((st = fx_sim_load_state(c, blob, bytes)) != FX_OK) break;
    double t = c->last_elapsed_s;
    if ((st = fx_sim_set_instrumentation(c, 0)) != FX_OK || (st = fx_sim_step(c, t += step_seconds, step_seconds)) != FX_OK) break;
    if ((st = fx_sim_set_instrumentation(c, FX_INSTR_KERNEL_TIMES)) != FX_OK) break;
    for (int k = 0; k < steps && st == FX_OK; ++k) st = fx_sim_step(c, t += step_seconds, step_seconds);
    uint32_t n = 0;
    if (st != FX_OK || (st = fx_sim_read_kernel_times(c, kt.data(), (uint32_t)kt.size(), &n)) != FX_OK) break;
    for (uint32_t i = 0; i < std::min<uint32_t>(n, (uint32_t)kt.size()); ++i)
      for (int k = 0; k < kBrickKernels; ++k)
        for (const char* name : kBrickKernelTimers[k])
          if (name && std::strcmp(kt[i].name, name) == 0) us[ci][k] += (float)(kt[i].total_ms * 1000.0 / steps);
  }
  if (st != FX_OK && c && !c->err.empty() && s->err.empty()) g_last_error = "fx_sim_autotune_bricks: " + c->err;
  if (c) fx_sim_destroy(c);
  cudaFree(blob);
  if (st != FX_OK) return st;
  const int dflt = 2;  // kCandidates[2] == kBrickCtasDefault
  static_assert(kBrickCtasDefault == 8, "the default grid is a candidate");
  for (int k = 0; k < kBrickKernels; ++k) {
    o->default_us[k] = us[dflt][k];
    int best = dflt;
    for (int ci = 0; ci < 5; ++ci)
      if (us[ci][k] > 0.0f && us[ci][k] < us[best][k]) best = ci;
    // closer than 3 % is within the run-to-run noise of a few steps
    if (!(us[dflt][k] > 0.0f) || us[best][k] > 0.97f * us[dflt][k]) best = dflt;
    o->ctas_per_sm[k] = kCandidates[best];
    o->us[k] = us[best][k];
    s->brick_ctas[k] = best == dflt ? 0 : (uint8_t)kCandidates[best];
  }
  return FX_OK;
}

fx_status fx_sim_set_sparse(fx_sim* s, int32_t on) {
  if (!s) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_sim_set_sparse: NULL handle");
  if (on && s->kernels != FX_KERNELS_FUSED) return fail(s, FX_ERR_UNSUPPORTED, "fx_sim_set_sparse: sparse mode needs the fused kernels");
  if (on && s->solver.mode == FX_SOLVER_VCYCLE) return fail(s, FX_ERR_UNSUPPORTED, "fx_sim_set_sparse: sparse mode has no V-cycle form");
  if (on && (s->bricks.x > 1024u || s->bricks.y > 1024u || s->bricks.z > 1024u))
    return fail(s, FX_ERR_UNSUPPORTED, "fx_sim_set_sparse: sparse mode supports at most 1024 bricks (8192 voxels) per axis");
  s->sparse = on != 0;
  return FX_OK;
}

fx_status fx_sim_get_sparse(fx_sim* s, int32_t* on) {
  if (!s || !on) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_get_sparse: NULL argument");
  *on = s->sparse ? 1 : 0;
  return FX_OK;
}

fx_status fx_sim_read_solver_stats(fx_sim* s, fx_solver_stats* o) {
  if (!s || !o) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_sim_read_solver_stats: NULL argument");
  std::memset(o, 0, sizeof *o);
  FX_CUDA(s, cudaSetDevice(s->device));
  SolverDev d{};
  FX_CUDA(s, cudaMemcpyAsync(&d, s->fw.solver, sizeof d, cudaMemcpyDeviceToHost, s->stream));
  FX_CUDA(s, cudaStreamSynchronize(s->stream));
  o->rhs_l2 = std::sqrt(d.rhs2);
  o->residual_l2 = std::sqrt(d.res2);
  o->relative_residual = o->rhs_l2 > 0 ? o->residual_l2 / o->rhs_l2 : (o->residual_l2 > 0 ? INFINITY : 0.0);
  double m;
  std::memcpy(&m, &d.maxdiv_bits, sizeof m);
  o->max_abs_divergence = m;
  o->cycles = d.cycles;
  o->converged = d.converged;
  return FX_OK;
}

}  // extern "C"

// ------------------------------------------------------------------- batches
// Independent simulations stepped together: each step is one CUDA graph in
// which every simulation's device sequence is a separate branch (captured on
// its own stream, forked from and joined to the batch stream), so the GPU runs
// them concurrently from a single launch. Host preparation (parameters,
// injection lists) is enqueued on the batch stream before the launch.
struct fx_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<fx_sim*> sims;
  std::vector<cudaStream_t> branch;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  bool use_graphs = true;
  struct Entry {
    cudaGraphExec_t exec;
    std::vector<FusedResult> results;
  };
  std::map<uint64_t, Entry> graphs;
  std::string err;
};

namespace {

fx_status batch_fail(fx_batch* b, fx_status code, const std::string& msg) {
  if (b) {
    if (b->err.empty()) b->err = msg;
  } else {
    g_last_error = msg;
  }
  return code;
}

// Enqueues every simulation's device sequence on its branch stream between the
// fork and join events (captured when the batch stream is capturing).
fx_status batch_sequences(fx_batch* b, std::vector<StepPlan>& sps, const std::vector<uint32_t>& ninj, std::vector<FusedResult>& res) {
  if (cudaEventRecord(b->fork, b->stream) != cudaSuccess) return batch_fail(b, FX_ERR_CUDA, "fx_batch_step: fork event failed");
  for (size_t i = 0; i < b->sims.size(); ++i) {
    FusedStep fs = sps[i].fs;
    fs.stream = b->branch[i];
    if (cudaStreamWaitEvent(b->branch[i], b->fork, 0) != cudaSuccess) return batch_fail(b, FX_ERR_CUDA, "fx_batch_step: fork wait failed");
    const fx_status st = fused_sequence(b->sims[i]->fw, fs, ninj[i], res[i]);
    if (st != FX_OK) return batch_fail(b, st, "fx_batch_step: simulation " + std::to_string(i) + ": " + res[i].error);
    if (cudaEventRecord(b->join[i], b->branch[i]) != cudaSuccess || cudaStreamWaitEvent(b->stream, b->join[i], 0) != cudaSuccess)
      return batch_fail(b, FX_ERR_CUDA, "fx_batch_step: join failed");
  }
  return FX_OK;
}

}  // namespace

extern "C" {

fx_status fx_batch_create(const fx_sim_options* const* options, uint32_t count, fx_batch** out) {
  g_last_error.clear();
  if (!out || !options || count == 0 || count > 4096)
    return batch_fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_batch_create: need 1..4096 option structs and an out pointer");
  *out = nullptr;
  for (uint32_t i = 0; i < count; ++i) {
    if (!options[i]) return batch_fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_batch_create: NULL options");
    if (options[i]->struct_size != sizeof(fx_sim_options))
      return batch_fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_batch_create: struct_size does not match this library's fx_sim_options");
    if (options[i]->kernels != FX_KERNELS_FUSED)
      return batch_fail(nullptr, FX_ERR_UNSUPPORTED, "fx_batch_create: batches run the fused kernels");
    if (options[i]->device != options[0]->device)
      return batch_fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_batch_create: every simulation of a batch is on one device");
  }
  fx_batch* b = new (std::nothrow) fx_batch;
  if (!b) return batch_fail(nullptr, FX_ERR_OUT_OF_MEMORY, "fx_batch_create: host allocation failed");
  b->device = options[0]->device;
  auto bail = [&](fx_status code, const std::string& msg) {
    fx_batch_destroy(b);
    return batch_fail(nullptr, code, msg);
  };
  if (cudaSetDevice(b->device) != cudaSuccess) return bail(FX_ERR_CUDA, "fx_batch_create: cudaSetDevice failed (no CUDA device?)");
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return bail(FX_ERR_CUDA, "fx_batch_create: stream creation failed");
  if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) return bail(FX_ERR_CUDA, "fx_batch_create: event creation failed");
  for (uint32_t i = 0; i < count; ++i) {
    fx_sim_options o = *options[i];
    o.stream = b->stream;
    fx_sim* sim = nullptr;
    const fx_status st = fx_sim_create(&o, &sim);
    if (st != FX_OK) return bail(st, "fx_batch_create: simulation " + std::to_string(i) + ": " + g_last_error);
    b->sims.push_back(sim);
    if ((o.flags & FX_OPT_NO_GRAPHS) != 0) b->use_graphs = false;
    cudaStream_t br = nullptr;
    cudaEvent_t ev = nullptr;
    if (cudaStreamCreateWithFlags(&br, cudaStreamNonBlocking) != cudaSuccess) return bail(FX_ERR_CUDA, "fx_batch_create: stream creation failed");
    b->branch.push_back(br);
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return bail(FX_ERR_CUDA, "fx_batch_create: event creation failed");
    b->join.push_back(ev);
  }
  *out = b;
  return FX_OK;
}

void fx_batch_destroy(fx_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second.exec);
  for (fx_sim* sim : b->sims) fx_sim_destroy(sim);
  for (cudaStream_t br : b->branch) cudaStreamDestroy(br);
  for (cudaEvent_t ev : b->join) cudaEventDestroy(ev);
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

fx_status fx_batch_size(fx_batch* b, uint32_t* count) {
  if (!b || !count) return batch_fail(b, FX_ERR_INVALID_ARGUMENT, "fx_batch_size: NULL argument");
  *count = (uint32_t)b->sims.size();
  return FX_OK;
}

fx_status fx_batch_get_sim(fx_batch* b, uint32_t index, fx_sim** sim) {
  if (!b || !sim) return batch_fail(b, FX_ERR_INVALID_ARGUMENT, "fx_batch_get_sim: NULL argument");
  if (index >= b->sims.size()) return batch_fail(b, FX_ERR_INVALID_ARGUMENT, "fx_batch_get_sim: index out of range");
  *sim = b->sims[index];
  return FX_OK;
}

fx_status fx_batch_step(fx_batch* b, double elapsed, double step_s) {
  if (!b) return batch_fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_batch_step: NULL handle");
  if (!b->err.empty()) return FX_ERR_STATE;
  if (cudaSetDevice(b->device) != cudaSuccess) return batch_fail(b, FX_ERR_CUDA, "fx_batch_step: cudaSetDevice failed");
  const size_t n = b->sims.size();
  std::vector<StepPlan> sps(n);
  std::vector<uint32_t> ninj(n, 0);
  std::vector<uint32_t> prep_launches(n, 0);
  bool timing = false;
  uint64_t key = 0xcbf29ce484222325ull;
  for (size_t i = 0; i < n; ++i) {
    fx_sim* sim = b->sims[i];
    if (!sim->err.empty()) return batch_fail(b, FX_ERR_STATE, "fx_batch_step: simulation " + std::to_string(i) + " has an error: " + sim->err);
    fx_status st = step_begin(sim, elapsed, step_s, sps[i]);
    if (st != FX_OK) return batch_fail(b, st, "fx_batch_step: simulation " + std::to_string(i) + ": " + sim->err);
    FusedResult prep;
    st = fused_prepare(sim->fw, sps[i].fs, &ninj[i], prep);
    if (st != FX_OK) return batch_fail(b, st, "fx_batch_step: simulation " + std::to_string(i) + ": " + prep.error);
    prep_launches[i] = prep.launches;
    timing = timing || sim->fw.timing;
    key = (key ^ (fused_key(sps[i].fs, ninj[i]) + 0x9e3779b97f4a7c15ull * (i + 1))) * 0x100000001b3ull;
  }
  std::vector<FusedResult> res(n);
  bool replay = false;
  if (b->use_graphs && !timing) {
    auto it = b->graphs.find(key);
    if (it == b->graphs.end()) {
      cudaGraph_t g = nullptr;
      if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess)
        return batch_fail(b, FX_ERR_CUDA, "fx_batch_step: stream capture failed to start");
      std::vector<FusedResult> tmp(n);
      const std::string before = b->err;
      const fx_status cst = batch_sequences(b, sps, ninj, tmp);
      const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
      cudaGraphExec_t ex = nullptr;
      cudaError_t ie = cudaErrorUnknown;
      if (cst == FX_OK && ce == cudaSuccess) ie = cudaGraphInstantiate(&ex, g, 0);
      if (g) cudaGraphDestroy(g);
      if (cst != FX_OK || ce != cudaSuccess || ie != cudaSuccess) {
        cudaGetLastError();
        b->err = before;  // a capture problem falls back to direct launches
        b->use_graphs = false;
      } else {
        it = b->graphs.emplace(key, fx_batch::Entry{ex, tmp}).first;
      }
    }
    if (b->use_graphs) {
      if (cudaGraphLaunch(it->second.exec, b->stream) != cudaSuccess) return batch_fail(b, FX_ERR_CUDA, "fx_batch_step: graph launch failed");
      res = it->second.results;
      replay = true;
    }
  }
  if (!replay) {
    const fx_status st = batch_sequences(b, sps, ninj, res);
    if (st != FX_OK) return st;
  }
  for (size_t i = 0; i < n; ++i) {
    res[i].launches += prep_launches[i];
    res[i].graph = replay;
    const fx_status st = step_finish(b->sims[i], FX_OK, &res[i], sps[i], elapsed);
    if (st != FX_OK) return batch_fail(b, st, "fx_batch_step: simulation " + std::to_string(i) + ": " + b->sims[i]->err);
  }
  return FX_OK;
}

fx_status fx_batch_synchronize(fx_batch* b) {
  if (!b) return batch_fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_batch_synchronize: NULL handle");
  if (cudaSetDevice(b->device) != cudaSuccess || cudaStreamSynchronize(b->stream) != cudaSuccess)
    return batch_fail(b, FX_ERR_CUDA, "fx_batch_synchronize: the batch stream failed");
  return FX_OK;
}

fx_status fx_batch_get_stream(fx_batch* b, void** stream) {
  if (!b || !stream) return batch_fail(b, FX_ERR_INVALID_ARGUMENT, "fx_batch_get_stream: NULL argument");
  *stream = (void*)b->stream;
  return FX_OK;
}

const char* fx_batch_last_error(fx_batch* b) { return b ? b->err.c_str() : g_last_error.c_str(); }

// Test hook: exhaustive comparison of the pressure kernels' division by 6 with
// the IEEE division on the device. Returns the mismatch count in *bad.
// Test entry (host arithmetic only): the planes per block a marching kernel
// launch uses for a w x h x d level with `slots` resident blocks. kind 0: one
// wave over 128 x 8 tiles (the fine sweeps, the projection); 1: the same in
// runs of an even number of planes (the divergence; d must be even); 2: whole
// waves over 32 x 8 tiles (the velocity advection).
fx_status fx_test_march_plan(int32_t kind, uint32_t w, uint32_t h, uint32_t d, int32_t slots, int32_t* run) {
  if (!run || w == 0 || h == 0 || d == 0 || slots < 1 || kind < 0 || kind > 2 || (kind == 1 && d % 2 != 0))
    return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_test_march_plan: invalid argument");
  const Dims dm{w, h, d};
  *run = kind == 0 ? march_plan_one_wave(dm, slots) : kind == 1 ? march_plan_pairs(dm, slots) : march_plan_waves(dm, 32, 8, slots);
  return FX_OK;
}

// Test entry (fault injection): from now on the `nth` device or pinned-host
// allocation that the library makes fails as an exhausted memory would
// (cudaErrorMemoryAllocation, without calling CUDA); 0 switches it off.
fx_status fx_test_fail_allocations(int32_t nth) {
  if (nth < 0) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_test_fail_allocations: negative count");
  g_alloc_countdown.store(nth);
  return FX_OK;
}

// Test entry (failure detection): the bound (ns) of every wait of the
// TMA-staged sparse sweep and extra bytes its tile stages expect. With extra > 0
// no stage ever completes, so each wait runs out after wait_ns, the kernel
// records it and returns, and the next synchronizing call reports
// FX_ERR_TIMEOUT. (0, 1e9) restores normal operation.
fx_status fx_test_sparse_tma_wait(fx_sim* s, uint64_t wait_ns, uint32_t extra_tx) {
  if (!s || wait_ns == 0) return fail(s, FX_ERR_INVALID_ARGUMENT, "fx_test_sparse_tma_wait: invalid argument");
  fused_set_tma_test(s->fw, wait_ns, extra_tx);
  return FX_OK;
}

// Test entry: sr_half(x[i], sr_draw(i, site, step)) on the device for host arrays
// (compared with the oracle's stochastic binary16 rounding bit for bit).
fx_status fx_test_sr_half(const float* host_x, float* host_out, uint32_t n, uint32_t site, uint32_t step) {
  if (!host_x || !host_out) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_test_sr_half: NULL argument");
  float* d = nullptr;
  if (cudaMalloc(&d, (size_t)n * 2 * sizeof(float)) != cudaSuccess) return FX_ERR_OUT_OF_MEMORY;
  cudaError_t e = cudaMemcpy(d, host_x, (size_t)n * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = sr_half_array(d, d + n, n, site, step);
  if (e == cudaSuccess) e = cudaMemcpy(host_out, d + n, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return e == cudaSuccess ? FX_OK : FX_ERR_CUDA;
}

fx_status fx_test_div6_exhaustive(unsigned long long* bad) {
  if (!bad) return FX_ERR_INVALID_ARGUMENT;
  return div6_exhaustive_check(bad) == cudaSuccess ? FX_OK : FX_ERR_CUDA;
}

}  // extern "C"

// ------------------------------------------------------------------------------
// Differentiable rollout: K plain FP32 steps from the simulation's state with an
// inflow patch as the control, the loss sum (density_K - target)^2, and its
// gradient with respect to the inflow values and the initial velocity by the
// adjoint kernels of fx_adjoint.cu. The forward keeps a state checkpoint every
// `checkpoint_interval` steps; the backward recomputes each segment from its
// checkpoint, then steps back through it, re-running each step with the copies
// its adjoint reads.
// ------------------------------------------------------------------------------
namespace {

struct HostState {
  int cur = 0;
  int64_t step_index = 0;
  bool initialized = false;
  double start_s = 0, last_elapsed_s = 0;
  int last_p = 0;
  bool debug_requested = false;
};

}  // namespace

// What the adjoint of one step reads of that step's forward: its tape (the
// fields the plain step's hooks record) and the fields the step leaves in the
// simulation (the input set after the injections, the output set, the set
// before combustion, the curl and its length, both brick flag arrays, the step
// uniform and the final pressure buffer's index).
struct StepTape {
  float* t1 = nullptr;
  float* r1 = nullptr;
  VelField v1{}, a{}, b{};
  ScalarSet in{}, out{}, snap{};
  VelField w{};
  float* wmag = nullptr;
  uint32_t* flags_in = nullptr;
  uint32_t* flags_out = nullptr;
  Params* P = nullptr;
  int last_p = 0;
};

struct fx_rollout {
  fx_sim* s = nullptr;
  int device = 0;
  fx_rollout_desc d{};
  InflowPatch patch{};
  size_t n = 0;
  uint32_t npatch = 0, nck = 0;
  void* arena = nullptr;
  float* inflow = nullptr;
  float* target = nullptr;
  float* grad_inflow = nullptr;
  double* loss = nullptr;
  float* ck = nullptr;   // nck states of 7 n floats: density, temperature, fuel, reaction, velocity x, y, z
  float* seg = nullptr;  // checkpoint_interval states
  float* fin = nullptr;  // the final state of the latest forward
  std::vector<HostState> ck_host, seg_host;
  HostState fin_host;
  float* t1 = nullptr;
  float* r1 = nullptr;
  VelField v1{}, a{}, b{};
  ScalarSet lam_s[2]{};
  VelField lam_v[2]{};
  VelField lam_c{}, lam_w{}, lam_g{};
  float* lam_wmag = nullptr;
  float* hot = nullptr;
  float* dens = nullptr;
  float* lam_p[3][2]{};
  float* lam_div[3]{};
  bool have_target = false;
  bool forward_done = false;
  // The untaped steps (the forward and the segment recomputation) run the fused
  // step when the simulation has the fused kernels and every inflow value is
  // within the speed limit (the fused velocity advection clamps on read, where
  // the plain step leaves the inflow values as they are); both give the same bits.
  bool fused_steps = false;
  // The taped re-runs of the backward use the fused step too (fused_steps), with
  // the tape recorded inside it; plain_tape (a test entry) keeps them plain.
  bool plain_tape = false;
  // reverse_pressure captured as a graph, for the schedule counts rp_key (qi[2..6])
  cudaGraphExec_t rp_exec = nullptr;
  int rp_key[5]{};
  // One StepTape per step of a segment, recorded while the segment is
  // recomputed; empty when they did not fit, and then each step is re-run taped
  // just before its adjoint. rerun_tape (a test entry) forces the re-runs.
  void* slot_arena = nullptr;
  std::vector<StepTape> slots;
  bool rerun_tape = false;
  // reverse_step of each (slot, o) as a graph, and the inputs it was captured for
  std::vector<cudaGraphExec_t> rs_exec;
  std::vector<std::array<uint64_t, 8>> rs_key;
};

namespace {

// Configuration and argument errors of the rollout are reported through
// fx_last_error and leave the simulation usable; CUDA failures are recorded on
// the simulation (sticky), like its own.
fx_status rollout_check(fx_rollout* r) {
  fx_sim* s = r->s;
  if (!s->err.empty()) return fail(nullptr, FX_ERR_STATE, "fx_rollout: the simulation has an error: " + s->err);
  if (s->half) return fail(nullptr, FX_ERR_UNSUPPORTED, "fx_rollout: the simulation must use f32 storage");
  if (s->sparse) return fail(nullptr, FX_ERR_UNSUPPORTED, "fx_rollout: the adjoint differentiates the dense step, not sparse mode");
  if (s->solver.mode != FX_SOLVER_REFERENCE || s->advect_mode != FX_ADVECT_MACCORMACK)
    return fail(nullptr, FX_ERR_UNSUPPORTED, "fx_rollout: needs the reference pressure schedule and MacCormack advection");
  if (s->qi[0] != 1 || s->qi[1] != 1)
    return fail(nullptr, FX_ERR_UNSUPPORTED, "fx_rollout: needs pressure and vorticity intervals of 1");
  return FX_OK;
}

HostState host_state(const fx_sim* s) {
  HostState h;
  h.cur = s->cur;
  h.step_index = s->step_index;
  h.initialized = s->initialized;
  h.start_s = s->start_s;
  h.last_elapsed_s = s->last_elapsed_s;
  h.last_p = s->last_p;
  h.debug_requested = s->debug_requested;
  return h;
}

fx_status save_state(fx_rollout* r, float* dst, HostState& h) {
  fx_sim* s = r->s;
  h = host_state(s);
  const size_t b = r->n * sizeof(float);
  for (int k = 0; k < 4; ++k) FX_CUDA(s, cudaMemcpyAsync(dst + k * r->n, s->sets[s->cur].f[k], b, cudaMemcpyDeviceToDevice, s->stream));
  for (int k = 0; k < 3; ++k) FX_CUDA(s, cudaMemcpyAsync(dst + (4 + k) * r->n, s->vcur.c[k], b, cudaMemcpyDeviceToDevice, s->stream));
  return FX_OK;
}

fx_status restore_state(fx_rollout* r, const float* src, const HostState& h) {
  fx_sim* s = r->s;
  // the fused path's per-brick bookkeeping is rebuilt from the restored fields
  if (s->kernels == FX_KERNELS_FUSED) fused_invalidate(s->fw, s->stream);
  s->cur = h.cur;
  s->step_index = h.step_index;
  s->initialized = h.initialized;
  s->start_s = h.start_s;
  s->last_elapsed_s = h.last_elapsed_s;
  s->last_p = h.last_p;
  s->debug_requested = h.debug_requested;
  const size_t b = r->n * sizeof(float);
  for (int k = 0; k < 4; ++k) FX_CUDA(s, cudaMemcpyAsync(s->sets[s->cur].f[k], src + k * r->n, b, cudaMemcpyDeviceToDevice, s->stream));
  for (int k = 0; k < 3; ++k) FX_CUDA(s, cudaMemcpyAsync(s->vcur.c[k], src + (4 + k) * r->n, b, cudaMemcpyDeviceToDevice, s->stream));
  return FX_OK;
}

fx_status rollout_step(fx_rollout* r, uint32_t k, const PlainHooks& hk) {
  fx_sim* s = r->s;
  const double elapsed = r->d.start_elapsed + (double)k * r->d.step_seconds;
  StepPlan sp;
  fx_status st = step_begin(s, elapsed, r->d.step_seconds, sp);
  if (st != FX_OK) return st;
  const bool taped = hk.t1 || hk.r1 || hk.v1.c[0] || hk.a.c[0] || hk.b.c[0];
  const bool full_tape = hk.t1 && hk.r1 && hk.v1.c[0] && hk.a.c[0] && hk.b.c[0];
  if (r->fused_steps && (!taped || (full_tape && !r->plain_tape))) {
    sp.fs.inflow = hk.inflow;
    sp.fs.inflow_patch = hk.patch;
    if (taped) {
      sp.fs.tape_t1 = hk.t1;
      sp.fs.tape_r1 = hk.r1;
      sp.fs.tape_v1 = hk.v1;
      sp.fs.tape_a = hk.a;
      sp.fs.tape_b = hk.b;
      sp.fs.debug_fields = true;  // the adjoint reads the curl w of the step
    }
    FusedResult fr;
    st = fused_step(s->fw, sp.fs, fr);
    if (st != FX_OK) fail(s, st, "fx_rollout: fused step failed: " + fr.error);
    return step_finish(s, st, &fr, sp, elapsed);
  }
  st = step_finish(s, step_plain(s, sp.vort_on, sp.pressure_on, sp.debug_on, &hk), nullptr, sp, elapsed);
  if (s->kernels == FX_KERNELS_FUSED) fused_invalidate(s->fw, s->stream);
  return st;
}

// The speed limit of the step uniform (speed_limit in fx_math.cuh), in the same
// f32 operations.
float speed_limit_of(const fx_sim* s) {
  const float dx = (float)(s->rp.world_size / (double)std::max(s->dm.w, s->dm.d));
  return 80.0f / (dx < 0.001f ? 0.001f : dx);
}

// PressureSolvePass.smooth (:129-143) in reverse.
// Each sweep's adjoint moves lam from the buffer the sweep wrote to the one it
// read, and that written buffer's adjoint is then spent. The first sweep
// undone adds to what its read buffer holds; every later one writes its read
// buffer whole, since that buffer's adjoint was spent by the sweep undone just
// before. The buffer left over at the end is cleared.
void reverse_smooth(fx_rollout* r, int l, int iters, int start) {
  fx_sim* s = r->s;
  const Dims dm = s->lv[l].dm;
  for (int k = iters - 1; k >= 0; --k) {
    const int a = start ^ (k & 1);
    adj_jacobi(s->stream, dm, r->lam_p[l][a ^ 1], r->lam_p[l][a], r->lam_div[l], k == iters - 1);
    if (k == 0) cudaMemsetAsync(r->lam_p[l][a ^ 1], 0, count_of(dm) * sizeof(float), s->stream);
  }
}

// PressureSolvePass.solve (:68-84) in reverse: from the adjoint of the final
// fine pressure buffer to the adjoint of the fine divergence (lam_div[0]).
void reverse_pressure(fx_rollout* r) {
  fx_sim* s = r->s;
  const int* q = s->qi;
  const int fine_pre = q[2] & 1, mid_pre = q[4] & 1, coarse = q[6] & 1;
  const int mid = mid_pre ^ (q[5] & 1);
  reverse_smooth(r, 0, q[3], fine_pre);
  adj_prolong(s->stream, s->lv[1].dm, s->lv[0].dm, r->lam_p[0][0], r->lam_p[1][mid]);
  reverse_smooth(r, 1, q[5], mid_pre);
  adj_prolong(s->stream, s->lv[2].dm, s->lv[1].dm, r->lam_p[1][0], r->lam_p[2][coarse]);
  reverse_smooth(r, 2, q[6], 0);
  adj_restrict(s->stream, s->lv[1].dm, s->lv[2].dm, r->lam_div[2], r->lam_div[1]);
  reverse_smooth(r, 1, q[4], 0);
  adj_restrict(s->stream, s->lv[0].dm, s->lv[1].dm, r->lam_div[1], r->lam_div[0]);
  reverse_smooth(r, 0, q[2], 0);
}

// reverse_pressure as one CUDA graph: its launches (45 small kernels and clears
// at the three levels for the 4/4/4/4/20 schedule) and their buffers are the
// same every step, so
// the graph is captured on first use and again only when the solve's schedule
// changes.
fx_status launch_reverse_pressure(fx_rollout* r) {
  fx_sim* s = r->s;
  const int* q = s->qi;
  if (!r->rp_exec || !std::equal(q + 2, q + 7, r->rp_key)) {
    if (r->rp_exec) {
      cudaGraphExecDestroy(r->rp_exec);
      r->rp_exec = nullptr;
    }
    FX_CUDA(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    reverse_pressure(r);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&r->rp_exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) r->rp_exec = nullptr;
    FX_CUDA(s, e);
    std::copy(q + 2, q + 7, r->rp_key);
  }
  FX_CUDA(s, cudaGraphLaunch(r->rp_exec, s->stream));
  return FX_OK;
}

// The tape of the step just run from a state whose current set index was
// `cur`, in place in the simulation and the rollout's single tape.
StepTape sim_tape(fx_rollout* r, int cur) {
  fx_sim* s = r->s;
  StepTape t;
  t.t1 = r->t1;
  t.r1 = r->r1;
  t.v1 = r->v1;
  t.a = r->a;
  t.b = r->b;
  t.in = s->sets[cur];
  t.out = s->sets[cur ^ 1];
  t.snap = s->sets[2];
  t.w = s->vort;
  t.wmag = s->vort_mag;
  t.flags_in = s->flags[cur];
  t.flags_out = s->flags[cur ^ 1];
  t.P = s->d_params;
  t.last_p = s->last_p;
  return t;
}

// Copies into the slot `t` (whose t1, r1, v1, a, b the step already wrote) the
// fields of the step just run from a state whose current set index was `cur`.
fx_status record_tape(fx_rollout* r, int cur, StepTape& t) {
  fx_sim* s = r->s;
  const StepTape src = sim_tape(r, cur);
  cudaStream_t st = s->stream;
  const size_t b = r->n * sizeof(float), fb = (size_t)s->nb * sizeof(uint32_t);
  for (int k = 0; k < 4; ++k) {
    FX_CUDA(s, cudaMemcpyAsync(t.in.f[k], src.in.f[k], b, cudaMemcpyDeviceToDevice, st));
    FX_CUDA(s, cudaMemcpyAsync(t.out.f[k], src.out.f[k], b, cudaMemcpyDeviceToDevice, st));
    FX_CUDA(s, cudaMemcpyAsync(t.snap.f[k], src.snap.f[k], b, cudaMemcpyDeviceToDevice, st));
  }
  for (int c = 0; c < 3; ++c) FX_CUDA(s, cudaMemcpyAsync(t.w.c[c], src.w.c[c], b, cudaMemcpyDeviceToDevice, st));
  FX_CUDA(s, cudaMemcpyAsync(t.wmag, src.wmag, b, cudaMemcpyDeviceToDevice, st));
  FX_CUDA(s, cudaMemcpyAsync(t.flags_in, src.flags_in, fb, cudaMemcpyDeviceToDevice, st));
  FX_CUDA(s, cudaMemcpyAsync(t.flags_out, src.flags_out, fb, cudaMemcpyDeviceToDevice, st));
  FX_CUDA(s, cudaMemcpyAsync(t.P, src.P, sizeof(Params), cudaMemcpyDeviceToDevice, st));
  t.last_p = src.last_p;
  return FX_OK;
}

// Device bytes of one StepTape slot: 27 fields of n floats, two brick flag
// arrays and the step uniform, each start 256-byte aligned.
size_t slot_bytes(size_t n, size_t nb) {
  auto al = [](size_t v) { return (v + 255) / 256 * 256; };
  return 27 * al(n * sizeof(float)) + 2 * al(nb * sizeof(uint32_t)) + al(sizeof(Params));
}

// Carves `count` slots out of the arena at `base`.
void carve_slots(fx_rollout* r, char* base, uint32_t count) {
  const size_t nb = r->s->nb;
  auto al = [](size_t v) { return (v + 255) / 256 * 256; };
  char* p = base;
  auto fl = [&]() {
    float* q = reinterpret_cast<float*>(p);
    p += al(r->n * sizeof(float));
    return q;
  };
  r->slots.assign(count, StepTape{});
  for (StepTape& t : r->slots) {
    t.t1 = fl();
    t.r1 = fl();
    for (VelField* v : {&t.v1, &t.a, &t.b, &t.w})
      for (int c = 0; c < 3; ++c) v->c[c] = fl();
    for (ScalarSet* q : {&t.in, &t.out, &t.snap})
      for (int k = 0; k < 4; ++k) q->f[k] = fl();
    t.wmag = fl();
    t.flags_in = reinterpret_cast<uint32_t*>(p);
    p += al(nb * sizeof(uint32_t));
    t.flags_out = reinterpret_cast<uint32_t*>(p);
    p += al(nb * sizeof(uint32_t));
    t.P = reinterpret_cast<Params*>(p);
    p += al(sizeof(Params));
  }
}

// The adjoint of one step from the state `state0`, whose forward fields are in
// `t`: lam_s[o], lam_v[o] hold the adjoint of the step's output state;
// lam_s[o ^ 1], lam_v[o ^ 1] receive the adjoint of its input state.
fx_status reverse_step(fx_rollout* r, const StepTape& t, const float* state0, int o, bool in_graph = false) {
  fx_sim* s = r->s;
  cudaStream_t st = s->stream;
  const Dims dm = s->dm;
  const size_t n = r->n;
  const Params* P = t.P;
  const uint32_t nsrc = std::max<uint32_t>(s->src_count, 1);
  ScalarSet S0;
  for (int k = 0; k < 4; ++k) S0.f[k] = const_cast<float*>(state0) + k * n;
  VelField V0;
  for (int k = 0; k < 3; ++k) V0.c[k] = const_cast<float*>(state0) + (4 + k) * n;
  const ScalarSet lo = r->lam_s[o], li = r->lam_s[o ^ 1];
  const VelField lvo = r->lam_v[o], lvi = r->lam_v[o ^ 1];
  for (int l = 0; l < 3; ++l) {
    const size_t c = count_of(s->lv[l].dm) * sizeof(float);
    FX_CUDA(s, cudaMemsetAsync(r->lam_p[l][0], 0, c, st));
    FX_CUDA(s, cudaMemsetAsync(r->lam_p[l][1], 0, c, st));
    FX_CUDA(s, cudaMemsetAsync(r->lam_div[l], 0, c, st));
  }
  adj_project(st, dm, lvo, r->lam_c, r->lam_p[0][t.last_p]);
  if (in_graph) {
    reverse_pressure(r);
  } else {
    fx_status ps = launch_reverse_pressure(r);
    if (ps != FX_OK) return ps;
  }
  adj_divergence(st, dm, r->lam_div[0], r->lam_c);
  adj_confinement(st, dm, P, t.w, t.wmag, t.out, t.b, r->lam_c, r->lam_w, r->lam_wmag, r->lam_g, lo);
  adj_vorticity(st, dm, t.w, t.wmag, r->lam_w, r->lam_wmag, r->lam_g, r->lam_c);
  adj_buoyancy(st, dm, s->bricks, P, t.out, t.flags_out, t.a, r->lam_c, lo, r->hot, r->dens);
  adj_combustion(st, dm, s->bricks, P, t.snap, t.flags_out, lo, r->hot);
  for (int k = 0; k < 4; ++k) FX_CUDA(s, cudaMemsetAsync(li.f[k], 0, n * sizeof(float), st));
  for (int k = 0; k < 3; ++k) FX_CUDA(s, cudaMemsetAsync(lvi.c[k], 0, n * sizeof(float), st));
  adj_advect_scalars(st, dm, s->bricks, P, t.in, t.a, t.flags_in, lo, li, r->lam_c);
  adj_advect_velocity(st, dm, P, t.v1, r->lam_c, lvi);
  adj_inject_igniter(st, dm, P, s->d_sources, nsrc, t.t1, t.in.f[2], t.r1, li);
  adj_inflow(st, dm, r->patch, lvi, r->grad_inflow);
  adj_inject_velocity(st, dm, P, s->d_sources, nsrc, V0, lvi);
  adj_inject_scalar(st, dm, P, s->d_sources, nsrc, S0, li);
  FX_CUDA(s, cudaGetLastError());
  return FX_OK;
}

// The inputs of a captured reverse step that can change between backward calls.
std::array<uint64_t, 8> reverse_key(fx_rollout* r, const StepTape& t) {
  const fx_sim* s = r->s;
  return {(uint64_t)(uintptr_t)s->d_sources, s->src_count, (uint64_t)s->qi[2], (uint64_t)s->qi[3], (uint64_t)s->qi[4],
          (uint64_t)s->qi[5], (uint64_t)s->qi[6], (uint64_t)t.last_p};
}

// reverse_step of slot j as one CUDA graph per (slot, o): within a segment the
// adjoint steps run back to back from the slots, with the same buffers every
// backward call, so each is captured on first use and replayed.
fx_status reverse_step_slot(fx_rollout* r, uint32_t j, int o) {
  fx_sim* s = r->s;
  const StepTape& t = r->slots[j];
  const float* state0 = r->seg + (size_t)j * 7 * r->n;
  const std::array<uint64_t, 8> key = reverse_key(r, t);
  const size_t idx = (size_t)j * 2 + (size_t)o;
  if (r->rs_exec.size() != r->slots.size() * 2) r->rs_exec.assign(r->slots.size() * 2, nullptr);
  if (r->rs_key.size() != r->rs_exec.size()) r->rs_key.assign(r->rs_exec.size(), {});
  cudaGraphExec_t& ex = r->rs_exec[idx];
  if (ex && r->rs_key[idx] != key) {
    cudaGraphExecDestroy(ex);
    ex = nullptr;
  }
  if (!ex) {
    FX_CUDA(s, cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    const fx_status st = reverse_step(r, t, state0, o, true);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (st != FX_OK) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&ex, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) ex = nullptr;
    FX_CUDA(s, e);
    r->rs_key[idx] = key;
  }
  FX_CUDA(s, cudaGraphLaunch(ex, s->stream));
  return FX_OK;
}

}  // namespace

extern "C" {

void fx_rollout_desc_default(fx_rollout_desc* d) {
  if (!d) return;
  std::memset(d, 0, sizeof *d);
  d->struct_size = sizeof *d;
  d->steps = 64;
  d->checkpoint_interval = 8;
  d->step_seconds = 1.0 / 60.0;
}

fx_status fx_rollout_create(fx_sim* s, const fx_rollout_desc* d, fx_rollout** out) {
  if (!s || !d || !out) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_rollout_create: NULL argument");
  *out = nullptr;
  if (d->struct_size < sizeof(fx_rollout_desc)) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_rollout_create: struct_size too small");
  if (d->steps == 0 || d->checkpoint_interval == 0 || !(d->step_seconds > 0.0) || !std::isfinite(d->start_elapsed))
    return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_rollout_create: steps, checkpoint_interval and step_seconds must be positive");
  if ((uint64_t)d->inflow_x0 + d->inflow_nx > s->dm.w || d->inflow_y >= s->dm.h || (uint64_t)d->inflow_z0 + d->inflow_nz > s->dm.d)
    return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_rollout_create: the inflow patch leaves the grid");
  auto r = new (std::nothrow) fx_rollout;
  if (!r) return fail(nullptr, FX_ERR_OUT_OF_MEMORY, "fx_rollout_create: host allocation failed");
  r->s = s;
  r->device = s->device;
  r->d = *d;
  r->patch = InflowPatch{d->inflow_x0, d->inflow_y, d->inflow_z0, d->inflow_nx, d->inflow_nz};
  r->n = s->n;
  r->npatch = d->inflow_nx * d->inflow_nz;
  r->nck = (d->steps + d->checkpoint_interval - 1) / d->checkpoint_interval;
  fx_status st = rollout_check(r);
  if (st != FX_OK) {
    delete r;
    return st;
  }
  const size_t n = r->n;
  const size_t n1 = count_of(s->lv[1].dm), n2 = count_of(s->lv[2].dm);
  const size_t ints = (size_t)r->npatch * 2 + 64;
  // floats: target, checkpoints, segment, final state, tape (11 n), adjoint (26 n), pressure adjoints
  const size_t floats = n + (size_t)r->nck * 7 * n + (size_t)d->checkpoint_interval * 7 * n + 7 * n + 11 * n + 26 * n +
                        3 * (n + n1 + n2) + ints;
  const size_t bytes = floats * sizeof(float) + 64 * 256 + sizeof(double) * 2;
  if (cudaSetDevice(s->device) != cudaSuccess || device_alloc(&r->arena, bytes) != cudaSuccess) {
    delete r;
    return fail(nullptr, FX_ERR_OUT_OF_MEMORY, "fx_rollout_create: device allocation of " + std::to_string(bytes) + " bytes failed");
  }
  char* p = static_cast<char*>(r->arena);
  auto take = [&](size_t count) {
    float* q = reinterpret_cast<float*>(p);
    p += (count * sizeof(float) + 255) / 256 * 256;
    return q;
  };
  r->loss = reinterpret_cast<double*>(take(4));
  r->inflow = take(r->npatch + 1);
  r->grad_inflow = take(r->npatch + 1);
  r->target = take(n);
  r->ck = take((size_t)r->nck * 7 * n);
  r->seg = take((size_t)d->checkpoint_interval * 7 * n);
  r->fin = take(7 * n);
  r->t1 = take(n);
  r->r1 = take(n);
  for (int k = 0; k < 3; ++k) {
    r->v1.c[k] = take(n);
    r->a.c[k] = take(n);
    r->b.c[k] = take(n);
  }
  for (int o = 0; o < 2; ++o) {
    for (int k = 0; k < 4; ++k) r->lam_s[o].f[k] = take(n);
    for (int k = 0; k < 3; ++k) r->lam_v[o].c[k] = take(n);
  }
  for (int k = 0; k < 3; ++k) {
    r->lam_c.c[k] = take(n);
    r->lam_w.c[k] = take(n);
    r->lam_g.c[k] = take(n);
  }
  r->lam_wmag = take(n);
  r->hot = take(n);
  r->dens = take(n);
  for (int l = 0; l < 3; ++l) {
    const size_t c = count_of(s->lv[l].dm);
    r->lam_p[l][0] = take(c);
    r->lam_p[l][1] = take(c);
    r->lam_div[l] = take(c);
  }
  if ((size_t)(p - static_cast<char*>(r->arena)) > bytes) {
    cudaFree(r->arena);
    delete r;
    return fail(nullptr, FX_ERR_STATE, "fx_rollout_create: internal layout error");
  }
  r->ck_host.resize(r->nck);
  r->seg_host.resize(d->checkpoint_interval);
  if (cudaMemsetAsync(r->arena, 0, bytes, s->stream) != cudaSuccess) {
    cudaFree(r->arena);
    delete r;
    return fail(nullptr, FX_ERR_CUDA, "fx_rollout_create: cudaMemsetAsync failed");
  }
  // The per-step tapes of a segment, when they take at most half of the free
  // device memory; without them the backward re-runs each step taped.
  const uint32_t nslots = std::min(d->checkpoint_interval, d->steps);
  const size_t sbytes = slot_bytes(n, s->nb) * nslots;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && sbytes <= free_b / 2) {
    if (device_alloc(&r->slot_arena, sbytes) == cudaSuccess) {
      carve_slots(r, static_cast<char*>(r->slot_arena), nslots);
    } else {
      r->slot_arena = nullptr;
      cudaGetLastError();  // a refused slot allocation is not an error of the rollout
    }
  }
  *out = r;
  return FX_OK;
}

// Touches only the rollout's own memory (cudaFree waits for the device), so it
// may run after the simulation was destroyed.
void fx_rollout_destroy(fx_rollout* r) {
  if (!r) return;
  cudaSetDevice(r->device);
  if (r->rp_exec) cudaGraphExecDestroy(r->rp_exec);
  for (cudaGraphExec_t ex : r->rs_exec)
    if (ex) cudaGraphExecDestroy(ex);
  if (r->slot_arena) cudaFree(r->slot_arena);
  if (r->arena) cudaFree(r->arena);
  delete r;
}

fx_status fx_rollout_set_target(fx_rollout* r, const float* target) {
  if (!r || !target) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_rollout_set_target: NULL argument");
  fx_sim* s = r->s;
  FX_CUDA(s, cudaSetDevice(s->device));
  FX_CUDA(s, cudaMemcpyAsync(r->target, target, r->n * sizeof(float), cudaMemcpyHostToDevice, s->stream));
  FX_CUDA(s, cudaStreamSynchronize(s->stream));
  r->have_target = true;
  return FX_OK;
}

fx_status fx_rollout_forward(fx_rollout* r, const float* inflow, double* loss) {
  if (!r || (!inflow && r->npatch) || !loss) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_rollout_forward: NULL argument");
  fx_sim* s = r->s;
  fx_status st = rollout_check(r);
  if (st != FX_OK) return st;
  if (!r->have_target) return fail(nullptr, FX_ERR_STATE, "fx_rollout_forward: no target (fx_rollout_set_target)");
  FX_CUDA(s, cudaSetDevice(s->device));
  r->forward_done = false;
  if (r->npatch)
    FX_CUDA(s, cudaMemcpyAsync(r->inflow, inflow, r->npatch * sizeof(float), cudaMemcpyHostToDevice, s->stream));
  r->fused_steps = s->kernels == FX_KERNELS_FUSED;
  const float lim = speed_limit_of(s);
  for (uint32_t k = 0; k < r->npatch; ++k)
    if (inflow[k] < -lim || inflow[k] > lim) r->fused_steps = false;
  PlainHooks hk;
  hk.inflow = r->npatch ? r->inflow : nullptr;
  hk.patch = r->patch;
  const uint32_t every = r->d.checkpoint_interval;
  for (uint32_t k = 0; k < r->d.steps; ++k) {
    if (k % every == 0 && save_state(r, r->ck + (size_t)(k / every) * 7 * r->n, r->ck_host[k / every]) != FX_OK) return FX_ERR_CUDA;
    st = rollout_step(r, k, hk);
    if (st != FX_OK) return st;
  }
  if (save_state(r, r->fin, r->fin_host) != FX_OK) return FX_ERR_CUDA;
  FX_CUDA(s, cudaMemsetAsync(r->loss, 0, sizeof(double), s->stream));
  adj_loss(s->stream, (uint32_t)r->n, s->sets[s->cur].f[0], r->target, nullptr, r->loss);
  FX_CUDA(s, cudaMemcpyAsync(loss, r->loss, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  FX_CUDA(s, cudaStreamSynchronize(s->stream));
  r->forward_done = true;
  return FX_OK;
}

// Test entry: 1 makes the rollout's taped re-runs use the plain step (the fused
// step records the same tape; the test compares the gradients of both), 0 the
// default.
fx_status fx_test_rollout_plain_tape(fx_rollout* r, int32_t on) {
  if (!r) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_test_rollout_plain_tape: NULL rollout");
  r->plain_tape = on != 0;
  return FX_OK;
}

// Test entry: 1 makes the backward re-run each step taped just before its
// adjoint instead of reading the tapes recorded while the segment was
// recomputed, 0 the default. *has_slots (optional) receives whether the
// recorded tapes were allocated.
fx_status fx_test_rollout_rerun_tape(fx_rollout* r, int32_t on, int32_t* has_slots) {
  if (!r) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_test_rollout_rerun_tape: NULL rollout");
  r->rerun_tape = on != 0;
  if (has_slots) *has_slots = r->slots.empty() ? 0 : 1;
  return FX_OK;
}

fx_status fx_rollout_backward(fx_rollout* r, float* grad_inflow, float* grad_velocity) {
  if (!r || (!grad_inflow && r->npatch)) return fail(nullptr, FX_ERR_INVALID_ARGUMENT, "fx_rollout_backward: NULL argument");
  fx_sim* s = r->s;
  if (!r->forward_done) return fail(nullptr, FX_ERR_STATE, "fx_rollout_backward: no forward to differentiate");
  fx_status st = rollout_check(r);
  if (st != FX_OK) return st;
  FX_CUDA(s, cudaSetDevice(s->device));
  cudaStream_t cs = s->stream;
  const size_t n = r->n;
  int o = 0;
  for (int k = 0; k < 4; ++k) FX_CUDA(s, cudaMemsetAsync(r->lam_s[0].f[k], 0, n * sizeof(float), cs));
  for (int k = 0; k < 3; ++k) FX_CUDA(s, cudaMemsetAsync(r->lam_v[0].c[k], 0, n * sizeof(float), cs));
  FX_CUDA(s, cudaMemsetAsync(r->grad_inflow, 0, (r->npatch + 1) * sizeof(float), cs));
  FX_CUDA(s, cudaMemsetAsync(r->hot, 0, n * sizeof(float), cs));
  FX_CUDA(s, cudaMemsetAsync(r->dens, 0, n * sizeof(float), cs));
  FX_CUDA(s, cudaMemsetAsync(r->loss + 1, 0, sizeof(double), cs));
  adj_loss(cs, (uint32_t)n, r->fin, r->target, r->lam_s[0].f[0], r->loss + 1);
  PlainHooks run;
  run.inflow = r->npatch ? r->inflow : nullptr;
  run.patch = r->patch;
  PlainHooks tape = run;
  tape.t1 = r->t1;
  tape.r1 = r->r1;
  tape.v1 = r->v1;
  tape.a = r->a;
  tape.b = r->b;
  const uint32_t every = r->d.checkpoint_interval;
  const bool slotted = !r->slots.empty() && !r->rerun_tape;
  for (int seg = (int)r->nck - 1; seg >= 0; --seg) {
    const uint32_t k0 = (uint32_t)seg * every, k1 = std::min(k0 + every, r->d.steps);
    if (restore_state(r, r->ck + (size_t)seg * 7 * n, r->ck_host[seg]) != FX_OK) return FX_ERR_CUDA;
    if (slotted) {
      // one taped pass over the segment records every step's tape
      for (uint32_t k = k0; k < k1; ++k) {
        if (save_state(r, r->seg + (size_t)(k - k0) * 7 * n, r->seg_host[k - k0]) != FX_OK) return FX_ERR_CUDA;
        StepTape& t = r->slots[k - k0];
        PlainHooks hk = run;
        hk.t1 = t.t1;
        hk.r1 = t.r1;
        hk.v1 = t.v1;
        hk.a = t.a;
        hk.b = t.b;
        const int cur = s->cur;
        if ((st = rollout_step(r, k, hk)) != FX_OK) return st;
        if ((st = record_tape(r, cur, t)) != FX_OK) return st;
      }
      for (int k = (int)k1 - 1; k >= (int)k0; --k) {
        if ((st = reverse_step_slot(r, k - k0, o)) != FX_OK) return st;
        o ^= 1;
      }
      continue;
    }
    for (uint32_t k = k0; k < k1; ++k) {
      if (save_state(r, r->seg + (size_t)(k - k0) * 7 * n, r->seg_host[k - k0]) != FX_OK) return FX_ERR_CUDA;
      if (k + 1 < k1 && (st = rollout_step(r, k, run)) != FX_OK) return st;
    }
    for (int k = (int)k1 - 1; k >= (int)k0; --k) {
      const float* state0 = r->seg + (size_t)(k - k0) * 7 * n;
      if (restore_state(r, state0, r->seg_host[k - k0]) != FX_OK) return FX_ERR_CUDA;
      const int cur = s->cur;
      if ((st = rollout_step(r, (uint32_t)k, tape)) != FX_OK) return st;
      if ((st = reverse_step(r, sim_tape(r, cur), state0, o)) != FX_OK) return st;
      o ^= 1;
    }
  }
  if (restore_state(r, r->fin, r->fin_host) != FX_OK) return FX_ERR_CUDA;
  if (r->npatch)
    FX_CUDA(s, cudaMemcpyAsync(grad_inflow, r->grad_inflow, r->npatch * sizeof(float), cudaMemcpyDeviceToHost, cs));
  if (grad_velocity)
    for (int k = 0; k < 3; ++k)
      FX_CUDA(s, cudaMemcpyAsync(grad_velocity + k * n, r->lam_v[o].c[k], n * sizeof(float), cudaMemcpyDeviceToHost, cs));
  FX_CUDA(s, cudaStreamSynchronize(cs));
  return FX_OK;
}

}  // extern "C"
