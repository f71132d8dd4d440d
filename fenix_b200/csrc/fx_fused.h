// The fused kernel path: the same step as the plain path with the same bits,
// computed by fewer, brick-list-driven kernels captured in a CUDA graph.
#pragma once

#include <cstdint>
#include <functional>
#include <map>
#include <string>
#include <vector>
#include <cuda.h>
#include <cuda_runtime.h>

#include "../../include/fenix_cuda.h"
#include "fx_kernels.h"
#include "fx_vcycle.h"

namespace fx {

struct FusedResult {
  int last_p = 0;
  bool final_vscr_is_2 = false;
  uint32_t launches = 0;
  bool graph = false;  // the step was a replay of a captured CUDA graph
  uint32_t cycle_launches = 0;  // kernels per V-cycle (not counted in `launches`, which covers the rest)
  std::string error;
};

// Device work buffers of the fused path, carved from the simulation's arena.
struct FusedWork {
  Dims dm{};
  uint3 bricks{};
  uint32_t nb = 0;
  // Per-brick energy summary of a scalar buffer at the reference's flag sample
  // points (bit 0: some sample above the activity threshold, bit 1: the brick
  // dilates), for the two scalar sets and the advected scratch set T.
  uint8_t* summary_set[2] = {nullptr, nullptr};
  uint8_t* summary_t = nullptr;
  // Bricks whose voxels may be non-zero, per scalar buffer.
  uint8_t* nz_set[2] = {nullptr, nullptr};
  uint8_t* nz_t = nullptr;
  // The current scalar set interleaved per voxel (d, t, f, r; 16 B in f32, 8 B in
  // binary16), rebuilt each step after the injection for the scalar advection's
  // gathers, and the bricks where that copy may be non-zero.
  void* aos = nullptr;
  uint8_t* nz_aos = nullptr;
  // Compacted brick lists.
  uint32_t* list_adv = nullptr;   // bricks the scalar advection kernel visits
  uint32_t* list_next = nullptr;  // bricks the combustion/buoyancy kernels visit
  uint32_t* list_inj = nullptr;   // bricks the injection kernel visits (host-filled)
  uint32_t* counters = nullptr;   // [0] adv count, [1] next count, [2] scratch, [3] inject count, [4..7] sparse lists
  // Sparse mode: per-brick "may be non-zero" bits of the velocity-side buffer
  // families (velocity scratch; curl, |curl| and the confined velocity; the fine
  // divergence and pressure; the velocity), the brick lists of the sparse
  // kernels, one per family, and whether the bits track the buffers (false
  // after a dense step or a host write: then every brick may be non-zero).
  uint8_t* nz_sp[4] = {nullptr, nullptr, nullptr, nullptr};
  uint32_t* list_sp[4] = {nullptr, nullptr, nullptr, nullptr};
  bool sp_known = true;
  // Tensor maps of the fine pressure buffers (16 x 10 x 10 boxes) and of the fine
  // divergence (8 x 8 x 8) for the TMA-staged sparse sweep; built on first use.
  CUtensorMap tmap_p[2]{};
  CUtensorMap tmap_div{};
  const float* tmap_base[3] = {nullptr, nullptr, nullptr};
  bool tmaps_ok = false;
  // Device error word: bit 0 is set when a bounded wait of a kernel ran out.
  uint32_t* dev_err = nullptr;
  SolverDev* solver = nullptr;     // FP64 solver statistics and the V-cycle loop state
  unsigned* vmax = nullptr;        // max |v| of the current velocity (float bits; all ones = unknown)
  cudaStream_t aux = nullptr;      // captures the V-cycle body graph
  cudaStream_t aux2 = nullptr;     // the mid and coarse pressure levels, beside the fine pre-sweeps
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  cudaStream_t aux3 = nullptr;     // the coarse level, beside the mid pre-sweeps on aux2
  cudaEvent_t fork2_ev = nullptr, join2_ev = nullptr;
  cudaEvent_t prep_fork_ev = nullptr, prep_join_ev = nullptr;  // the copy and flags beside the velocity advection
  int* host_cont = nullptr;        // pinned: the continue flag, read by the host loop without graphs
  uint32_t* host_list_inj = nullptr;  // pinned staging for list_inj (+ count at [nb])
  cudaEvent_t inj_event = nullptr;
  std::vector<uint8_t> host_mark;
  std::vector<uint32_t> host_list;
  bool valid = false;  // false: the per-brick bookkeeping must be rebuilt from the fields
  uint64_t tma_wait_ns = 1000000000ull;  // bound of a TMA tile wait (1 s; a tile takes microseconds)
  uint32_t tma_extra_tx = 0;
  std::vector<uint32_t> uploaded_list;  // injection list currently on the device
  // CUDA graphs of the device part of the step, keyed by its configuration.
  struct GraphEntry {
    cudaGraphExec_t exec;
    FusedResult result;
    bool taped;  // writes a rollout's tape (its key holds the tape's pointers)
  };
  bool use_graphs = true;
  std::string graph_note;
  std::map<uint64_t, GraphEntry> graphs;
  // kernel timing
  bool timing = false;
  struct TimedPair {
    const char* name;
    int a, b;
  };
  std::vector<cudaEvent_t> timing_events;
  std::vector<TimedPair> timing_pending;
  int timing_next = 0;
  int next_event();
};

// The brick-list kernels whose grid is tunable (fx_sim_autotune_bricks): each
// block walks the brick list with a stride of the grid, so any grid gives the
// same results. The grid is SMs x CTAs per SM, at most one block per brick.
enum BrickKernel {
  BK_INJECT, BK_ADVECT_SCALARS, BK_COMBUSTION, BK_BUOYANCY,
  BK_SP_ADVECT_VELOCITY, BK_SP_VORTICITY, BK_SP_CONFINEMENT, BK_SP_DIV_FIRST, BK_SP_SWEEP, BK_SP_PROLONG_FINE, BK_SP_PROJECT,
  kBrickKernels
};
constexpr int kBrickCtasDefault = 8;
constexpr int kBrickCtasMax = 64;

struct FusedStep {
  cudaStream_t stream;
  const float* inflow = nullptr;  // device values of the inflow patch (NULL: none)
  InflowPatch inflow_patch{};
  Dims dm;
  uint3 bricks;
  const Params* params;
  Params host_params;
  const float* sources;
  uint32_t nsrc;
  const float* host_sources;  // packed sources (NULL when none)
  uint32_t host_nsrc;
  int advect_mode;
  int cur_index;  // index of the current scalar set (0 or 1)
  ScalarSet cur, next, scratch;  // float* each, or binary16 buffers when half_storage
  bool half_storage;
  uint32_t *flags_cur, *flags_next;
  VelField vcur, vscr, vscr2, vort;
  float *vort_mag, *conf_mag, *vel_mag;
  LevelBuf lv[3];
  LevelBuf xlv[3];  // V-cycle levels 3..5
  int q[7];
  int sweep_variant[3];  // sweep kernel of the fine, mid and coarse level (-1 = default)
  uint8_t brick_ctas[kBrickKernels] = {};  // CTAs per SM of each brick kernel (0 = kBrickCtasDefault)
  int solver_mode;    // 0: the reference schedule, 1: the V-cycle
  VCycleConfig vc;
  bool solver_norms;  // FP64 statistics after the reference schedule too
  bool vort_on, pressure_on, debug_on, debug_fields;
  bool sparse = false;  // sparse mode (extension): velocity passes on the active bricks only
  // The differentiable rollout's tape (f32 storage, dense mode; all NULL otherwise):
  // temperature and reaction after the scalar injection and before the igniter,
  // and the velocity after the injection and inflow, after advection and after
  // buoyancy, as the plain step records them.
  float* tape_t1 = nullptr;
  float* tape_r1 = nullptr;
  VelField tape_v1{}, tape_a{}, tape_b{};
  int last_p;
};


// aos_voxel_bytes: bytes per voxel of the interleaved scalar copy (16 for f32
// storage, 8 for binary16).
size_t fused_work_bytes(Dims dm, uint3 bricks, size_t aos_voxel_bytes);
void fused_work_carve(FusedWork& w, char* base, Dims dm, uint3 bricks, size_t aos_voxel_bytes);
fx_status fused_init(FusedWork& w, cudaStream_t s);
fx_status fused_reset(FusedWork& w, cudaStream_t s);
fx_status fused_invalidate(FusedWork& w, cudaStream_t s);
void fused_release(FusedWork& w);
fx_status fused_step(FusedWork& w, const FusedStep& st, FusedResult& out);

// The parts of fused_step, for callers that build their own graphs (batches):
// host-side preparation on st.stream outside any graph (bookkeeping rebuild,
// injection-list upload; *ninj = bricks to inject), the configuration key of the
// device sequence, and the device sequence itself (capturable on st.stream).
fx_status fused_prepare(FusedWork& w, const FusedStep& st, uint32_t* ninj, FusedResult& out);
uint64_t fused_key(const FusedStep& st, uint32_t ninj);
fx_status fused_sequence(FusedWork& w, const FusedStep& st, uint32_t ninj, FusedResult& out);
fx_status fused_count_active(FusedWork& w, cudaStream_t s, const uint32_t* flags, uint32_t nb, uint32_t* out);
// FX_ERR_TIMEOUT when a bounded wait of a kernel ran out since the simulation
// was created (waits for the stream), FX_OK otherwise.
fx_status fused_check_device_error(FusedWork& w, cudaStream_t s);
// Test hook: the TMA-staged sweep's wait limit (ns) and the extra bytes its
// stages expect (0 in normal use; a non-zero value makes every wait run out).
void fused_set_tma_test(FusedWork& w, uint64_t wait_ns, uint32_t extra_tx);

// Adds the active bricks of `flags` and their voxel count to acc[0] and acc[1].
cudaError_t fused_accumulate_active(cudaStream_t s, Dims dm, uint3 bricks, const uint32_t* flags, unsigned long long* acc);

// Kernel timing of the fused path (events recorded inside its graphs).
void fused_set_timing(FusedWork& w, bool on);
void fused_drain_timing(FusedWork& w, const std::function<void(const char*, uint32_t, double)>& sink);

}  // namespace fx
