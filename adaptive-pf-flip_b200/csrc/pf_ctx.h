// pf_ctx.h -- host-side context of libpfgpu (one grid + one particle set on
// one device).  Internal: the public ABI is include/pfgpu.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "pf_internal.cuh"

struct pf_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  pf::Geom g{};

  // ---- tile pool ----
  int* tile_slot = nullptr;   // [ntiles] dense block-pointer array
  int* slot_tile = nullptr;   // [ntiles] slot -> tile
  int nslots = 0;             // host copy of the pool size
  int* d_nslots = nullptr;    // device copy
  // The pool grows without a host round trip: pool_commit leaves the new size
  // on the device (slot loops read d_nslots, their grids are sized to
  // capacity) and copies it to h_nslots behind pool_ev; pool_sync waits for
  // that copy before the host uses nslots again.
  bool pool_pending = false;
  int* h_nslots = nullptr;    // pinned
  cudaEvent_t pool_ev = nullptr;
  uint8_t* tile_need = nullptr;  // [ntiles] activation requests
  int* tile_new = nullptr;       // [ntiles] scratch for slot assignment
  int* tile_rank = nullptr;      // [ntiles] scratch for slot assignment
  float* fld[PF_NFIELDS] = {};
  float* saved[PF_NSAVED] = {};
  uint8_t* act4[PF_NFIELDS] = {};
  size_t act4_n[PF_NFIELDS] = {};
  // first-touch key of each 4^3 marker block: the position, in the reference's
  // markCells order (wall loops, then particles), of the write that activated it
  uint32_t* mk_first = nullptr;
  void* rc_buf = nullptr;  // render-cache export scratch, grown on demand
  size_t rc_bytes = 0;
  std::vector<int> wall_tiles;  // tiles written by markCells walls / applyWallBoundary
  int* d_wall_tiles = nullptr;
  bool saved_valid = false;
  bool bins_valid = false;  // tile_start/perm bin the current particle positions (set by P2G)

  // ---- particles (SoA FP32) ----
  size_t cap = 0, np = 0;
  float *px = nullptr, *py = nullptr, *pz = nullptr;
  float *vx = nullptr, *vy = nullptr, *vz = nullptr;
  float* vol = nullptr;
  uint8_t* type = nullptr;
  void* staging = nullptr;  // upload/download staging (cap * 3 doubles)
  size_t staging_bytes = 0;
  // asynchronous downloads: two device staging slots, copied to the host on copy_stream
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t dl_packed[2] = {}, dl_copied[2] = {};
  bool dl_recorded[2] = {};
  void* dl_staging[2] = {};
  size_t dl_bytes = 0;
  int dl_slot = 0;
  int dl_last = -1;  // slot of the most recent asynchronous download
  // asynchronous uploads: a second particle set filled on up_stream and swapped
  // in by the next call that uses the particles (take_upload)
  cudaStream_t up_stream = nullptr;
  cudaEvent_t up_done = nullptr, back_free = nullptr;
  bool back_free_recorded = false, up_pending = false;
  float *bpx = nullptr, *bpy = nullptr, *bpz = nullptr, *bvx = nullptr, *bvy = nullptr, *bvz = nullptr;
  float* bvol = nullptr;
  uint8_t* btype = nullptr;
  float* up_staging = nullptr;  // pos and vel, n x 3 each, as uploaded
  size_t np_next = 0;

  // ---- binning ----
  int* tile_count = nullptr;  // [ntiles+1]
  int* tile_start = nullptr;  // [ntiles+1]
  int* pkey = nullptr;        // [cap]
  int* prank = nullptr;       // [cap]
  int* perm = nullptr;        // [cap]
  float2* splat_stage = nullptr;  // [ntiles * kSplatStageTile] per-tile P2G staging boxes (momentum, raw mass)
  bool splat_fresh = false;       // splat_stage holds the last P2G's boxes, not yet normalised

  // ---- scan scratch ----
  std::vector<int*> scan_levels;
  int* d_scalar = nullptr;  // small device scratch (ints)

  // ---- projection / PCG (pool layout, cap slots * 512) ----
  size_t cells_cap = 0;
  double *x = nullptr, *r = nullptr, *p = nullptr, *Ap = nullptr;
  double *diag = nullptr, *cx = nullptr, *cy = nullptr, *cz = nullptr;
  double* partials = nullptr;  // [kMaxRedBlocks * 4]
  int* nbr_plain = nullptr;    // [cells_cap / 512 * 6] neighbour slots of each pooled tile (PLAIN PCG)
  double* z_plain = nullptr;   // [cells_cap] PLAIN PCG's z (r / diag), from its update to its direction pass
  uint8_t* kind = nullptr;     // per cell: 0 not an unknown, 1 fluid, 2 pinned
  pf::SolveCtl* ctl = nullptr;
  pf::SolveCtl* h_ctl = nullptr;  // pinned mirror
  pf::SolveCtl* ctl_outer = nullptr;  // outer iteration of the inner-outer solves
  // mixed precision
  float *xf = nullptr, *rf = nullptr, *pf32 = nullptr, *Apf = nullptr;
  float *diagf = nullptr, *cxf = nullptr, *cyf = nullptr, *czf = nullptr;
  uint16_t *pbf = nullptr, *cbf = nullptr;  // bf16 direction / coefficients (3 per cell)
  double* b64 = nullptr;  // right-hand side kept in FP64
  // learned preconditioner state lives in its own module
  void* learned = nullptr;
  // the 2-level multires grid (pf_mr.cu), made on first use
  void* mr = nullptr;
  // the secondary droplet and bubble sets (pf_secondary.cu), made on first use
  void* secondary = nullptr;
  // particle adaptivity: scratch (its own module) and the step's settings
  void* adapt = nullptr;
  bool adapt_on = false;
  pf_adapt_cfg adapt_cfg{};
  pf_adapt_stats adapt_last{};
  // interface diagnostics: scratch (its own module) and the last result
  void* idiag = nullptr;
  pf_interface_stats diag_last{};
  // the step's adaptive timestep and volume correction
  pf_step_controls controls{0, 0.5, 1e-5, 0, 1.0, 0.0};
  pf_step_control_stats controls_last{};
  // surface tension in the step (strength 0: off) and its last statistics
  double st_strength = 0.0, st_max_dv = 0.0;
  int st_radius = 0;
  pf_surface_stats surface_last{};

  // ---- misc ----
  int* d_clamp = nullptr;      // 8 counters
  int* d_flags = nullptr;      // escape flags / scratch [cap]
  void* esc_buf = nullptr;     // escape records, grown on demand
  size_t esc_bytes = 0;
  int* h_pinned_ints = nullptr;
  int32_t* cell_flags = nullptr;  // dense nx*ny*nz scratch for compaction
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;

  long long launches = 0;  // kernels launched by this context

  // ---- optional per-stage timing ----
  bool timing_on = false;
  cudaEvent_t open_ev[PF_NSTAGES] = {};  // start event of each open stage
  struct TimedStage { int stage; cudaEvent_t a, b; };
  std::vector<TimedStage> timed;
  double acc_ms[PF_NSTAGES] = {};
  long long acc_n[PF_NSTAGES] = {};
};

namespace pf {

int set_cuda_error(pf_ctx* ctx, cudaError_t e, const char* what, const char* file, int line);
int set_error(pf_ctx* ctx, int code, const std::string& msg);

// launch helpers
inline int nblocks(size_t n, int nt) { return (int)((n + (size_t)nt - 1) / (size_t)nt); }

// scan.cu
int scan_exclusive(pf_ctx* ctx, const int* in, int* out, int n, int* total_dev);
int scan_alloc(pf_ctx* ctx, size_t max_n);

// pool.cu
int pool_reset(pf_ctx* ctx);
int pool_commit(pf_ctx* ctx);  // give slots to requested tiles; the new size stays on the device
int pool_sync(pf_ctx* ctx);    // wait for a deferred nslots read-back
int slot_blocks(const pf_ctx* ctx, int cap);  // grid for a slot loop reading d_nslots
int field_clear(pf_ctx* ctx, int f, bool data = true);
int request_wall_tiles(pf_ctx* ctx);
DevGrid dev_grid(const pf_ctx* ctx);
int grid_set_field(pf_ctx* ctx, int f, const float* dense, const uint8_t* act4);
int grid_get_field(pf_ctx* ctx, int f, float* dense, uint8_t* act4);
int active_blocks4(pf_ctx* ctx, int f, int32_t* ids, size_t* n);
int active_cells(pf_ctx* ctx, int32_t* cells, size_t* n);

// transfer.cu
int mark_cells(pf_ctx* ctx);
int p2g(pf_ctx* ctx, const pf_phase* ph, double Vp);
int save_velocity(pf_ctx* ctx);
int apply_gravity(pf_ctx* ctx, double dt, double gravity);
int apply_walls(pf_ctx* ctx);
int normalize_save_gravity(pf_ctx* ctx, bool save, bool gravity, double dt, double gval);
int g2p(pf_ctx* ctx, const pf_ctx* saved, double aL, double aG);
int advect(pf_ctx* ctx, double dt, int order, pf_clamp_stats* st, double* esc, size_t* nesc);
int g2p_advect(pf_ctx* ctx, double aL, double aG, double dt, int order, pf_clamp_stats* st,
               int* esc_flags = nullptr);
int calibrate(pf_ctx* ctx, const pf_phase* ph, double Vp, double* out);

// project.cu
int project(pf_ctx* ctx, const pf_phase* ph, double dt, const pf_solve_cfg* cfg,
            pf_solve_stats* st);

// adapt.cu
int narrow_band_air(pf_ctx* ctx, int radius, pf_band_stats* st);
int coarsen_particles(pf_ctx* ctx, int ptype, int target, unsigned seed, pf_coarsen_stats* st);
int refill_liquid(pf_ctx* ctx, int target, unsigned seed, int interface_only, int interface_radius, int max_added,
                  pf_refill_stats* st);
int apply_adaptivity(pf_ctx* ctx, const pf_adapt_cfg& cfg, pf_adapt_stats* st);
int step_controls(pf_ctx* ctx, double dt, double Vp, const pf_step_controls& c, pf_step_control_stats* st,
                  bool wait = true);
int step_controls_finish(pf_ctx* ctx, pf_step_control_stats* st);  // statistics of a wait == false launch
void adapt_free(pf_ctx* ctx);

// diag.cu
int interface_diagnostics(pf_ctx* ctx, const pf_phase* ph, pf_interface_stats* st, bool wait = true);
int interface_diagnostics_finish(pf_ctx* ctx);  // statistics of a launch made with wait == false
int surface_tension(pf_ctx* ctx, const pf_phase* ph, double dt, double strength, double max_dv, int radius,
                    pf_surface_stats* st);
void diag_free(pf_ctx* ctx);

// mr.cu
void mr_free(pf_ctx* ctx);

// secondary.cu
bool secondary_active(const pf_ctx* ctx);
bool secondary_reabsorbs(const pf_ctx* ctx);
int* secondary_escape_flags(pf_ctx* ctx);
int secondary_lifecycle(pf_ctx* ctx, double dt, double gravity, double Vp);
int secondary_after_advect(pf_ctx* ctx, const int* esc_flags, double Vp, const pf_interface_stats& iface);
void secondary_free(pf_ctx* ctx);

// capi.cu: the second particle set (asynchronous uploads, compaction target)
int ensure_back_set(pf_ctx* ctx);

// P2G staging box of one tile: per face field the nodes its cells reach,
// 11 along the normal axis and 10 along each transverse axis (float2 each).
constexpr int kSplatStageTile = 3 * 11 * 10 * 10;

constexpr int kMaxRedBlocks = 1184;  // 8 CTAs per SM on 148 SMs
constexpr int kRedSlots = 4;         // partial values one reduction CTA may write

// pf_timing.cu
using TimedStage = pf_ctx::TimedStage;
void stage_begin(pf_ctx* ctx, int stage);
void stage_end(pf_ctx* ctx, int stage);
int get_timing(pf_ctx* ctx, pf_timing* out, int reset);

struct StageScope {
  pf_ctx* c;
  int s;
  StageScope(pf_ctx* ctx, int stage) : c(ctx), s(stage) { stage_begin(c, s); }
  ~StageScope() { stage_end(c, s); }
};

}  // namespace pf
