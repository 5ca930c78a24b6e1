// pf_noalloc.cu -- pf_project_noalloc: the pressure projection for callers
// that may not allocate device memory.
//
// Some hosts own every byte of device memory themselves: an application that
// reserves its whole budget up front and hands out sub-ranges from its own
// allocator, a plug-in loaded into such an application, or a fixed-rate loop
// that must not stall on the driver's allocator.  They can pass their own
// input and output buffers, but cannot let a library call cudaMalloc.  This
// entry point takes dense device arrays in and out and keeps every piece of
// working memory (tile tables, the eight pooled fields, the PCG vectors and
// reduction scratch) in one file-scope __device__ array of fixed size, so it
// calls no allocator at all.
//
// It runs pf_project's PLAIN set-up, Jacobi-PCG recurrences and velocity
// update (the launchers in pf_project.cu and pf_pcg.cu) on a pool in which
// every tile is active.  Its SpMV finds cross-tile neighbours through the tile
// map in shared memory (k_spmv_plain); pf_project's PLAIN solve reads them
// from a per-solve neighbour-slot table (k_spmv_plain_tab), which would need
// memory this entry point does not have.  Both give the same rows.
#include <cmath>
#include <cstring>

#include "pf_ctx.h"
#include "pf_solver.cuh"

namespace pf {
void launch_project_setup(const DevGrid& G, int nslots, int nred, SolveCtl* ctl, uint8_t* kind,
                          PcgVec<double> vec, double scale, double cdiv, const pf_phase* ph, double* partials,
                          cudaStream_t s);
void launch_project_finish(const DevGrid& G, int nslots, int nred, const uint8_t* kind, const double* x,
                           double dt_over_dx, const pf_phase* ph, cudaStream_t s);
void launch_pcg_plain_iteration(const DevGrid& G, int nslots, int nred, SolveCtl* ctl, const uint8_t* kind,
                                PcgVec<double> v, double scale, double* partials, cudaStream_t s);
}  // namespace pf

using namespace pf;

namespace {

// Capacity: 125 tiles of 8^3 cells, e.g. up to 39^3 cells (a tile lattice of
// ceil((n+1)/8) per axis must multiply to at most 125).
constexpr int kMaxTiles = PF_NOALLOC_MAX_TILES;
constexpr size_t kCells = (size_t)kMaxTiles * PF_TV;
constexpr size_t kAct4 = 8 * (size_t)kMaxTiles;  // 4^3 blocks per field: at most 2x2x2 per tile

constexpr size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

// byte offsets of the parts of the scratch array
constexpr size_t kOffTileSlot = 0;
constexpr size_t kOffSlotTile = align256(kOffTileSlot + kMaxTiles * sizeof(int));
constexpr size_t kOffFields = align256(kOffSlotTile + kMaxTiles * sizeof(int));
constexpr size_t kOffAct4 = align256(kOffFields + PF_NFIELDS * kCells * sizeof(float));
constexpr size_t kOffKind = align256(kOffAct4 + PF_NFIELDS * kAct4);
constexpr size_t kOffVec = align256(kOffKind + kCells);
constexpr size_t kOffPartials = align256(kOffVec + 8 * kCells * sizeof(double));
constexpr size_t kOffCtl = align256(kOffPartials + (size_t)kMaxRedBlocks * 3 * sizeof(double));
constexpr size_t kScratchBytes = align256(kOffCtl + sizeof(SolveCtl));

// The scratch array: every GPU that loads the library holds it until exit.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch in the context current on the calling
// thread (the host-side name is not a device address).  It is looked up on
// every call, not cached: the address belongs to a context, and between two
// calls the caller may have reset the device or made another context of its
// own current.  Once the library's module is loaded in that context the
// lookup allocates nothing.
int scratch_base(unsigned char** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p) return PF_ERR_CUDA;
  *out = (unsigned char*)p;
  return PF_OK;
}

Geom make_geom(int nx, int ny, int nz, double dx) {
  Geom g{};
  g.nx = nx; g.ny = ny; g.nz = nz;
  g.dx = dx; g.inv_dx = 1.0 / dx;
  {
    int e = 0;
    g.dx_pow2 = std::frexp(dx, &e) == 0.5 ? 1 : 0;
  }
  g.TX = (nx + 1 + 7) / 8; g.TY = (ny + 1 + 7) / 8; g.TZ = (nz + 1 + 7) / 8;
  g.ntiles = g.TX * g.TY * g.TZ;
  const int dims[PF_NFIELDS][3] = {{nx + 1, ny, nz}, {nx, ny + 1, nz}, {nx, ny, nz + 1}, {nx + 1, ny, nz},
                                   {nx, ny + 1, nz}, {nx, ny, nz + 1}, {nx, ny, nz},     {nx, ny, nz}};
  for (int f = 0; f < PF_NFIELDS; ++f)
    for (int a = 0; a < 3; ++a) {
      g.fdim[f][a] = dims[f][a];
      g.bdim[f][a] = (dims[f][a] + 3) / 4;
    }
  return g;
}

struct DenseIn {
  const float* f[PF_NFIELDS];  // u, v, w, mu, mv, mw, (p unused), mk
};

// Dense caller arrays -> every tile of the pool (identity tile->slot map).
__global__ void k_na_pack(DevGrid G, int* tile_slot, int* slot_tile, DenseIn in) {
  const int t = blockIdx.x, l = threadIdx.x;
  if (l == 0) {
    tile_slot[t] = t;
    slot_tile[t] = t;
  }
  const int tx = t % G.g.TX, q = t / G.g.TX, ty = q % G.g.TY, tz = q / G.g.TY;
  const int i = tx * 8 + (l & 7), j = ty * 8 + ((l >> 3) & 7), k = tz * 8 + (l >> 6);
  const size_t o = (size_t)t * PF_TV + l;
#pragma unroll
  for (int f = 0; f < PF_NFIELDS; ++f) {
    float v = 0.0f;
    if (f != PF_P && in_field(G.g, f, i, j, k))
      v = in.f[f][(size_t)i + (size_t)G.g.fdim[f][0] * ((size_t)j + (size_t)G.g.fdim[f][1] * k)];
    G.fld[f][o] = v;
  }
}

// Pool -> the caller's dense p, u, v, w.
__global__ void k_na_unpack(DevGrid G, float* p, float* u, float* v, float* w) {
  const int t = blockIdx.x, l = threadIdx.x;
  const int tx = t % G.g.TX, q = t / G.g.TX, ty = q % G.g.TY, tz = q / G.g.TY;
  const int i = tx * 8 + (l & 7), j = ty * 8 + ((l >> 3) & 7), k = tz * 8 + (l >> 6);
  const size_t o = (size_t)t * PF_TV + l;
  float* out[4] = {u, v, w, p};
  const int fs[4] = {PF_U, PF_V, PF_W, PF_P};
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int f = fs[a];
    if (in_field(G.g, f, i, j, k))
      out[a][(size_t)i + (size_t)G.g.fdim[f][0] * ((size_t)j + (size_t)G.g.fdim[f][1] * k)] = G.fld[f][o];
  }
}

}  // namespace

extern "C" int pf_project_noalloc(int nx, int ny, int nz, double dx, const float* mk, const float* mu,
                                  const float* mv, const float* mw, float* u, float* v, float* w, float* p,
                                  const pf_phase* phase, double dt, int max_iter, double abs_tol, double rel_tol,
                                  double c_div, pf_solve_stats* stats, void* stream) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || !(dx > 0.0) || !phase || !mk || !mu || !mv || !mw || !u || !v || !w ||
      !p || max_iter < 0 || !(abs_tol >= 0.0) || !(rel_tol >= 0.0))
    return PF_ERR_INVALID;
  const Geom g = make_geom(nx, ny, nz, dx);
  if (g.ntiles > kMaxTiles) return PF_ERR_INVALID;  // beyond the fixed scratch capacity
  unsigned char* base = nullptr;
  int rc = scratch_base(&base);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;

  int* tile_slot = (int*)(base + kOffTileSlot);
  int* slot_tile = (int*)(base + kOffSlotTile);
  DevGrid G{};
  G.g = g;
  G.tile_slot = tile_slot;
  G.slot_tile = slot_tile;
  for (int f = 0; f < PF_NFIELDS; ++f) {
    G.fld[f] = (float*)(base + kOffFields) + (size_t)f * kCells;
    G.act4[f] = base + kOffAct4 + (size_t)f * kAct4;
  }
  uint8_t* kind = base + kOffKind;
  double* vb = (double*)(base + kOffVec);
  PcgVec<double> vec{vb, vb + kCells, vb + 2 * kCells, vb + 3 * kCells,
                     vb + 4 * kCells, vb + 5 * kCells, vb + 6 * kCells, vb + 7 * kCells};
  double* partials = (double*)(base + kOffPartials);
  SolveCtl* ctl = (SolveCtl*)(base + kOffCtl);

  // every block of every field is active in a dense grid
  for (int f = 0; f < PF_NFIELDS; ++f) {
    const size_t nb = (size_t)g.bdim[f][0] * g.bdim[f][1] * g.bdim[f][2];
    if (cudaMemsetAsync(G.act4[f], 1, nb, s) != cudaSuccess) return PF_ERR_CUDA;
  }
  DenseIn in{};
  in.f[PF_U] = u; in.f[PF_V] = v; in.f[PF_W] = w;
  in.f[PF_MU] = mu; in.f[PF_MV] = mv; in.f[PF_MW] = mw;
  in.f[PF_MK] = mk; in.f[PF_P] = nullptr;
  k_na_pack<<<g.ntiles, PF_TV, 0, s>>>(G, tile_slot, slot_tile, in);

  SolveCtl init{};
  init.min_fluid = 0x7fffffff;
  init.pin = -1;
  init.max_iter = max_iter;
  init.tol_abs = abs_tol;
  init.tol_rel = rel_tol;
  if (cudaMemcpyAsync(ctl, &init, sizeof(SolveCtl), cudaMemcpyHostToDevice, s) != cudaSuccess) return PF_ERR_CUDA;

  const int nslots = g.ntiles;
  const int nred = nslots < kMaxRedBlocks ? nslots : kMaxRedBlocks;
  const double scale = dt / (dx * dx);
  launch_project_setup(G, nslots, nred, ctl, kind, vec, scale, c_div, phase, partials, s);
  if (cudaGetLastError() != cudaSuccess) return PF_ERR_CUDA;

  SolveCtl c{};
  if (cudaMemcpyAsync(&c, ctl, sizeof(SolveCtl), cudaMemcpyDeviceToHost, s) != cudaSuccess) return PF_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return PF_ERR_CUDA;
  const double res0 = c.res0, tol = c.tol;
  int launched = 0, batch = 4;
  while (!c.done && launched < max_iter) {
    const int nb = batch < max_iter - launched ? batch : max_iter - launched;
    for (int q = 0; q < nb; ++q) launch_pcg_plain_iteration(G, nslots, nred, ctl, kind, vec, scale, partials, s);
    if (cudaGetLastError() != cudaSuccess) return PF_ERR_CUDA;
    launched += nb;
    if (cudaMemcpyAsync(&c, ctl, sizeof(SolveCtl), cudaMemcpyDeviceToHost, s) != cudaSuccess) return PF_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PF_ERR_CUDA;
    batch = batch * 2 < 64 ? batch * 2 : 64;
  }
  launch_project_finish(G, nslots, nred, kind, vec.x, dt / dx, phase, s);
  k_na_unpack<<<g.ntiles, PF_TV, 0, s>>>(G, p, u, v, w);
  if (cudaGetLastError() != cudaSuccess) return PF_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return PF_ERR_CUDA;
  if (stats) {
    pf_solve_stats st{};
    st.iterations = c.it;
    st.n_cells = c.n_cells;
    st.pin_cell = c.pin;
    st.res0 = res0;
    st.res_final = c.it > 0 ? c.res : res0;
    st.tol_effective = tol;
    st.converged = c.done == 1;
    st.breakdown = c.done == 2;
    *stats = st;
  }
  return c.done == 4 ? PF_ERR_NONFINITE : PF_OK;
}
