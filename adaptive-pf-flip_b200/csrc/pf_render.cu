// Render-cache export: writeSparseRenderCache3D (src/driver/render_cache3d.h:551-600)
// from the device pool.
//
// The phase-field section is the expensive part: every cell of every active
// 4^3 marker block (or pressure block, when no marker block is active) with
// marker != 0 or phi > 1e-8, phi being the mean of the cell's six faces'
// phi(raw mass) (sparseCellPhi, :327-340).  Two kernels over the 4^3 blocks
// (count, then an order-preserving write after an exclusive scan of the
// counts) produce the compacted cell records on the device; only the kept
// cells cross PCIe.  The JSONL text is formatted on the host with the same
// std::ostream settings (setprecision(17)) as the reference, so every line it
// writes is byte-identical for the same state.
//
// Block order: the reference lists cells block by block in the order its
// marker blocks were first activated (activeBlockIds: markCells' wall loops,
// then the particles in index order), cells within a block in lz, ly, lx
// order.  markCells here keeps each marker block's first-touch key (its
// position in that sequence; ascending block id for an imported marker
// field), and the blocks are listed sorted by it, so the file lists the cells
// in the reference's order and sums the liquid volume in that order too.
// With no marker block active the pressure blocks are listed in ascending
// block id.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <limits>
#include <string>
#include <vector>

#include "pf_ctx.h"

namespace pf {
namespace {

struct RcPhiK {
  double rmin, den;
};

struct RcCell {
  int i, j, k, marker;
  double phi;
};

// phiFromRawDensity (src/physics/phasefield.h:11-16)
__device__ __forceinline__ double rc_phi_of_raw(double raw, const RcPhiK& P) {
  if (raw < P.rmin) return 0.0;
  double e = __dsub_rn(raw, P.rmin);
  if (e < 0.0) e = 0.0;
  const double v = sqrt(__ddiv_rn(e, P.den));
  return 1.0 < v ? 1.0 : v;
}

// Cell t (lx fastest) of 4^3 block b: kept when the block is active in field
// fsel, the cell is inside the grid and marker != 0 or phi > 1e-8
// (sparsePhaseCells, render_cache3d.h:497-526).
__device__ __forceinline__ bool rc_cell(const DevGrid& G, const RcPhiK& P, int fsel, int b, int t, RcCell* c) {
  const Geom& g = G.g;
  const int nbx = g.bdim[PF_MK][0], nby = g.bdim[PF_MK][1];
  if (!G.act4[fsel][b]) return false;
  const int bx = b % nbx, by = (b / nbx) % nby, bz = b / (nbx * nby);
  const int i = bx * 4 + (t & 3), j = by * 4 + ((t >> 2) & 3), k = bz * 4 + (t >> 4);
  if (!in_cells(g, i, j, k)) return false;
  const int marker = cell_marker(G, i, j, k);
  double s = 0.0;
  s = __dadd_rn(s, rc_phi_of_raw((double)fget(G, PF_MU, i, j, k), P));
  s = __dadd_rn(s, rc_phi_of_raw((double)fget(G, PF_MU, i + 1, j, k), P));
  s = __dadd_rn(s, rc_phi_of_raw((double)fget(G, PF_MV, i, j, k), P));
  s = __dadd_rn(s, rc_phi_of_raw((double)fget(G, PF_MV, i, j + 1, k), P));
  s = __dadd_rn(s, rc_phi_of_raw((double)fget(G, PF_MW, i, j, k), P));
  s = __dadd_rn(s, rc_phi_of_raw((double)fget(G, PF_MW, i, j, k + 1), P));
  const double phi = __ddiv_rn(s, 6.0);
  if (marker == 0 && phi <= 1e-8) return false;
  *c = RcCell{i, j, k, marker, phi};
  return true;
}

// The active blocks of field fsel, each with its listing key (the marker
// field's first-touch key, or the block id), compacted in any order: the sort
// that follows fixes it.
__global__ void k_rc_list(const uint8_t* act, const uint32_t* first, int nb4, int* nlist, uint32_t* key, int* list) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb4 || !act[b]) return;
  const int q = atomicAdd(nlist, 1);
  key[q] = first ? first[b] : (uint32_t)b;
  list[q] = b;
}

// One 64-thread CTA per listed block (grid-stride): its kept-cell count.
__global__ void __launch_bounds__(64) k_rc_count(DevGrid G, RcPhiK P, int fsel, const int* list, int n, int* cnt) {
  for (int q = blockIdx.x; q < n; q += gridDim.x) {
    RcCell c;
    const int keep = rc_cell(G, P, fsel, list[q], threadIdx.x, &c) ? 1 : 0;
    const int k = __syncthreads_count(keep);
    if (threadIdx.x == 0) cnt[q] = k;
  }
}

// Same walk; each kept cell goes to off[q] + its rank among the block's kept
// cells in lz, ly, lx order.
__global__ void __launch_bounds__(64) k_rc_write(DevGrid G, RcPhiK P, int fsel, const int* list, int n,
                                                 const int* off, RcCell* out) {
  __shared__ unsigned w0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int q = blockIdx.x; q < n; q += gridDim.x) {
    RcCell c;
    const bool keep = rc_cell(G, P, fsel, list[q], threadIdx.x, &c);
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (threadIdx.x == 0) w0 = m;
    __syncthreads();
    const int base = warp ? __popc(w0) : 0;
    if (keep) out[off[q] + base + __popc(m & ((1u << lane) - 1u))] = c;
    __syncthreads();
  }
}

struct Bounds {
  double mn[3], mx[3];
  bool valid = false;
};

void include_point(Bounds& b, const double p[3]) {
  if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) return;
  if (!b.valid) {
    for (int a = 0; a < 3; ++a) b.mn[a] = b.mx[a] = p[a];
    b.valid = true;
    return;
  }
  for (int a = 0; a < 3; ++a) {
    b.mn[a] = std::min(b.mn[a], p[a]);
    b.mx[a] = std::max(b.mx[a], p[a]);
  }
}

void write_vec(std::ostream& out, const char* key, const double v[3]) {
  out << "\"" << key << "\":[" << v[0] << "," << v[1] << "," << v[2] << "]";
}

void write_bounds(std::ostream& out, const char* kmin, const char* kmax, const Bounds& b, const Bounds& fb) {
  const Bounds& u = b.valid ? b : fb;
  write_vec(out, kmin, u.mn);
  out << ",";
  write_vec(out, kmax, u.mx);
}

bool finite3(const double v[3]) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }

// A JSON string literal with the escapes of writeJsonString
// (src/driver/render_cache3d.h:121-146): quote, backslash and the named
// control characters by their short escapes, other bytes below 0x20 as
// \u00XX, everything else verbatim.
void write_json_string(std::ostream& out, const char* s) {
  static const char digits[] = "0123456789abcdef";
  out << '"';
  for (const unsigned char* p = (const unsigned char*)s; *p; ++p) {
    const unsigned char c = *p;
    if (c == '"') out << "\\\"";
    else if (c == '\\') out << "\\\\";
    else if (c == '\b') out << "\\b";
    else if (c == '\f') out << "\\f";
    else if (c == '\n') out << "\\n";
    else if (c == '\r') out << "\\r";
    else if (c == '\t') out << "\\t";
    else if (c < 0x20) out << "\\u00" << digits[c >> 4] << digits[c & 15];
    else out << (char)c;
  }
  out << '"';
}

}  // namespace

// The export's device scratch, kept by the context and grown on demand.
static int rc_scratch(pf_ctx* ctx, size_t bytes, char** out) {
  if (bytes > ctx->rc_bytes) {
    if (ctx->rc_buf) PF_CUDA_TRY(cudaFree(ctx->rc_buf));
    ctx->rc_buf = nullptr;
    ctx->rc_bytes = 0;
    PF_CUDA_TRY(cudaMalloc(&ctx->rc_buf, bytes));
    ctx->rc_bytes = bytes;
  }
  *out = (char*)ctx->rc_buf;
  return PF_OK;
}

static size_t align_up(size_t v) { return (v + 255) & ~(size_t)255; }

// Kept phase cells of the current grid, compacted on the device in the
// reference's block order.
int render_cells(pf_ctx* ctx, const pf_phase* ph, std::vector<RcCell>* cells) {
  const Geom& g = ctx->g;
  const int nb4 = g.bdim[PF_MK][0] * g.bdim[PF_MK][1] * g.bdim[PF_MK][2];
  RcPhiK P;
  P.rmin = std::log(ph->rho_l / ph->rho_g) * ph->rho_g * ph->rho_tilde_0;
  P.den = ph->alpha_phi * ph->rho_tilde_0 * ph->rho_l;
  const DevGrid G = dev_grid(ctx);
  // scratch: keys and lists (unsorted, sorted), counts, offsets, list size,
  // then the cub temporary storage of the sort and the scan
  size_t sort_tmp = 0, scan_tmp = 0;
  PF_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_tmp, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                              (int*)nullptr, (int*)nullptr, nb4, 0, 32, ctx->stream));
  PF_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_tmp, (int*)nullptr, (int*)nullptr, nb4 + 1, ctx->stream));
  const size_t n4 = align_up((size_t)(nb4 + 1) * 4);
  const size_t tmp_bytes = align_up(std::max(sort_tmp, scan_tmp));
  const size_t fixed = 6 * n4 + 256 + tmp_bytes;
  char* buf = nullptr;
  int rc = rc_scratch(ctx, fixed, &buf);
  if (rc) return rc;
  uint32_t* key_in = (uint32_t*)buf;
  uint32_t* key = (uint32_t*)(buf + n4);
  int* list_in = (int*)(buf + 2 * n4);
  int* list = (int*)(buf + 3 * n4);
  int* cnt = (int*)(buf + 4 * n4);
  int* off = (int*)(buf + 5 * n4);
  int* nlist = (int*)(buf + 6 * n4);
  void* tmp = buf + 6 * n4 + 256;
  // activeBlockIds of mkf, or of pf when no marker block is active
  int n = 0, fsel = PF_MK;
  for (int pass = 0; pass < 2; ++pass) {
    PF_CUDA_TRY(cudaMemsetAsync(nlist, 0, sizeof(int), ctx->stream));
    (++ctx->launches), k_rc_list<<<nblocks(nb4, 256), 256, 0, ctx->stream>>>(
        ctx->act4[fsel], fsel == PF_MK ? ctx->mk_first : nullptr, nb4, nlist, key_in, list_in);
    PF_CUDA_TRY(cudaGetLastError());
    PF_CUDA_TRY(cudaMemcpyAsync(ctx->h_pinned_ints, nlist, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    n = ctx->h_pinned_ints[0];
    if (n > 0 || fsel == PF_P) break;
    fsel = PF_P;
  }
  cells->clear();
  if (n == 0) return PF_OK;
  size_t tb = tmp_bytes;
  PF_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tb, key_in, key, list_in, list, n, 0, 32, ctx->stream));
  const int grid = std::max(1, std::min(n, 148 * 32));
  (++ctx->launches), k_rc_count<<<grid, 64, 0, ctx->stream>>>(G, P, fsel, list, n, cnt);
  PF_CUDA_TRY(cudaMemsetAsync(cnt + n, 0, sizeof(int), ctx->stream));
  tb = tmp_bytes;
  PF_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tb, cnt, off, n + 1, ctx->stream));
  PF_CUDA_TRY(cudaMemcpyAsync(ctx->h_pinned_ints, off + n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  const int total = ctx->h_pinned_ints[0];
  if (total == 0) return PF_OK;
  // the cell records after the fixed part (the scratch grows, keeping nothing of the fixed part's contents
  // that is still needed: list and offsets are copied into the grown buffer first when it moves)
  const size_t need = fixed + (size_t)total * sizeof(RcCell);
  if (need > ctx->rc_bytes) {
    char* old = buf;
    void* grown = nullptr;
    PF_CUDA_TRY(cudaMalloc(&grown, need));
    PF_CUDA_TRY(cudaMemcpyAsync(grown, old, fixed, cudaMemcpyDeviceToDevice, ctx->stream));
    PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    PF_CUDA_TRY(cudaFree(ctx->rc_buf));
    ctx->rc_buf = grown;
    ctx->rc_bytes = need;
    buf = (char*)grown;
    list = (int*)(buf + 3 * n4);
    off = (int*)(buf + 5 * n4);
  }
  RcCell* dc = (RcCell*)(buf + fixed);
  (++ctx->launches), k_rc_write<<<grid, 64, 0, ctx->stream>>>(G, P, fsel, list, n, off, dc);
  PF_CUDA_TRY(cudaGetLastError());
  cells->resize((size_t)total);
  PF_CUDA_TRY(cudaMemcpyAsync(cells->data(), dc, (size_t)total * sizeof(RcCell), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return PF_OK;
}

}  // namespace pf

extern "C" {

// writeSparseRenderCache3D (src/driver/render_cache3d.h:551-600): the
// primary particles and the context's secondary droplet and bubble sets
// (empty unless the step branches escaped particles or emits spray).
int pf_write_render_cache(pf_ctx* ctx, const char* path, int frame, double time, double dt, const pf_phase* ph,
                          double Vp, const pf_render_camera* cam, long long* bytes_written) {
  if (!ctx || !path || !path[0] || !ph) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  const pf::Geom& g = ctx->g;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const double dx = g.dx;
  pf_render_camera c{};
  if (cam) {
    c = *cam;
  } else {
    pf_default_render_camera(nx, ny, nz, dx, &c);
  }
  // writeHeader's argument check (:386-394)
  if (nx <= 0 || ny <= 0 || nz <= 0 || dx <= 0.0 || !std::isfinite(dx) || !std::isfinite(dt) ||
      !std::isfinite(time) || !pf::finite3(c.position) || !pf::finite3(c.target) || !pf::finite3(c.up) ||
      c.fov_degrees <= 0.0 || !std::isfinite(c.fov_degrees) || c.near_clip <= 0.0 || c.far_clip <= c.near_clip ||
      !std::isfinite(c.near_clip) || !std::isfinite(c.far_clip) || c.focal_length_mm <= 0.0 ||
      !std::isfinite(c.focal_length_mm))
    return PF_ERR_INVALID;

  std::vector<pf::RcCell> cells;
  int rc = pf::render_cells(ctx, ph, &cells);
  if (rc) return rc;
  const size_t n = ctx->np;
  std::vector<float> pos(3 * n), vel(3 * n), vol(n);
  std::vector<uint8_t> typ(n);
  if (n) {
    rc = pf_download_particles(ctx, pos.data(), vel.data(), typ.data(), vol.data());
    if (rc) return rc;
  }

  double liquid = 0.0;
  const double cell_volume = dx * dx * dx;
  for (const pf::RcCell& x : cells) liquid += x.phi * cell_volume;
  size_t n_liq = 0, n_gas = 0;
  double v_liq = 0.0, v_gas = 0.0;
  pf::Bounds water;
  for (size_t p = 0; p < n; ++p) {
    const double v = (double)vol[p] * Vp;
    if (typ[p] == 0) {
      ++n_liq;
      v_liq += v;
      const double q[3] = {pos[3 * p], pos[3 * p + 1], pos[3 * p + 2]};
      pf::include_point(water, q);
    } else if (typ[p] == 1) {
      ++n_gas;
      v_gas += v;
    }
  }
  for (const pf::RcCell& x : cells) {  // waterBounds (:302-314), level 0
    if (x.phi <= 0.0 && x.phi * cell_volume <= 0.0) continue;
    const double lo[3] = {x.i * dx, x.j * dx, x.k * dx};
    const double hi[3] = {(x.i + 1) * dx, (x.j + 1) * dx, (x.k + 1) * dx};
    pf::include_point(water, lo);
    pf::include_point(water, hi);
  }
  pf::Bounds domain;
  domain.valid = true;
  domain.mn[0] = domain.mn[1] = domain.mn[2] = 0.0;
  domain.mx[0] = nx * dx;
  domain.mx[1] = ny * dx;
  domain.mx[2] = nz * dx;
  // the secondary sets (escaped_droplets, escaped_bubbles and their ages)
  struct Set {
    std::vector<double> pos, vel, vol;
    std::vector<int> age;
    size_t n = 0;
  } sec[2];
  for (int w = 0; w < 2; ++w) {
    rc = pf_secondary_count(ctx, w, &sec[w].n);
    if (rc) return rc;
    Set& t = sec[w];
    t.pos.resize(3 * t.n);
    t.vel.resize(3 * t.n);
    t.vol.resize(t.n);
    t.age.resize(t.n);
    if (t.n) {
      rc = pf_get_secondary(ctx, w, t.pos.data(), t.vel.data(), t.vol.data(), t.age.data());
      if (rc) return rc;
    }
  }
  // secondaryVolume, secondaryAgeRange, secondaryBounds and the render
  // channels of secondaryRenderChannelCounts (:190-300)
  double sec_vol[2] = {0.0, 0.0};
  int age_min[2] = {0, 0}, age_max[2] = {0, 0};
  size_t ch_droplet = 0, ch_spray = 0, ch_foam = 0, ch_bubble = 0;
  std::vector<const char*> channel[2];
  pf::Bounds secondary{};
  for (int w = 0; w < 2; ++w) {
    const Set& t = sec[w];
    int mn = std::numeric_limits<int>::max(), mx = 0;
    channel[w].resize(t.n);
    for (size_t p = 0; p < t.n; ++p) {
      sec_vol[w] += t.vol[p] * Vp;
      const int a = std::max(0, t.age[p]);
      mn = std::min(mn, a);
      mx = std::max(mx, a);
      pf::include_point(secondary, &t.pos[3 * p]);
      const char* ch = "bubble";
      if (w == 0) {
        const double* v = &t.vel[3 * p];
        const double speed = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        ch = (a >= 4 && speed <= 0.5) ? "foam" : (a <= 1 || speed >= 1.0) ? "spray" : "droplet";
      }
      channel[w][p] = ch;
      if (ch[0] == 'f') ++ch_foam;
      else if (ch[0] == 's') ++ch_spray;
      else if (ch[0] == 'd') ++ch_droplet;
      else ++ch_bubble;
    }
    if (t.n) {
      age_min[w] = mn == std::numeric_limits<int>::max() ? 0 : mn;
      age_max[w] = mx;
    }
  }
  const double shutter_close = time + std::max(0.0, dt);

  std::ofstream out(path);
  if (!out) return PF_ERR_INVALID;
  out << std::setprecision(17);
  // writeHeader (:375-427)
  out << "{\"section\":\"header\",\"lsfs_cache3d_version\":1"
      << ",\"cache_schema_version\":2"
      << ",\"sim_kind\":\"sparse3d_tp\""
      << ",\"frame\":" << frame << ",\"time\":" << time << ",\"dt\":" << dt << ",\"dims\":[" << nx << "," << ny
      << "," << nz << "]"
      << ",\"dx\":" << dx << ",\"world_units\":\"cell\""
      << ",\"shutter_open\":" << time << ",\"shutter_close\":" << shutter_close << ",\"frame_bounds_min\":["
      << domain.mn[0] << "," << domain.mn[1] << "," << domain.mn[2] << "]"
      << ",\"frame_bounds_max\":[" << domain.mx[0] << "," << domain.mx[1] << "," << domain.mx[2] << "]"
      << ",\"phase\":{\"rho_l\":" << ph->rho_l << ",\"rho_g\":" << ph->rho_g << ",\"alpha_phi\":" << ph->alpha_phi
      << ",\"rho_tilde_0\":" << ph->rho_tilde_0 << "}}\n";
  out << "{\"section\":\"camera\",";
  pf::write_vec(out, "position", c.position);
  out << ",";
  pf::write_vec(out, "target", c.target);
  out << ",";
  pf::write_vec(out, "up", c.up);
  out << ",\"fov_degrees\":" << c.fov_degrees << ",\"vertical_fov_degrees\":" << c.fov_degrees
      << ",\"near_clip\":" << c.near_clip << ",\"far_clip\":" << c.far_clip
      << ",\"focal_length_mm\":" << c.focal_length_mm << "}\n";
  // writeWaterSummary (:429-458)
  out << "{\"section\":\"water_volume\""
      << ",\"primary_liquid_volume\":" << v_liq << ",\"primary_gas_volume\":" << v_gas
      << ",\"secondary_droplet_volume\":" << sec_vol[0] << ",\"secondary_bubble_volume\":" << sec_vol[1]
      << ",\"phase_field_liquid_volume\":" << liquid << ",\"phase_field_cells\":" << cells.size()
      << ",\"primary_liquid_count\":" << n_liq << ",\"primary_gas_count\":" << n_gas
      << ",\"secondary_droplet_count\":" << sec[0].n << ",\"secondary_bubble_count\":" << sec[1].n
      << ",\"secondary_particle_count\":" << sec[0].n + sec[1].n
      << ",\"secondary_droplet_age_min\":" << age_min[0] << ",\"secondary_droplet_age_max\":" << age_max[0]
      << ",\"secondary_bubble_age_min\":" << age_min[1] << ",\"secondary_bubble_age_max\":" << age_max[1]
      << "}\n";
  // writeSecondaryChannels (:460-476)
  out << "{\"section\":\"secondary_channels\",\"encoding\":\"render_channel_counts\""
      << ",\"channel_names\":[\"droplet\",\"spray\",\"foam\",\"bubble\"]"
      << ",\"droplet_count\":" << ch_droplet << ",\"spray_count\":" << ch_spray << ",\"foam_count\":" << ch_foam
      << ",\"bubble_count\":" << ch_bubble << ",\"total_count\":" << ch_droplet + ch_spray + ch_foam + ch_bubble
      << "}\n";
  // writeCinematicMetadata (:478-523)
  out << "{\"section\":\"cinematic_metadata\",\"cache_schema_version\":2,\"world_units\":\"cell\""
      << ",\"shutter_open\":" << time << ",\"shutter_close\":" << shutter_close << ",\"frame_time\":" << time
      << ",\"phase_field_sampling_stride\":1"
      << ",\"water_bounds_valid\":" << (water.valid ? "true" : "false")
      << ",\"secondary_bounds_valid\":" << (secondary.valid ? "true" : "false")
      << ",\"primary_particle_count\":" << n << ",\"primary_liquid_count\":" << n_liq
      << ",\"primary_gas_count\":" << n_gas
      << ",\"secondary_droplet_count\":" << sec[0].n << ",\"secondary_bubble_count\":" << sec[1].n
      << ",\"secondary_spray_count\":" << ch_spray << ",\"secondary_foam_count\":" << ch_foam;
  out << ",";
  pf::write_bounds(out, "frame_bounds_min", "frame_bounds_max", domain, domain);
  out << ",";
  pf::write_bounds(out, "water_bounds_min", "water_bounds_max", water, domain);
  out << ",";
  pf::write_bounds(out, "secondary_bounds_min", "secondary_bounds_max", secondary, domain);
  out << "}\n";
  // writePhaseField (:525-539)
  out << "{\"section\":\"phase_field\",\"encoding\":\"jsonl_cells\",\"count\":" << cells.size() << "}\n";
  for (const pf::RcCell& x : cells)
    out << "{\"section\":\"phase_cell\",\"i\":" << x.i << ",\"j\":" << x.j << ",\"k\":" << x.k
        << ",\"level\":0,\"marker\":" << x.marker << ",\"phi\":" << x.phi
        << ",\"liquid_volume\":" << x.phi * cell_volume << "}\n";
  // writeParticleSection (:541-560), primary then the two secondary sets
  out << "{\"section\":\"particles\",\"kind\":\"primary\",\"count\":" << n << "}\n";
  for (size_t p = 0; p < n; ++p) {
    const bool liq = typ[p] == 0;
    out << "{\"section\":\"particle\",\"kind\":\"primary\",\"render_channel\":\"" << (liq ? "water" : "air")
        << "\",\"index\":" << p << ",\"phase\":\"" << (liq ? "liquid" : "gas") << "\""
        << ",\"position\":[" << (double)pos[3 * p] << "," << (double)pos[3 * p + 1] << "," << (double)pos[3 * p + 2]
        << "]"
        << ",\"velocity\":[" << (double)vel[3 * p] << "," << (double)vel[3 * p + 1] << "," << (double)vel[3 * p + 2]
        << "]"
        << ",\"volume\":" << (double)vol[p] * Vp << "}\n";
  }
  for (int w = 0; w < 2; ++w) {
    const Set& t = sec[w];
    const char* kind = w == 0 ? "secondary_droplet" : "secondary_bubble";
    out << "{\"section\":\"particles\",\"kind\":\"" << kind << "\",\"count\":" << t.n << "}\n";
    for (size_t p = 0; p < t.n; ++p) {
      const double* q = &t.pos[3 * p];
      const double* v = &t.vel[3 * p];
      out << "{\"section\":\"particle\",\"kind\":\"" << kind << "\",\"render_channel\":\"" << channel[w][p]
          << "\",\"index\":" << p << ",\"phase\":\"" << (w == 0 ? "liquid" : "gas") << "\""
          << ",\"position\":[" << q[0] << "," << q[1] << "," << q[2] << "]"
          << ",\"velocity\":[" << v[0] << "," << v[1] << "," << v[2] << "]"
          << ",\"volume\":" << t.vol[p] * Vp << ",\"age\":" << t.age[p] << "}\n";
    }
  }
  out.flush();
  if (!out) return PF_ERR_INVALID;
  if (bytes_written) *bytes_written = (long long)out.tellp();
  return PF_OK;
}

// defaultRenderCacheCamera3D (src/driver/render_cache3d.h:47-61)
int pf_default_render_camera(int nx, int ny, int nz, double dx, pf_render_camera* cam) {
  if (!cam) return PF_ERR_INVALID;
  const double cx = 0.5 * nx * dx, cy = 0.5 * ny * dx, cz = 0.5 * nz * dx;
  const double span = std::max({nx * dx, ny * dx, nz * dx, dx});
  *cam = pf_render_camera{{cx, cy + 0.2 * span, cz + 2.0 * span}, {cx, cy, cz}, {0.0, 1.0, 0.0}, 45.0,
                          0.05 * dx, 5.0 * span, 50.0};
  return PF_OK;
}

int pf_write_render_manifest(const char* path, const char* sim_kind, int nx, int ny, int nz, double dx,
                             const pf_render_manifest_frame* frames, int n_frames) {
  // requireValidPath and requireManifestArgs (:101-105, :149-164)
  if (!path || !path[0] || !sim_kind || !sim_kind[0] || nx <= 0 || ny <= 0 || nz <= 0 || !(dx > 0.0) ||
      !std::isfinite(dx) || n_frames < 0 || (n_frames > 0 && !frames))
    return PF_ERR_INVALID;
  for (int i = 0; i < n_frames; ++i) {
    const pf_render_manifest_frame& f = frames[i];
    if (f.frame < 0 || f.step < 0 || !f.path || !f.path[0] || f.bytes < 0 || !std::isfinite(f.time))
      return PF_ERR_INVALID;
  }
  std::ofstream out(path);
  if (!out) return PF_ERR_INVALID;
  out << std::setprecision(17);
  const double ex = nx * dx, ey = ny * dx, ez = nz * dx;
  out << "{\n";
  out << "  \"lsfs_cache3d_manifest_version\":1,\n";
  out << "  \"cache_schema_version\":2,\n";
  out << "  \"world_units\":\"cell\",\n";
  out << "  \"sim_kind\":";
  pf::write_json_string(out, sim_kind);
  out << ",\n";
  out << "  \"dims\":[" << nx << "," << ny << "," << nz << "],\n";
  out << "  \"dx\":" << dx << ",\n";
  out << "  \"frame_bounds_min\":[0,0,0],\n";
  out << "  \"frame_bounds_max\":[" << ex << "," << ey << "," << ez << "],\n";
  out << "  \"frame_count\":" << n_frames << ",\n";
  out << "  \"frames\":[\n";
  for (int i = 0; i < n_frames; ++i) {
    const pf_render_manifest_frame& f = frames[i];
    out << "    {\"frame\":" << f.frame << ",\"step\":" << f.step << ",\"time\":" << f.time
        << ",\"shutter_open\":" << f.time << ",\"shutter_close\":" << f.time << ",\"frame_bounds_min\":[0,0,0]"
        << ",\"frame_bounds_max\":[" << ex << "," << ey << "," << ez << "]"
        << ",\"path\":";
    pf::write_json_string(out, f.path);
    out << ",\"bytes\":" << f.bytes << "}";
    if (i + 1 < n_frames) out << ",";
    out << "\n";
  }
  out << "  ]\n";
  out << "}\n";
  return out ? PF_OK : PF_ERR_INVALID;
}

}  // extern "C"
