// pf_learned.cu -- the learned coarse solve of the LEARNED mode.
//
// The coarse correction is a learned symmetric positive semi-definite
// operator applied to the restricted residual:
//
//   e = S G^T G S r_c,    S = diag(d_c)^-1/2 over live coarse unknowns,
//   G r = (h_0, ..., h_{L-1}),  h_0 = g_0 * C_0 r,  h_l = g_l * C_min(l,3) P h_{l-1},
//
// where C_l are 3x3x3 convolutions (2->16, then 16->16 channels) on the tile
// lattice and its 2x coarser levels down to 2 tiles per axis (L = 4..8, the
// last convolution shared by the levels below the fourth), P is 2x2x2
// average pooling and the g_l are per-position, per-channel gates -- a
// learned multilevel (BPX-like) additive operator.  The gates depend on the coarse
// operator only: a 4-level U-Net (3x3x3 convolutions with bias and ReLU,
// 16-64 channels, skip concatenations) maps scale-free features of A_c to
// g_0 once per solve, and g_{l+1} = P g_l.  Because e is linear and
// symmetric positive semi-definite in r_c, the two-level preconditioner
// D^-1 + P_c (S G^T G S) P_c^T is a fixed SPD operator during a solve and
// the flexible PCG keeps the convergence theory of PCG; the network only
// decides how good it is.  Scaling A by a constant scales e inversely.
//
// Training minimises the energy-norm error (e - e*)^T A_c (e - e*) / (e*^T r_c)
// against exact coarse solves e* harvested from EXACT_COARSE solves, with the
// gradient written out by hand (G^T, G, the gates, the U-Net) and Adam.
#include "pf_learned_kernels.cuh"

namespace pf {

namespace {

constexpr int kMaxLevels = 8;

Dims make_dims(int X, int Y, int Z) { return Dims{X, Y, Z, X * Y * Z}; }

Dims halve(const Dims& d) { return make_dims((d.X + 1) / 2, (d.Y + 1) / 2, (d.Z + 1) / 2); }

// levels of G: halve until every extent is <= 2 (at least 4, at most kMaxLevels)
int g_levels(Dims d) {
  int n = 1;
  while (std::max(d.X, std::max(d.Y, d.Z)) > 2 && n < kMaxLevels) {
    d = halve(d);
    ++n;
  }
  return std::max(4, n);
}

// G layer of level l: the last one is shared by every deeper level
int g_layer(int l) { return L_G0 + std::min(l, 3); }

// Device buffers for one batch size and lattice: the gate U-Net (one sample)
// and the G path (B samples).  Every G-path tensor has channel stride kGS.
struct Work {
  int B = 0, Balloc = 0;
  bool bwd = false;    // backward buffers allocated
  bool train = false;  // the current use keeps the forward intermediates for a backward pass
  int NL = 0;  // levels of G (the U-Net uses the first four)
  Dims D[kMaxLevels]{};
  size_t cap[kMaxLevels] = {};
  // U-Net forward (one sample)
  float *F = nullptr, *a0 = nullptr, *s0 = nullptr, *q1 = nullptr, *a1 = nullptr, *s1 = nullptr, *q2 = nullptr,
        *a2 = nullptr, *s2 = nullptr, *q3 = nullptr, *a3 = nullptr, *b3 = nullptr, *c2 = nullptr, *u2 = nullptr,
        *c1 = nullptr, *u1 = nullptr, *c0 = nullptr, *u0 = nullptr, *o = nullptr, *sc = nullptr;
  // U-Net backward scratch
  float *g0a = nullptr, *g0b = nullptr, *g0c = nullptr, *g1a = nullptr, *g1b = nullptr, *g1c = nullptr,
        *g2a = nullptr, *g2b = nullptr, *g2c = nullptr, *g3a = nullptr, *g3b = nullptr;
  // gates (one sample) and their gradients
  float *gam[kMaxLevels] = {}, *dgam[kMaxLevels] = {};
  // G path (B samples); q[0] is the scaled input S rc
  float *a[kMaxLevels] = {}, *h[kMaxLevels] = {}, *q[kMaxLevels] = {}, *b[kMaxLevels] = {}, *t[kMaxLevels] = {},
        *v[kMaxLevels] = {}, *e = nullptr;
  float *de = nullptr, *dt[kMaxLevels] = {}, *dh[kMaxLevels] = {}, *dv[kMaxLevels] = {}, *da[kMaxLevels] = {},
        *dq[kMaxLevels] = {};
  double *v64 = nullptr, *den = nullptr, *loss = nullptr;
  std::vector<void*> owned;
};

}  // namespace

struct LearnedState {
  int loaded = 0;
  size_t nparams = 0;
  size_t woff[kNumLayers] = {}, boff[kNumLayers] = {};
  float *params = nullptr, *grads = nullptr, *adam_m = nullptr, *adam_v = nullptr;
  uint2 *wf[kNumLayers] = {}, *wt[kNumLayers] = {};
  int adam_step = 0;
  float* wpart = nullptr;
  double* gstat = nullptr;  // gradient clipping state (k_grad_clip)
  Work inf, train, eval;
  // training set: systems (coarse operators) and (rc, e*) pairs
  struct System {
    Dims d;
    float* cop = nullptr;
    std::vector<size_t> pairs;  // float offsets into pool (rc then e*, 2 * nt each)
  };
  int harvesting = 0, harvest_stride = 1, harvest_max = 64, harvest_tick = 0;
  std::vector<System> systems;
  float* pool = nullptr;
  size_t pool_cap = 0, pool_used = 0;  // floats
  float *batch_rc = nullptr, *batch_tgt = nullptr;
  size_t batch_cap = 0;  // floats
};

namespace {

constexpr int kWgradCtas = 24;

unsigned long long splitmix(unsigned long long& s) {
  unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double uniform01(unsigned long long& s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

int grid_for(size_t n, int threads = 256) {
  size_t b = (n + threads - 1) / threads;
  if (b > 148 * 16) b = 148 * 16;
  return (int)(b > 0 ? b : 1);
}

size_t frag_count(int cin, int cout) { return (size_t)27 * (pad16(cin) / 16) * (pad8(cout) / 8) * 32; }

int allow_brick_smem(pf_ctx* ctx);
int work_ensure(pf_ctx* ctx, Work& W, Dims d0, int B, bool bwd);

int state_init(pf_ctx* ctx, LearnedState* L) {
  size_t o = 0;
  for (int l = 0; l < kNumLayers; ++l) {
    L->woff[l] = o;
    o += (size_t)27 * kLayers[l].cin * kLayers[l].cout;
    L->boff[l] = o;
    o += kLayers[l].cout;
  }
  L->nparams = o;
  float** arr[4] = {&L->params, &L->grads, &L->adam_m, &L->adam_v};
  for (float** q : arr) {
    PF_CUDA_TRY(cudaMalloc(q, o * sizeof(float)));
    PF_CUDA_TRY(cudaMemset(*q, 0, o * sizeof(float)));
  }
  for (int l = 0; l < kNumLayers; ++l) {
    const int ci = kLayers[l].cin, co = kLayers[l].cout;
    PF_CUDA_TRY(cudaMalloc(&L->wf[l], frag_count(ci, co) * sizeof(uint2)));
    PF_CUDA_TRY(cudaMalloc(&L->wt[l], frag_count(co, ci) * sizeof(uint2)));
  }
  PF_CUDA_TRY(cudaMalloc(&L->wpart, (size_t)kWgradCtas * 27 * 128 * 64 * sizeof(float)));
  PF_CUDA_TRY(cudaMalloc(&L->gstat, 4 * sizeof(double)));
  PF_CUDA_TRY(cudaMemset(L->gstat, 0, 4 * sizeof(double)));
  int rc = allow_brick_smem(ctx);
  if (rc) return rc;
  // the solver's working memory for this context's tile lattice, so that no
  // solve allocates: the gate network and G path, the neighbour-slot table
  CoarseCtx* c = (CoarseCtx*)ctx->learned;
  rc = work_ensure(ctx, L->inf, make_dims(c->op.TX, c->op.TY, c->op.TZ), 1, false);
  if (rc) return rc;
  int* nbr = nullptr;
  return build_neighbor_table(ctx, 0, &nbr);
}

LearnedState* get_state(pf_ctx* ctx, int* rc) {
  *rc = coarse_ensure(ctx);
  if (*rc) return nullptr;
  CoarseCtx* c = (CoarseCtx*)ctx->learned;
  if (!c->net) {
    c->net = new LearnedState();
    *rc = state_init(ctx, c->net);
    if (*rc) return nullptr;
  }
  return c->net;
}

int repack(pf_ctx* ctx, LearnedState* L) {
  for (int l = 0; l < kNumLayers; ++l) {
    const int ci = kLayers[l].cin, co = kLayers[l].cout;
    (++ctx->launches), k_pack<<<grid_for(frag_count(ci, co)), 256, 0, ctx->stream>>>(L->params + L->woff[l], ci, co,
                                                                                      0, L->wf[l]);
    (++ctx->launches), k_pack<<<grid_for(frag_count(co, ci)), 256, 0, ctx->stream>>>(L->params + L->woff[l], ci, co,
                                                                                      1, L->wt[l]);
  }
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

void work_free(Work& W) {
  for (void* p : W.owned) cudaFree(p);
  W.owned.clear();
  W = Work{};
}

int work_ensure(pf_ctx* ctx, Work& W, Dims d0, int B, bool bwd) {
  const int NL = g_levels(d0);
  Dims D[kMaxLevels];
  D[0] = d0;
  for (int l = 1; l < NL; ++l) D[l] = halve(D[l - 1]);
  // buffers hold Balloc samples of up to cap[l] positions per level
  bool fits = W.Balloc >= B && (W.bwd || !bwd);
  for (int l = 0; l < NL && fits; ++l) fits = (size_t)D[l].n <= W.cap[l];
  W.train = bwd;
  if (fits) {
    W.B = B;
    W.NL = NL;
    for (int l = 0; l < NL; ++l) W.D[l] = D[l];
    return PF_OK;
  }
  work_free(W);
  size_t n[kMaxLevels], P[kMaxLevels];
  for (int l = 0; l < NL; ++l) {
    n[l] = (size_t)D[l].n;
    P[l] = (size_t)B * n[l];
    W.cap[l] = n[l];
    W.D[l] = D[l];
  }
  W.NL = NL;
  W.B = B;
  W.Balloc = B;
  W.bwd = bwd;
  W.train = bwd;
  int rc = 0;
  auto alloc = [&](float** q, size_t count) {
    if (rc) return;
    if (cudaMalloc(q, count * sizeof(float)) != cudaSuccess || cudaMemset(*q, 0, count * sizeof(float)) != cudaSuccess) {
      rc = set_error(ctx, PF_ERR_CUDA, "learned: out of device memory");
      return;
    }
    W.owned.push_back(*q);
  };
  alloc(&W.F, n[0] * kInCh);
  alloc(&W.a0, n[0] * 16);
  alloc(&W.s0, n[0] * 16);
  alloc(&W.q1, n[1] * 16);
  alloc(&W.a1, n[1] * 32);
  alloc(&W.s1, n[1] * 32);
  alloc(&W.q2, n[2] * 32);
  alloc(&W.a2, n[2] * 64);
  alloc(&W.s2, n[2] * 64);
  alloc(&W.q3, n[3] * 64);
  alloc(&W.a3, n[3] * 64);
  alloc(&W.b3, n[3] * 64);
  alloc(&W.c2, n[2] * 128);
  alloc(&W.u2, n[2] * 64);
  alloc(&W.c1, n[1] * 96);
  alloc(&W.u1, n[1] * 32);
  alloc(&W.c0, n[0] * 48);
  alloc(&W.u0, n[0] * 16);
  alloc(&W.o, n[0] * 16);
  alloc(&W.sc, 2);
  W.gam[0] = W.o;
  for (int l = 1; l < NL; ++l) alloc(&W.gam[l], n[l] * kGS);
  for (int l = 0; l < NL; ++l) {
    alloc(&W.a[l], P[l] * kGS);
    alloc(&W.h[l], P[l] * kGS);
    alloc(&W.t[l], P[l] * kGS);
    alloc(&W.v[l], P[l] * kGS);
    alloc(&W.q[l], P[l] * kGS);
    if (bwd && l < NL - 1) alloc(&W.b[l], P[l] * kGS);
  }
  alloc(&W.e, P[0] * 2);
  if (bwd) {
    alloc(&W.g0a, n[0] * 48);
    alloc(&W.g0b, n[0] * 48);
    alloc(&W.g0c, n[0] * 48);
    alloc(&W.g1a, n[1] * 96);
    alloc(&W.g1b, n[1] * 96);
    alloc(&W.g1c, n[1] * 96);
    alloc(&W.g2a, n[2] * 128);
    alloc(&W.g2b, n[2] * 128);
    alloc(&W.g2c, n[2] * 128);
    alloc(&W.g3a, n[3] * 64);
    alloc(&W.g3b, n[3] * 64);
    alloc(&W.de, P[0] * kGS);
    for (int l = 0; l < NL; ++l) {
      alloc(&W.dgam[l], n[l] * kGS);
      alloc(&W.dt[l], P[l] * kGS);
      alloc(&W.dh[l], P[l] * kGS);
      alloc(&W.dv[l], P[l] * kGS);
      alloc(&W.da[l], P[l] * kGS);
      alloc(&W.dq[l], P[l] * kGS);
    }
    double** dd[3] = {&W.v64, &W.den, &W.loss};
    size_t dn[3] = {P[0] * 2, (size_t)B, (size_t)B};
    for (int q = 0; q < 3 && !rc; ++q) {
      if (cudaMalloc(dd[q], dn[q] * sizeof(double)) != cudaSuccess) {
        rc = set_error(ctx, PF_ERR_CUDA, "learned: out of device memory");
        break;
      }
      W.owned.push_back(*dd[q]);
    }
  }
  return rc;
}

// ---------------------------------------------------------------------------
// layers

int conv(pf_ctx* ctx, LearnedState* L, int layer, const float* x, int xs, const float* gate, bool transpose,
         float* y, int ys, Dims d, int B, const SolveCtl* skip, const float* gmul = nullptr) {
  const LayerSpec& s = kLayers[layer];
  ConvArgs a;
  a.x = x;
  a.gate = gate;
  a.xs = xs;
  a.wf = transpose ? L->wt[layer] : L->wf[layer];
  a.bias = (!transpose && s.bias) ? L->params + L->boff[layer] : nullptr;
  a.cout = transpose ? s.cin : s.cout;
  a.relu = transpose ? 0 : s.relu;
  a.y = y;
  a.ys = ys;
  a.d = d;
  a.P = B * d.n;
  a.skip = skip;
  a.gmul = gmul;
  if (xs != pad16(transpose ? s.cout : s.cin) || ys < pad8(a.cout) || (gmul && (a.bias || a.relu)))
    return set_error(ctx, PF_ERR_INVALID, "learned: channel stride mismatch");
  const int NT = pad8(a.cout) / 8;
  const int bx = (d.X + kBrick - 1) / kBrick, by = (d.Y + kBrick - 1) / kBrick, bz = (d.Z + kBrick - 1) / kBrick;
  const int blocks = B * bx * by * bz;
  const int KC = xs / 16;
  a.stage_w = brick_smem_w(KC, NT) <= kStageWeightsMax ? 1 : 0;
  const size_t smem = (size_t)brick_smem_halo(KC) + (a.stage_w ? brick_smem_w(KC, NT) : 0);
  ++ctx->launches;
  switch (NT) {
    case 1: k_conv_brick<1><<<blocks, 128, smem, ctx->stream>>>(a, bx, by, bz); break;
    case 2: k_conv_brick<2><<<blocks, 128, smem, ctx->stream>>>(a, bx, by, bz); break;
    case 4: k_conv_brick<4><<<blocks, 128, smem, ctx->stream>>>(a, bx, by, bz); break;
    case 6: k_conv_brick<6><<<blocks, 128, smem, ctx->stream>>>(a, bx, by, bz); break;
    case 8: k_conv_brick<8><<<blocks, 128, smem, ctx->stream>>>(a, bx, by, bz); break;
    case 12: k_conv_brick<12><<<blocks, 128, smem, ctx->stream>>>(a, bx, by, bz); break;
    case 16: k_conv_brick<16><<<blocks, 128, smem, ctx->stream>>>(a, bx, by, bz); break;
    default: return set_error(ctx, PF_ERR_INVALID, "learned: unsupported channel count");
  }
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

// the widest input (128 channels) stages 58.75 KB, more than the default 48 KB
int allow_brick_smem(pf_ctx* ctx) {
  const int bytes = brick_smem_halo(8) + kStageWeightsMax;
  PF_CUDA_TRY(cudaFuncSetAttribute(k_conv_brick<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  PF_CUDA_TRY(cudaFuncSetAttribute(k_conv_brick<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  PF_CUDA_TRY(cudaFuncSetAttribute(k_conv_brick<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  PF_CUDA_TRY(cudaFuncSetAttribute(k_conv_brick<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  PF_CUDA_TRY(cudaFuncSetAttribute(k_conv_brick<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  PF_CUDA_TRY(cudaFuncSetAttribute(k_conv_brick<12>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  PF_CUDA_TRY(cudaFuncSetAttribute(k_conv_brick<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  return PF_OK;
}

// grads[W of layer] += sum_p x[p + tap] (outer) dz[p], dz = dy gated by y > 0 when `gate`
int wgrad_acc(pf_ctx* ctx, LearnedState* L, int layer, const float* x, int xs, const float* dy, const float* gate,
              int ds, Dims d, int B) {
  const LayerSpec& s = kLayers[layer];
  const int P = B * d.n;
  const size_t count = (size_t)27 * s.cin * s.cout;
  const int nchunks = (P + kWChunk - 1) / kWChunk;
  const int nctas = nchunks < kWgradCtas ? nchunks : kWgradCtas;
  WgradArgs w{x, xs, s.cin, dy, gate, ds, s.cout, L->wpart, d, P};
  ++ctx->launches;
  k_wgrad<<<dim3(nctas, 27), 256, 0, ctx->stream>>>(w);
  ++ctx->launches;
  k_wgrad_reduce<<<grid_for(count), 256, 0, ctx->stream>>>(L->wpart, nctas, (int)count, L->grads + L->woff[layer]);
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

// one U-Net layer backward: weight and bias gradients; dx (optional) = conv^T(gated dy)
int layer_backward(pf_ctx* ctx, LearnedState* L, int layer, const float* x, int xs, const float* dy,
                   const float* y, int ds, float* dx, int dxs, Dims d) {
  const LayerSpec& s = kLayers[layer];
  const float* gate = s.relu ? y : nullptr;
  int rc = wgrad_acc(ctx, L, layer, x, xs, dy, gate, ds, d, 1);
  if (rc) return rc;
  ++ctx->launches;
  k_bias_grad<<<s.cout, 256, 0, ctx->stream>>>(dy, gate, ds, d.n, L->grads + L->boff[layer]);
  PF_CUDA_TRY(cudaGetLastError());
  if (dx) return conv(ctx, L, layer, dy, ds, gate, true, dx, dxs, d, 1, nullptr);
  return PF_OK;
}

// ---------------------------------------------------------------------------
// the gate U-Net (one sample): features of A_c -> g_0 (16 channels), deeper gates by pooling

int unet_forward(pf_ctx* ctx, LearnedState* L, Work& W, const float* cop, const SolveCtl* skip) {
  const Dims* D = W.D;
  ++ctx->launches;
  k_scales<<<2, 256, 0, ctx->stream>>>(cop, nullptr, D[0].n, 1, W.sc, skip);
  ++ctx->launches;
  k_features<<<grid_for(D[0].n), 256, 0, ctx->stream>>>(cop, nullptr, D[0], 1, W.sc, W.F, skip);
  int rc = 0;
  auto pool_to = [&](const float* x, int cs, int lf, float* y) {
    ++ctx->launches;
    k_pool<<<grid_for((size_t)D[lf + 1].n * cs), 256, 0, ctx->stream>>>(x, cs, D[lf], D[lf + 1], 1, y, skip);
  };
  auto up_cat = [&](const float* coarse, int cu, int lc, const float* sk, int csk, float* out) {
    ++ctx->launches;
    k_up_concat<<<grid_for((size_t)D[lc - 1].n * (cu + csk)), 256, 0, ctx->stream>>>(coarse, cu, D[lc], sk, csk,
                                                                                      D[lc - 1], 1, out, skip);
  };
  rc = rc ? rc : conv(ctx, L, L_E0A, W.F, kInCh, nullptr, false, W.a0, 16, D[0], 1, skip);
  rc = rc ? rc : conv(ctx, L, L_E0B, W.a0, 16, nullptr, false, W.s0, 16, D[0], 1, skip);
  pool_to(W.s0, 16, 0, W.q1);
  rc = rc ? rc : conv(ctx, L, L_E1A, W.q1, 16, nullptr, false, W.a1, 32, D[1], 1, skip);
  rc = rc ? rc : conv(ctx, L, L_E1B, W.a1, 32, nullptr, false, W.s1, 32, D[1], 1, skip);
  pool_to(W.s1, 32, 1, W.q2);
  rc = rc ? rc : conv(ctx, L, L_E2A, W.q2, 32, nullptr, false, W.a2, 64, D[2], 1, skip);
  rc = rc ? rc : conv(ctx, L, L_E2B, W.a2, 64, nullptr, false, W.s2, 64, D[2], 1, skip);
  pool_to(W.s2, 64, 2, W.q3);
  rc = rc ? rc : conv(ctx, L, L_E3A, W.q3, 64, nullptr, false, W.a3, 64, D[3], 1, skip);
  rc = rc ? rc : conv(ctx, L, L_E3B, W.a3, 64, nullptr, false, W.b3, 64, D[3], 1, skip);
  up_cat(W.b3, 64, 3, W.s2, 64, W.c2);
  rc = rc ? rc : conv(ctx, L, L_D2, W.c2, 128, nullptr, false, W.u2, 64, D[2], 1, skip);
  up_cat(W.u2, 64, 2, W.s1, 32, W.c1);
  rc = rc ? rc : conv(ctx, L, L_D1, W.c1, 96, nullptr, false, W.u1, 32, D[1], 1, skip);
  up_cat(W.u1, 32, 1, W.s0, 16, W.c0);
  rc = rc ? rc : conv(ctx, L, L_D0, W.c0, 48, nullptr, false, W.u0, 16, D[0], 1, skip);
  rc = rc ? rc : conv(ctx, L, L_OUT, W.u0, 16, nullptr, false, W.o, 16, D[0], 1, skip);
  if (rc) return rc;
  for (int l = 0; l + 1 < W.NL; ++l) pool_to(W.gam[l], kGS, l, W.gam[l + 1]);
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

// U-Net backward from W.g0a (= dL/dg_0, stride 16)
int unet_backward(pf_ctx* ctx, LearnedState* L, Work& W) {
  const Dims* D = W.D;
  int rc = 0;
  auto pool_bwd = [&](const float* dy, int cs, int lf, float* dx) {
    ++ctx->launches;
    k_pool_bwd<<<grid_for((size_t)D[lf].n * cs), 256, 0, ctx->stream>>>(dy, cs, D[lf], D[lf + 1], 1, dx);
  };
  auto cat_bwd = [&](const float* dout, int cu, int csk, int lc, float* dcoarse, float* dskip) {
    ++ctx->launches;
    k_up_concat_bwd<<<grid_for((size_t)D[lc - 1].n * (cu + csk)), 256, 0, ctx->stream>>>(dout, cu, csk, D[lc],
                                                                                          D[lc - 1], 1, dcoarse,
                                                                                          dskip);
  };
  rc = rc ? rc : layer_backward(ctx, L, L_OUT, W.u0, 16, W.g0a, W.o, 16, W.g0b, 16, D[0]);      // g0b = du0
  rc = rc ? rc : layer_backward(ctx, L, L_D0, W.c0, 48, W.g0b, W.u0, 16, W.g0c, 48, D[0]);      // g0c = dc0
  cat_bwd(W.g0c, 32, 16, 1, W.g1a, W.g0a);                                                      // du1, ds0
  rc = rc ? rc : layer_backward(ctx, L, L_D1, W.c1, 96, W.g1a, W.u1, 32, W.g1b, 96, D[1]);      // dc1
  cat_bwd(W.g1b, 64, 32, 2, W.g2a, W.g1c);                                                      // du2, ds1
  rc = rc ? rc : layer_backward(ctx, L, L_D2, W.c2, 128, W.g2a, W.u2, 64, W.g2b, 128, D[2]);    // dc2
  cat_bwd(W.g2b, 64, 64, 3, W.g3a, W.g2c);                                                      // db3, ds2
  rc = rc ? rc : layer_backward(ctx, L, L_E3B, W.a3, 64, W.g3a, W.b3, 64, W.g3b, 64, D[3]);     // da3
  rc = rc ? rc : layer_backward(ctx, L, L_E3A, W.q3, 64, W.g3b, W.a3, 64, W.g3a, 64, D[3]);     // dq3
  pool_bwd(W.g3a, 64, 2, W.g2c);                                                                // ds2 += P^T dq3
  rc = rc ? rc : layer_backward(ctx, L, L_E2B, W.a2, 64, W.g2c, W.s2, 64, W.g2a, 64, D[2]);     // da2
  rc = rc ? rc : layer_backward(ctx, L, L_E2A, W.q2, 32, W.g2a, W.a2, 64, W.g2b, 32, D[2]);     // dq2
  pool_bwd(W.g2b, 32, 1, W.g1c);                                                                // ds1 += P^T dq2
  rc = rc ? rc : layer_backward(ctx, L, L_E1B, W.a1, 32, W.g1c, W.s1, 32, W.g1a, 32, D[1]);     // da1
  rc = rc ? rc : layer_backward(ctx, L, L_E1A, W.q1, 16, W.g1a, W.a1, 32, W.g1b, 16, D[1]);     // dq1
  pool_bwd(W.g1b, 16, 0, W.g0a);                                                                // ds0 += P^T dq1
  rc = rc ? rc : layer_backward(ctx, L, L_E0B, W.a0, 16, W.g0a, W.s0, 16, W.g0b, 16, D[0]);     // da0
  rc = rc ? rc : layer_backward(ctx, L, L_E0A, W.F, kInCh, W.g0b, W.a0, 16, nullptr, 0, D[0]);
  return rc;
}

// ---------------------------------------------------------------------------
// the G path (B samples): e = S G^T G S rc

// Inference: 2 NL launches of the 16-channel G kernel (pool, gates, upsampling
// and the diagonal scaling folded into its staging and epilogue).  The first
// launch waits for every earlier kernel, the weights' packing included; the
// others are programmatic dependent launches that copy their weights while
// their predecessor drains.
int gtg_apply(pf_ctx* ctx, LearnedState* L, Work& W, const float* cop, const float* rc_in, float* e_out,
              const SolveCtl* skip) {
  const int NL = W.NL;
  const Dims* D = W.D;
  auto args = [&](int l) {
    GConvArgs a{};
    a.d = D[l];
    a.dc = l + 1 < NL ? D[l + 1] : D[l];
    a.bx = (D[l].X + kGBX - 1) / kGBX;
    a.by = (D[l].Y + kGBY - 1) / kGBY;
    a.gate = W.gam[l];
    a.cop = cop;
    a.skip = skip;
    return a;
  };
  auto grid = [&](int l) {
    return dim3((unsigned)(((D[l].X + kGBX - 1) / kGBX) * ((D[l].Y + kGBY - 1) / kGBY) * ((D[l].Z + kGBZ - 1) / kGBZ)),
                (unsigned)W.B);
  };
  for (int l = 0; l < NL; ++l) {
    GConvArgs a = args(l);
    a.wf = L->wf[g_layer(l)];
    a.y = W.h[l];
    a.pool = l + 1 < NL ? W.q[l + 1] : nullptr;
    ++ctx->launches;
    if (l == 0) {
      a.x = rc_in;
      k_gconv<GIN_SCALE, GOUT_GATE, 2><<<grid(l), 128, 0, ctx->stream>>>(a);
    } else {
      a.x = W.q[l];
      PF_CUDA_TRY(launch_pdl(k_gconv<GIN_PLAIN, GOUT_GATE, 2>, grid(l), dim3(128), ctx->stream, a));
    }
  }
  for (int l = NL - 1; l >= 0; --l) {
    GConvArgs a = args(l);
    a.x = W.h[l];
    a.vpar = l + 1 < NL ? W.v[l + 1] : nullptr;
    ++ctx->launches;
    if (l > 0) {
      a.wf = L->wt[g_layer(l)];
      a.y = W.v[l];
      PF_CUDA_TRY(launch_pdl(k_gconv<GIN_TGATE, GOUT_PLAIN, 2>, grid(l), dim3(128), ctx->stream, a));
    } else {
      a.wf = L->wt[L_G0];
      a.y = e_out;
      PF_CUDA_TRY(launch_pdl(k_gconv<GIN_TGATE, GOUT_SCALE, 1>, grid(l), dim3(128), ctx->stream, a));
    }
  }
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

int gtg_forward(pf_ctx* ctx, LearnedState* L, Work& W, const float* cop, const float* rc_in, float* e_out,
                const SolveCtl* skip) {
  if (!W.train) return gtg_apply(ctx, L, W, cop, rc_in, e_out, skip);
  const int B = W.B, NL = W.NL;
  const Dims* D = W.D;
  int rc = 0;
  auto n16 = [&](int l) { return (size_t)B * D[l].n * kGS; };
  ++ctx->launches;
  k_scale_in<<<grid_for(n16(0)), 256, 0, ctx->stream>>>(rc_in, 0, cop, D[0].n, B, W.q[0], skip);
  for (int l = 0; l < NL && !rc; ++l) {
    if (l > 0) {
      ++ctx->launches;
      k_pool<<<grid_for(n16(l)), 256, 0, ctx->stream>>>(W.h[l - 1], kGS, D[l - 1], D[l], B, W.q[l], skip);
    }
    if (W.train) {  // training keeps the ungated a_l for the gate gradient
      rc = conv(ctx, L, g_layer(l), W.q[l], kGS, nullptr, false, W.a[l], kGS, D[l], B, skip);
      ++ctx->launches;
      k_gmul<<<grid_for(n16(l)), 256, 0, ctx->stream>>>(W.h[l], W.gam[l], W.a[l], D[l].n, B, skip);
    } else {
      rc = conv(ctx, L, g_layer(l), W.q[l], kGS, nullptr, false, W.h[l], kGS, D[l], B, skip, W.gam[l]);
    }
  }
  if (rc) return rc;
  ++ctx->launches;
  k_gmul<<<grid_for(n16(NL - 1)), 256, 0, ctx->stream>>>(W.t[NL - 1], W.gam[NL - 1], W.h[NL - 1], D[NL - 1].n, B,
                                                         skip);
  for (int l = NL - 1; l >= 1 && !rc; --l) {
    rc = conv(ctx, L, g_layer(l), W.t[l], kGS, nullptr, true, W.v[l], kGS, D[l], B, skip);
    if (rc) break;
    ++ctx->launches;
    k_up_add_gate<<<grid_for(n16(l - 1)), 256, 0, ctx->stream>>>(W.h[l - 1], W.v[l], W.gam[l - 1], D[l - 1], D[l], B,
                                                                  W.b[l - 1], W.t[l - 1], skip);
  }
  if (rc) return rc;
  rc = conv(ctx, L, L_G0, W.t[0], kGS, nullptr, true, W.v[0], kGS, D[0], B, skip);
  if (rc) return rc;
  ++ctx->launches;
  k_scale_out<<<grid_for((size_t)B * D[0].n * 2), 256, 0, ctx->stream>>>(W.v[0], cop, D[0].n, B, e_out, skip);
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

// gradients of <de, e> into the G weights (accumulated) and dgam[0] (gates folded to level 0)
int gtg_backward(pf_ctx* ctx, LearnedState* L, Work& W, const float* cop) {
  const int B = W.B, NL = W.NL;
  const Dims* D = W.D;
  auto n16 = [&](int l) { return (size_t)B * D[l].n * kGS; };
  auto g16 = [&](int l) { return (size_t)D[l].n * kGS; };
  int rc = 0;
  for (int l = 0; l < NL; ++l) {
    ++ctx->launches;
    k_zero_f<<<grid_for(g16(l)), 256, 0, ctx->stream>>>(W.dgam[l], g16(l));
  }
  // transposed half, fine to coarse: dv_l = (l ? P dh_{l-1} : S de), dt_l = C_l dv_l
  for (int l = 0; l < NL && !rc; ++l) {
    ++ctx->launches;
    if (l == 0)
      k_scale_in<<<grid_for(n16(0)), 256, 0, ctx->stream>>>(W.de, 1, cop, D[0].n, B, W.dv[0], nullptr);
    else
      k_pool<<<grid_for(n16(l)), 256, 0, ctx->stream>>>(W.dh[l - 1], kGS, D[l - 1], D[l], B, W.dv[l], nullptr);
    rc = conv(ctx, L, g_layer(l), W.dv[l], kGS, nullptr, false, W.dt[l], kGS, D[l], B, nullptr);
    rc = rc ? rc : wgrad_acc(ctx, L, g_layer(l), W.dv[l], kGS, W.t[l], nullptr, kGS, D[l], B);
    ++ctx->launches;
    k_gate_grad<<<grid_for(g16(l)), 256, 0, ctx->stream>>>(W.dgam[l], W.dt[l], l < NL - 1 ? W.b[l] : W.h[l], D[l].n,
                                                          B);
    ++ctx->launches;
    k_gmul<<<grid_for(n16(l)), 256, 0, ctx->stream>>>(W.dh[l], W.gam[l], W.dt[l], D[l].n, B, nullptr);
  }
  // forward half, coarse to fine
  for (int l = NL - 1; l >= 0 && !rc; --l) {
    ++ctx->launches;
    k_gmul<<<grid_for(n16(l)), 256, 0, ctx->stream>>>(W.da[l], W.gam[l], W.dh[l], D[l].n, B, nullptr);
    ++ctx->launches;
    k_gate_grad<<<grid_for(g16(l)), 256, 0, ctx->stream>>>(W.dgam[l], W.a[l], W.dh[l], D[l].n, B);
    rc = wgrad_acc(ctx, L, g_layer(l), W.q[l], kGS, W.da[l], nullptr, kGS, D[l], B);
    if (l > 0 && !rc) {
      rc = conv(ctx, L, g_layer(l), W.da[l], kGS, nullptr, true, W.dq[l], kGS, D[l], B, nullptr);
      ++ctx->launches;
      k_pool_bwd<<<grid_for(n16(l - 1)), 256, 0, ctx->stream>>>(W.dq[l], kGS, D[l - 1], D[l], B, W.dh[l - 1]);
    }
  }
  if (rc) return rc;
  // g_{l+1} = P g_l
  for (int l = NL - 2; l >= 0; --l) {
    ++ctx->launches;
    k_pool_bwd<<<grid_for(g16(l)), 256, 0, ctx->stream>>>(W.dgam[l + 1], kGS, D[l], D[l + 1], 1, W.dgam[l]);
  }
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

// loss over B pairs of one system and the gradient of every parameter (into L->grads)
int loss_backward(pf_ctx* ctx, LearnedState* L, Work& W, const float* cop, const float* rc_in, const float* tgt) {
  const int B = W.B;
  const Dims d = W.D[0];
  PF_CUDA_TRY(cudaMemsetAsync(L->grads, 0, L->nparams * sizeof(float), ctx->stream));
  int r = unet_forward(ctx, L, W, cop, nullptr);
  r = r ? r : gtg_forward(ctx, L, W, cop, rc_in, W.e, nullptr);
  if (r) return r;
  ++ctx->launches;
  k_loss_prep<<<B, 256, 0, ctx->stream>>>(W.e, tgt, rc_in, cop, d.n, W.v64, W.den);
  ++ctx->launches;
  k_zero_f<<<grid_for((size_t)B * d.n * kGS), 256, 0, ctx->stream>>>(W.de, (size_t)B * d.n * kGS);
  ++ctx->launches;
  k_loss_grad<<<B, 256, 0, ctx->stream>>>(W.v64, W.den, cop, d, B, W.de, W.loss);
  PF_CUDA_TRY(cudaGetLastError());
  r = gtg_backward(ctx, L, W, cop);
  if (r) return r;
  PF_CUDA_TRY(cudaMemcpyAsync(W.g0a, W.dgam[0], (size_t)d.n * kGS * sizeof(float), cudaMemcpyDeviceToDevice,
                              ctx->stream));
  return unet_backward(ctx, L, W);
}

// One Adam step on L->grads; `clip` applies the training loop's gradient-norm
// clipping first (the step counter still advances on a skipped step).
int adam_step(pf_ctx* ctx, LearnedState* L, double lr, bool clip) {
  L->adam_step += 1;
  const double b1 = 0.9, b2 = 0.999;
  const double c1 = 1.0 - std::pow(b1, L->adam_step), c2 = 1.0 - std::pow(b2, L->adam_step);
  if (clip) {
    ctx->launches += 2;
    k_grad_sumsq<<<grid_for(L->nparams), 256, 0, ctx->stream>>>(L->grads, L->nparams, L->gstat);
    k_grad_clip<<<1, 1, 0, ctx->stream>>>(L->gstat);
  }
  ++ctx->launches;
  k_adam<<<grid_for(L->nparams), 256, 0, ctx->stream>>>(L->params, L->grads, L->adam_m, L->adam_v, L->nparams,
                                                       (float)lr, (float)b1, (float)b2, (float)c1, (float)c2, 1e-8f,
                                                       clip ? L->gstat + 1 : nullptr);
  PF_CUDA_TRY(cudaGetLastError());
  return repack(ctx, L);
}

}  // namespace

// ---------------------------------------------------------------------------
// hooks used by the solver

bool coarse_net_ready(const pf_ctx* ctx) {
  const CoarseCtx* c = (const CoarseCtx*)ctx->learned;
  return c && c->net && c->net->loaded;
}

int coarse_prepare_net(pf_ctx* ctx) {
  if (!coarse_net_ready(ctx)) return set_error(ctx, PF_ERR_INVALID, "no learned network loaded");
  CoarseCtx* c = (CoarseCtx*)ctx->learned;
  LearnedState* L = c->net;
  CoarseOp& A = c->op;
  int rc = work_ensure(ctx, L->inf, make_dims(A.TX, A.TY, A.TZ), 1, false);
  if (rc) return rc;
  return unet_forward(ctx, L, L->inf, A.cop, nullptr);
}

int coarse_solve_net(pf_ctx* ctx, const SolveCtl* skip) {
  if (!coarse_net_ready(ctx)) return set_error(ctx, PF_ERR_INVALID, "no learned network loaded");
  CoarseCtx* c = (CoarseCtx*)ctx->learned;
  LearnedState* L = c->net;
  return gtg_forward(ctx, L, L->inf, c->op.cop, c->op.rc, c->op.ec, skip);
}

void coarse_new_system(pf_ctx* ctx) {
  CoarseCtx* c = (CoarseCtx*)ctx->learned;
  if (!c || !c->net || !c->net->harvesting) return;
  LearnedState* L = c->net;
  LearnedState::System s;
  s.d = make_dims(c->op.TX, c->op.TY, c->op.TZ);
  const size_t bytes = (size_t)c->op.nt * kCopStride * sizeof(float);
  if (cudaMalloc(&s.cop, bytes) != cudaSuccess) {
    cudaGetLastError();
    L->harvesting = 0;
    return;
  }
  cudaMemcpyAsync(s.cop, c->op.cop, bytes, cudaMemcpyDeviceToDevice, ctx->stream);
  L->systems.push_back(s);
  L->harvest_tick = 0;
}

int coarse_harvest(pf_ctx* ctx, const SolveCtl*) {
  CoarseCtx* c = (CoarseCtx*)ctx->learned;
  if (!c || !c->net || !c->net->harvesting || c->net->systems.empty()) return PF_OK;
  LearnedState* L = c->net;
  LearnedState::System& s = L->systems.back();
  const int tick = L->harvest_tick++;
  if (tick % L->harvest_stride != 0 || (int)s.pairs.size() >= L->harvest_max) return PF_OK;
  const size_t n2 = 2 * (size_t)s.d.n;
  if (L->pool_used + 2 * n2 > L->pool_cap) return PF_OK;  // full: keep what we have
  const size_t off = L->pool_used;
  PF_CUDA_TRY(cudaMemcpyAsync(L->pool + off, c->op.rc, n2 * sizeof(float), cudaMemcpyDeviceToDevice, ctx->stream));
  PF_CUDA_TRY(cudaMemcpyAsync(L->pool + off + n2, c->op.ec, n2 * sizeof(float), cudaMemcpyDeviceToDevice,
                              ctx->stream));
  L->pool_used += 2 * n2;
  s.pairs.push_back(off);
  return PF_OK;
}

void learned_release(CoarseCtx* c) {
  LearnedState* L = c->net;
  if (!L) return;
  float* fl[] = {L->params, L->grads, L->adam_m, L->adam_v, L->wpart, L->pool, L->batch_rc, L->batch_tgt};
  for (float* q : fl)
    if (q) cudaFree(q);
  if (L->gstat) cudaFree(L->gstat);
  for (int l = 0; l < kNumLayers; ++l) {
    if (L->wf[l]) cudaFree(L->wf[l]);
    if (L->wt[l]) cudaFree(L->wt[l]);
  }
  for (auto& s : L->systems)
    if (s.cop) cudaFree(s.cop);
  work_free(L->inf);
  work_free(L->train);
  work_free(L->eval);
  delete L;
  c->net = nullptr;
}

}  // namespace pf

// ===========================================================================
// C ABI

using namespace pf;

extern "C" {

size_t pf_learned_num_params(void) {
  size_t o = 0;
  for (int l = 0; l < kNumLayers; ++l) o += (size_t)27 * kLayers[l].cin * kLayers[l].cout + kLayers[l].cout;
  return o;
}

int pf_learned_init(pf_ctx* ctx, unsigned long long seed) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  int rc = 0;
  LearnedState* L = get_state(ctx, &rc);
  if (!L) return rc;
  std::vector<float> h(L->nparams, 0.0f);
  unsigned long long s = seed ^ 0xD1B54A32D192ED03ull;
  for (int l = 0; l < kNumLayers; ++l) {
    const int ci = kLayers[l].cin, co = kLayers[l].cout;
    // He normal over the used inputs for the ReLU layers, 1/fan-in for the
    // linear ones; the gate layer starts near 1 (bias 1, small weights)
    const int fan = 27 * (l == L_E0A ? 19 : ci);
    double sd = kLayers[l].relu ? std::sqrt(2.0 / fan) : std::sqrt(1.0 / fan);
    if (l == L_OUT) sd *= 0.1;
    for (size_t q = 0; q < (size_t)27 * ci * co; ++q) {
      const double u1 = uniform01(s), u2 = uniform01(s);
      h[L->woff[l] + q] = (float)(sd * std::sqrt(-2.0 * std::log(u1 + 1e-300)) * std::cos(6.283185307179586 * u2));
    }
    if (l == L_OUT)
      for (int q = 0; q < co; ++q) h[L->boff[l] + q] = 1.0f;
  }
  PF_CUDA_TRY(cudaMemcpyAsync(L->params, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  PF_CUDA_TRY(cudaMemsetAsync(L->adam_m, 0, L->nparams * sizeof(float), ctx->stream));
  PF_CUDA_TRY(cudaMemsetAsync(L->adam_v, 0, L->nparams * sizeof(float), ctx->stream));
  PF_CUDA_TRY(cudaMemsetAsync(L->gstat, 0, 4 * sizeof(double), ctx->stream));
  L->adam_step = 0;
  rc = repack(ctx, L);
  if (rc) return rc;
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  L->loaded = 1;
  return PF_OK;
}

int pf_learned_load(pf_ctx* ctx, const float* params, size_t n) {
  if (!ctx || !params) return PF_ERR_INVALID;
  if (n != pf_learned_num_params()) return set_error(ctx, PF_ERR_INVALID, "pf_learned_load: wrong parameter count");
  for (size_t q = 0; q < n; ++q)
    if (!std::isfinite(params[q])) return set_error(ctx, PF_ERR_INVALID, "pf_learned_load: non-finite parameter");
  cudaSetDevice(ctx->device);
  int rc = 0;
  LearnedState* L = get_state(ctx, &rc);
  if (!L) return rc;
  PF_CUDA_TRY(cudaMemcpyAsync(L->params, params, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  PF_CUDA_TRY(cudaMemsetAsync(L->adam_m, 0, n * sizeof(float), ctx->stream));
  PF_CUDA_TRY(cudaMemsetAsync(L->adam_v, 0, n * sizeof(float), ctx->stream));
  PF_CUDA_TRY(cudaMemsetAsync(L->gstat, 0, 4 * sizeof(double), ctx->stream));
  L->adam_step = 0;
  rc = repack(ctx, L);
  if (rc) return rc;
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  L->loaded = 1;
  return PF_OK;
}

int pf_learned_params(pf_ctx* ctx, float* out, size_t n) {
  if (!ctx || !out) return PF_ERR_INVALID;
  if (!coarse_net_ready(ctx)) return set_error(ctx, PF_ERR_INVALID, "no learned network loaded");
  if (n != pf_learned_num_params()) return set_error(ctx, PF_ERR_INVALID, "pf_learned_params: wrong parameter count");
  cudaSetDevice(ctx->device);
  LearnedState* L = ((CoarseCtx*)ctx->learned)->net;
  PF_CUDA_TRY(cudaMemcpyAsync(out, L->params, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return PF_OK;
}

int pf_learned_harvest(pf_ctx* ctx, int enable, int stride, int max_per_system, size_t capacity_floats) {
  if (!ctx || stride < 1 || max_per_system < 0) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  int rc = 0;
  LearnedState* L = get_state(ctx, &rc);
  if (!L) return rc;
  L->harvesting = enable ? 1 : 0;
  L->harvest_stride = stride;
  L->harvest_max = max_per_system;
  if (enable && capacity_floats > L->pool_cap) {
    PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    float* np = nullptr;
    PF_CUDA_TRY(cudaMalloc(&np, capacity_floats * sizeof(float)));
    if (L->pool_used) PF_CUDA_TRY(cudaMemcpy(np, L->pool, L->pool_used * sizeof(float), cudaMemcpyDeviceToDevice));
    if (L->pool) cudaFree(L->pool);
    L->pool = np;
    L->pool_cap = capacity_floats;
  }
  return PF_OK;
}

int pf_learned_dataset(pf_ctx* ctx, int* systems, int* pairs) {
  if (!ctx) return PF_ERR_INVALID;
  const CoarseCtx* c = (const CoarseCtx*)ctx->learned;
  int ns = 0, np = 0;
  if (c && c->net) {
    for (const auto& s : c->net->systems) {
      if (s.pairs.empty()) continue;
      ++ns;
      np += (int)s.pairs.size();
    }
  }
  if (systems) *systems = ns;
  if (pairs) *pairs = np;
  return PF_OK;
}

// Append src's training set (systems and pairs) to dst's; both contexts must
// live on the same device.  Lets one optimiser train on grids of several sizes.
int pf_learned_merge_dataset(pf_ctx* dst, pf_ctx* src) {
  if (!dst || !src || dst == src) return PF_ERR_INVALID;
  pf_ctx* ctx = dst;  // errors are reported on the destination
  if (dst->device != src->device) return set_error(ctx, PF_ERR_INVALID, "merge: contexts on different devices");
  const CoarseCtx* cs = (const CoarseCtx*)src->learned;
  if (!cs || !cs->net || cs->net->systems.empty()) return PF_OK;
  cudaSetDevice(dst->device);
  int rc = 0;
  LearnedState* D = get_state(dst, &rc);
  if (!D) return rc;
  const LearnedState* S = cs->net;
  PF_CUDA_TRY(cudaStreamSynchronize(src->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(dst->stream));
  const size_t need = D->pool_used + S->pool_used;
  if (need > D->pool_cap) {
    float* np = nullptr;
    PF_CUDA_TRY(cudaMalloc(&np, need * sizeof(float)));
    if (D->pool_used) PF_CUDA_TRY(cudaMemcpy(np, D->pool, D->pool_used * sizeof(float), cudaMemcpyDeviceToDevice));
    if (D->pool) cudaFree(D->pool);
    D->pool = np;
    D->pool_cap = need;
  }
  if (S->pool_used)
    PF_CUDA_TRY(cudaMemcpy(D->pool + D->pool_used, S->pool, S->pool_used * sizeof(float), cudaMemcpyDeviceToDevice));
  for (const auto& s : S->systems) {
    if (s.pairs.empty()) continue;
    LearnedState::System t;
    t.d = s.d;
    const size_t bytes = (size_t)s.d.n * kCopStride * sizeof(float);
    PF_CUDA_TRY(cudaMalloc(&t.cop, bytes));
    PF_CUDA_TRY(cudaMemcpy(t.cop, s.cop, bytes, cudaMemcpyDeviceToDevice));
    for (size_t off : s.pairs) t.pairs.push_back(off + D->pool_used);
    D->systems.push_back(t);
  }
  D->pool_used = need;
  return PF_OK;
}

int pf_learned_clear_dataset(pf_ctx* ctx) {
  if (!ctx) return PF_ERR_INVALID;
  CoarseCtx* c = (CoarseCtx*)ctx->learned;
  if (!c || !c->net) return PF_OK;
  cudaSetDevice(ctx->device);
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  for (auto& s : c->net->systems)
    if (s.cop) cudaFree(s.cop);
  c->net->systems.clear();
  c->net->pool_used = 0;
  return PF_OK;
}

int pf_learned_train(pf_ctx* ctx, int steps, int batch, double lr, unsigned long long seed, double* losses) {
  if (!ctx || steps < 0 || batch < 1 || !(lr > 0.0)) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  CoarseCtx* c = (CoarseCtx*)ctx->learned;
  if (!coarse_net_ready(ctx)) return set_error(ctx, PF_ERR_INVALID, "pf_learned_train: initialise or load first");
  LearnedState* L = c->net;
  std::vector<int> usable;
  int maxn = 0;
  for (int q = 0; q < (int)L->systems.size(); ++q)
    if (!L->systems[q].pairs.empty()) {
      usable.push_back(q);
      maxn = std::max(maxn, L->systems[q].d.n);
    }
  if (usable.empty()) return set_error(ctx, PF_ERR_INVALID, "pf_learned_train: empty training set");
  const size_t need = (size_t)batch * maxn * 2;
  if (L->batch_cap < need) {
    if (L->batch_rc) cudaFree(L->batch_rc);
    if (L->batch_tgt) cudaFree(L->batch_tgt);
    L->batch_rc = L->batch_tgt = nullptr;
    PF_CUDA_TRY(cudaMalloc(&L->batch_rc, need * sizeof(float)));
    PF_CUDA_TRY(cudaMalloc(&L->batch_tgt, need * sizeof(float)));
    L->batch_cap = need;
  }
  unsigned long long s = seed ^ 0xA0761D6478BD642Full;
  std::vector<double> hl(batch);
  for (int it = 0; it < steps; ++it) {
    const LearnedState::System& sys = L->systems[usable[splitmix(s) % usable.size()]];
    const size_t n2 = 2 * (size_t)sys.d.n;
    for (int b = 0; b < batch; ++b) {
      const size_t off = sys.pairs[splitmix(s) % sys.pairs.size()];
      PF_CUDA_TRY(cudaMemcpyAsync(L->batch_rc + b * n2, L->pool + off, n2 * sizeof(float), cudaMemcpyDeviceToDevice,
                                  ctx->stream));
      PF_CUDA_TRY(cudaMemcpyAsync(L->batch_tgt + b * n2, L->pool + off + n2, n2 * sizeof(float),
                                  cudaMemcpyDeviceToDevice, ctx->stream));
    }
    int rc = work_ensure(ctx, L->train, sys.d, batch, true);
    if (rc) return rc;
    rc = loss_backward(ctx, L, L->train, sys.cop, L->batch_rc, L->batch_tgt);
    if (rc) return rc;
    rc = adam_step(ctx, L, lr, true);
    if (rc) return rc;
    if (losses) {
      PF_CUDA_TRY(cudaMemcpyAsync(hl.data(), L->train.loss, batch * sizeof(double), cudaMemcpyDeviceToHost,
                                  ctx->stream));
      PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
      double m = 0.0;
      for (double v : hl) m += v;
      losses[it] = m / batch;
    }
  }
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return PF_OK;
}

// The learned correction on a caller-given coarse system (tests, gradient
// checks): e for B residuals; with a target also the mean loss and the
// parameter gradient.
int pf_learned_eval(pf_ctx* ctx, int X, int Y, int Z, const float* cop, const float* rc, const float* target,
                    int B, float* e_out, double* loss_out, float* grad_out) {
  if (!ctx || X < 1 || Y < 1 || Z < 1 || B < 1 || !cop || !rc || !e_out) return PF_ERR_INVALID;
  if (!coarse_net_ready(ctx)) return set_error(ctx, PF_ERR_INVALID, "no learned network loaded");
  cudaSetDevice(ctx->device);
  LearnedState* L = ((CoarseCtx*)ctx->learned)->net;
  const Dims d = make_dims(X, Y, Z);
  int r = work_ensure(ctx, L->eval, d, B, target != nullptr);
  if (r) return r;
  float *dcop = nullptr, *drc = nullptr, *dtg = nullptr;
  const size_t n2 = (size_t)B * d.n * 2;
  PF_CUDA_TRY(cudaMalloc(&dcop, (size_t)d.n * kCopStride * sizeof(float)));
  PF_CUDA_TRY(cudaMalloc(&drc, n2 * sizeof(float)));
  PF_CUDA_TRY(cudaMemcpyAsync(dcop, cop, (size_t)d.n * kCopStride * sizeof(float), cudaMemcpyHostToDevice,
                              ctx->stream));
  PF_CUDA_TRY(cudaMemcpyAsync(drc, rc, n2 * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  if (target) {
    PF_CUDA_TRY(cudaMalloc(&dtg, n2 * sizeof(float)));
    PF_CUDA_TRY(cudaMemcpyAsync(dtg, target, n2 * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    r = loss_backward(ctx, L, L->eval, dcop, drc, dtg);
  } else {
    r = unet_forward(ctx, L, L->eval, dcop, nullptr);
    r = r ? r : gtg_forward(ctx, L, L->eval, dcop, drc, L->eval.e, nullptr);
  }
  if (!r) {
    PF_CUDA_TRY(cudaMemcpyAsync(e_out, L->eval.e, n2 * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    if (target && grad_out)
      PF_CUDA_TRY(cudaMemcpyAsync(grad_out, L->grads, L->nparams * sizeof(float), cudaMemcpyDeviceToHost,
                                  ctx->stream));
    std::vector<double> hl(B, 0.0);
    if (target)
      PF_CUDA_TRY(cudaMemcpyAsync(hl.data(), L->eval.loss, B * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (loss_out) {
      double m = 0.0;
      for (double v : hl) m += v;
      *loss_out = m / B;
    }
  }
  cudaFree(dcop);
  cudaFree(drc);
  if (dtg) cudaFree(dtg);
  return r;
}

// One Adam step with a caller-given gradient (tests of the optimiser).
int pf_learned_adam(pf_ctx* ctx, const float* grad, size_t n, double lr) {
  if (!ctx || !grad || !(lr > 0.0)) return PF_ERR_INVALID;
  if (!coarse_net_ready(ctx)) return set_error(ctx, PF_ERR_INVALID, "no learned network loaded");
  if (n != pf_learned_num_params()) return set_error(ctx, PF_ERR_INVALID, "pf_learned_adam: wrong parameter count");
  cudaSetDevice(ctx->device);
  LearnedState* L = ((CoarseCtx*)ctx->learned)->net;
  PF_CUDA_TRY(cudaMemcpyAsync(L->grads, grad, n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  int r = adam_step(ctx, L, lr, false);
  if (r) return r;
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return PF_OK;
}

}  // extern "C"
