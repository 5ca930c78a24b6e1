// pf_learned_kernels.cuh -- device kernels of the learned coarse solve
// (included by pf_learned.cu only).
//
// Every convolution is a 3x3x3 implicit GEMM on the tensor cores
// (mma.sync m16n8k16, BF16 operands, FP32 accumulation): M = positions,
// N = output channels, K = 27 taps x input channels.  Activations are FP32 in
// HBM, channels-last with the channel stride padded to 16; the operands are
// rounded to BF16 when the fragments are built.  Weights keep an FP32 master
// copy (Adam) and are repacked into BF16 fragment order after every update.
#pragma once

#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "pf_coarse.cuh"
#include "pf_solver.cuh"

namespace pf {

namespace {

struct LayerSpec {
  int cin, cout, relu, bias;
};
// gate U-Net (layers 0-11), then the linear operator G (layers 12-15, no bias)
constexpr int kNumLayers = 16;
constexpr LayerSpec kLayers[kNumLayers] = {
    {32, 16, 1, 1}, {16, 16, 1, 1}, {16, 32, 1, 1}, {32, 32, 1, 1}, {32, 64, 1, 1}, {64, 64, 1, 1},
    {64, 64, 1, 1}, {64, 64, 1, 1}, {128, 64, 1, 1}, {96, 32, 1, 1}, {48, 16, 1, 1}, {16, 16, 0, 1},
    {2, 16, 0, 0},  {16, 16, 0, 0}, {16, 16, 0, 0}, {16, 16, 0, 0}};
enum { L_E0A, L_E0B, L_E1A, L_E1B, L_E2A, L_E2B, L_E3A, L_E3B, L_D2, L_D1, L_D0, L_OUT, L_G0, L_G1, L_G2, L_G3 };
constexpr int kInCh = 32;
constexpr int kGS = 16;  // channels (and channel stride) of every tensor of the G path

__host__ __device__ constexpr int pad16(int c) { return (c + 15) & ~15; }
__host__ __device__ constexpr int pad8(int c) { return (c + 7) & ~7; }

struct Dims {
  int X, Y, Z, n;
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16(float* c, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// tap k = (dz+1)*9 + (dy+1)*3 + (dx+1)
__device__ __forceinline__ int tap_dx(int k) { return k % 3 - 1; }
__device__ __forceinline__ int tap_dy(int k) { return (k / 3) % 3 - 1; }
__device__ __forceinline__ int tap_dz(int k) { return k / 9 - 1; }

// Position p + tap within the same sample, or -1 outside the lattice.
__device__ __forceinline__ int neighbor(const Dims& d, int b, int x, int y, int z, int k) {
  const int xx = x + tap_dx(k), yy = y + tap_dy(k), zz = z + tap_dz(k);
  if (xx < 0 || yy < 0 || zz < 0 || xx >= d.X || yy >= d.Y || zz >= d.Z) return -1;
  return b * d.n + xx + d.X * (yy + d.Y * zz);
}

// ---------------------------------------------------------------------------
// weight packing: FP32 master W[27][cin][cout] -> BF16 B fragments
//   fwd: (tap, kc, nt, lane) -> {W[tap][kc*16+2t(+1)][nt*8+g], W[tap][kc*16+2t+8(+9)][nt*8+g]}
//   bwd: the same for W'[tap][co][ci] = W[26 - tap][ci][co] (transposed, flipped)

__global__ void k_pack(const float* W, int cin, int cout, int transpose, uint2* out) {
  const int ci_n = transpose ? cout : cin;   // GEMM K extent (input channels of this conv)
  const int co_n = transpose ? cin : cout;   // GEMM N extent
  const int KC = pad16(ci_n) / 16, NT = pad8(co_n) / 8;
  const int total = 27 * KC * NT * 32;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += gridDim.x * blockDim.x) {
    const int lane = q & 31;
    int r = q >> 5;
    const int nt = r % NT;
    r /= NT;
    const int kc = r % KC;
    const int tap = r / KC;
    const int g = lane >> 2, t = lane & 3;
    const int n = nt * 8 + g;
    float v[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int k = kc * 16 + 2 * t + (e & 1) + (e >> 1) * 8;
      float w = 0.0f;
      if (k < ci_n && n < co_n) {
        w = transpose ? W[((size_t)(26 - tap) * cin + n) * cout + k] : W[((size_t)tap * cin + k) * cout + n];
      }
      v[e] = w;
    }
    out[q] = make_uint2(pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]));
  }
}

// ---------------------------------------------------------------------------
// convolution: y[p][co] = act(bias[co] + sum_tap sum_ci x[p+tap][ci] w[tap][ci][co])

struct ConvArgs {
  const float* x;
  const float* gate;  // optional: x counts only where gate > 0 (ReLU backward)
  int xs;             // channel stride of x and gate (multiple of 16) = 16 * KC
  const uint2* wf;
  const float* bias;  // optional
  int cout, relu;
  float* y;
  int ys;             // channel stride of y (multiple of 16, >= NT*8)
  Dims d;
  int P;              // positions (batch * d.n)
  const SolveCtl* skip;
  const float* gmul;  // optional: y = gmul[p mod d.n] * acc (one sample, stride ys; layers without bias/ReLU)
  int stage_w;        // brick kernel: copy the weight fragments to shared memory first
};

// ---------------------------------------------------------------------------
// The input is staged once per CTA: a CTA owns a 4x4x4
// brick of positions of one sample and loads the brick plus its one-position
// halo (6x6x6 positions, every input channel, gated) into shared memory as
// BF16; the 27 taps then read their A fragments from there.  Warp w computes
// z-slice w of the brick (16 positions = the M rows of one mma tile).

constexpr int kBrick = 4;
constexpr int kHalo = kBrick + 2;
constexpr int kHaloN = kHalo * kHalo * kHalo;

__host__ __device__ constexpr int brick_pitch(int KC) { return KC * 16 + 8; }  // BF16 per halo position
__host__ __device__ constexpr int brick_smem_halo(int KC) { return (kHaloN * brick_pitch(KC) * 2 + 15) & ~15; }
// weight fragments of a layer with KC input and NT output chunks, in bytes
__host__ __device__ constexpr int brick_smem_w(int KC, int NT) { return 27 * KC * NT * 32 * 8; }
constexpr int kStageWeightsMax = 16 * 1024;  // stage weight fragments up to this size

template <int NT>
__global__ void __launch_bounds__(128) k_conv_brick(ConvArgs a, int bx, int by, int bz) {
  if (a.skip && a.skip->done) return;
  extern __shared__ __align__(16) unsigned char conv_smem[];
  __nv_bfloat16* S = reinterpret_cast<__nv_bfloat16*>(conv_smem);
  const int KC = a.xs / 16;
  const int pitch = brick_pitch(KC);
  int brick = blockIdx.x;
  const int per_sample = bx * by * bz;
  const int b = brick / per_sample;
  brick -= b * per_sample;
  const int X0 = (brick % bx) * kBrick, Y0 = ((brick / bx) % by) * kBrick, Z0 = (brick / (bx * by)) * kBrick;
  // small layers also stage their weight fragments (after the halo block)
  const int nw = a.stage_w ? 27 * KC * NT * 32 : 0;
  uint2* SW = reinterpret_cast<uint2*>(conv_smem + brick_smem_halo(KC));
  for (int e = threadIdx.x; e < nw; e += blockDim.x) SW[e] = __ldg(a.wf + e);
  // stage the halo block, two channels per item
  const int half = a.xs / 2;
#pragma unroll 4
  for (int e = threadIdx.x; e < kHaloN * half; e += blockDim.x) {
    const int hp = e / half, c2 = (e - hp * half) * 2;
    const int x = X0 + hp % kHalo - 1, y = Y0 + (hp / kHalo) % kHalo - 1, z = Z0 + hp / (kHalo * kHalo) - 1;
    float2 v = make_float2(0.0f, 0.0f);
    if (x >= 0 && y >= 0 && z >= 0 && x < a.d.X && y < a.d.Y && z < a.d.Z) {
      const size_t q = (size_t)b * a.d.n + x + (size_t)a.d.X * (y + (size_t)a.d.Y * z);
      v = *reinterpret_cast<const float2*>(a.x + q * a.xs + c2);
      if (a.gate) {
        const float2 gv = *reinterpret_cast<const float2*>(a.gate + q * a.xs + c2);
        if (!(gv.x > 0.0f)) v.x = 0.0f;
        if (!(gv.y > 0.0f)) v.y = 0.0f;
      }
    }
    *reinterpret_cast<uint32_t*>(S + (size_t)hp * pitch + c2) = pack_bf16(v.x, v.y);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  // rows g and g + 8 of this warp's 16 positions: (x, y) = (g % 4, g / 4) and (g % 4, g / 4 + 2), z = warp
  const int lx = g & 3, ly0 = g >> 2, ly1 = ly0 + 2, lz = warp;
  float acc[NT][4];
#pragma unroll
  for (int j = 0; j < NT; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
  for (int k = 0; k < 27; ++k) {
    const int hx = lx + 1 + tap_dx(k), hz = lz + 1 + tap_dz(k);
    const int hp0 = hx + kHalo * (ly0 + 1 + tap_dy(k) + kHalo * hz);
    const int hp1 = hx + kHalo * (ly1 + 1 + tap_dy(k) + kHalo * hz);
    const __nv_bfloat16* r0 = S + (size_t)hp0 * pitch + 2 * t;
    const __nv_bfloat16* r1 = S + (size_t)hp1 * pitch + 2 * t;
    for (int kc = 0; kc < KC; ++kc) {
      const uint32_t a0 = *reinterpret_cast<const uint32_t*>(r0 + kc * 16);
      const uint32_t a1 = *reinterpret_cast<const uint32_t*>(r1 + kc * 16);
      const uint32_t a2 = *reinterpret_cast<const uint32_t*>(r0 + kc * 16 + 8);
      const uint32_t a3 = *reinterpret_cast<const uint32_t*>(r1 + kc * 16 + 8);
      const size_t wo = ((size_t)(k * KC + kc) * NT) * 32 + lane;
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        const uint2 bw = nw ? SW[wo + j * 32] : __ldg(a.wf + wo + j * 32);
        mma_bf16(acc[j], a0, a1, a2, a3, bw.x, bw.y);
      }
    }
  }
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int x = X0 + lx, y = Y0 + (h ? ly1 : ly0), z = Z0 + lz;
    if (x >= a.d.X || y >= a.d.Y || z >= a.d.Z) continue;
    const int tpos = x + a.d.X * (y + a.d.Y * z);
    float* yr = a.y + ((size_t)b * a.d.n + tpos) * a.ys;
    const float* gr = a.gmul ? a.gmul + (size_t)tpos * a.ys : nullptr;
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      const int c0 = j * 8 + 2 * t;
      float o0 = acc[j][2 * h], o1 = acc[j][2 * h + 1];
      if (gr) {
        o0 *= gr[c0];
        o1 *= gr[c0 + 1];
      }
      if (c0 < a.cout) {
        if (a.bias) o0 += a.bias[c0];
        if (a.relu) o0 = fmaxf(o0, 0.0f);
      } else {
        o0 = 0.0f;
      }
      if (c0 + 1 < a.cout) {
        if (a.bias) o1 += a.bias[c0 + 1];
        if (a.relu) o1 = fmaxf(o1, 0.0f);
      } else {
        o1 = 0.0f;
      }
      *reinterpret_cast<float2*>(yr + c0) = make_float2(o0, o1);
    }
    for (int c = NT * 8 + 2 * t; c < a.ys; c += 8) *reinterpret_cast<float2*>(yr + c) = make_float2(0.0f, 0.0f);
  }
}

// ---------------------------------------------------------------------------
// weight gradient: part[cta][tap][ci][co] = sum_{p in the CTA's chunks} x[p+tap][ci] dz[p][co]
// with dz = dy (gated by y > 0 for ReLU layers).  Grid (nctas, 27), 8 warps;
// each chunk of 64 positions is staged transposed in shared memory as BF16.

constexpr int kWChunk = 64;
constexpr int kWPitch = kWChunk + 8;  // BF16 elements per staged row (bank-conflict-free fragments)

struct WgradArgs {
  const float* x;
  int xs, cin;
  const float* dy;
  const float* gate;
  int ds, cout;
  float* part;
  Dims d;
  int P;
};

__global__ void __launch_bounds__(256) k_wgrad(WgradArgs a) {
  __shared__ __align__(16) __nv_bfloat16 XT[128][kWPitch];
  __shared__ __align__(16) __nv_bfloat16 DT[64][kWPitch];
  const int tap = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int MT = pad16(a.cin) / 16, NTt = pad8(a.cout) / 8;
  const int cin16 = MT * 16, cout8 = NTt * 8;
  const int tiles = MT * NTt;
  float acc[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
  const int nchunks = (a.P + kWChunk - 1) / kWChunk;
  for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
    __syncthreads();
    for (int e = threadIdx.x; e < kWChunk * cin16; e += blockDim.x) {
      const int pl = e / cin16, ci = e - pl * cin16;
      const int p = c * kWChunk + pl;
      float v = 0.0f;
      if (p < a.P && ci < a.cin) {
        const int b = p / a.d.n, tt = p - b * a.d.n;
        const int q = neighbor(a.d, b, tt % a.d.X, (tt / a.d.X) % a.d.Y, tt / (a.d.X * a.d.Y), tap);
        if (q >= 0) v = a.x[(size_t)q * a.xs + ci];
      }
      XT[ci][pl] = __float2bfloat16_rn(v);
    }
    for (int e = threadIdx.x; e < kWChunk * cout8; e += blockDim.x) {
      const int pl = e / cout8, co = e - pl * cout8;
      const int p = c * kWChunk + pl;
      float v = 0.0f;
      if (p < a.P && co < a.cout) {
        v = a.dy[(size_t)p * a.ds + co];
        if (a.gate && !(a.gate[(size_t)p * a.ds + co] > 0.0f)) v = 0.0f;
      }
      DT[co][pl] = __float2bfloat16_rn(v);
    }
    __syncthreads();
    for (int j = 0; j < 8; ++j) {
      const int tile = warp + 8 * j;
      if (tile >= tiles) break;
      const int mt = tile / NTt, nt = tile - mt * NTt;
#pragma unroll
      for (int ks = 0; ks < kWChunk / 16; ++ks) {
        const int kk = ks * 16 + 2 * t;
        const uint32_t a0 = *reinterpret_cast<const uint32_t*>(&XT[mt * 16 + g][kk]);
        const uint32_t a1 = *reinterpret_cast<const uint32_t*>(&XT[mt * 16 + g + 8][kk]);
        const uint32_t a2 = *reinterpret_cast<const uint32_t*>(&XT[mt * 16 + g][kk + 8]);
        const uint32_t a3 = *reinterpret_cast<const uint32_t*>(&XT[mt * 16 + g + 8][kk + 8]);
        const uint32_t b0 = *reinterpret_cast<const uint32_t*>(&DT[nt * 8 + g][kk]);
        const uint32_t b1 = *reinterpret_cast<const uint32_t*>(&DT[nt * 8 + g][kk + 8]);
        mma_bf16(acc[j], a0, a1, a2, a3, b0, b1);
      }
    }
  }
  float* out = a.part + ((size_t)blockIdx.x * 27 + tap) * a.cin * a.cout;
  for (int j = 0; j < 8; ++j) {
    const int tile = warp + 8 * j;
    if (tile >= tiles) break;
    const int mt = tile / NTt, nt = tile - mt * NTt;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int ci = mt * 16 + g + 8 * (e >> 1), co = nt * 8 + 2 * t + (e & 1);
      if (ci < a.cin && co < a.cout) out[(size_t)ci * a.cout + co] = acc[j][e];
    }
  }
}

// dW += sum over CTA partials (fixed order)
__global__ void k_wgrad_reduce(const float* part, int nparts, int count, float* dW) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int c = 0; c < nparts; ++c) s += part[(size_t)c * count + q];
    dW[q] += s;
  }
}

// db[co] += sum_p dz[p][co], one CTA per output channel, FP64 fixed-order sums
__global__ void __launch_bounds__(256) k_bias_grad(const float* dy, const float* gate, int ds, int P, float* db) {
  const int co = blockIdx.x;
  double s = 0.0;
  for (int p = threadIdx.x; p < P; p += blockDim.x) {
    float v = dy[(size_t)p * ds + co];
    if (gate && !(gate[(size_t)p * ds + co] > 0.0f)) v = 0.0f;
    s += v;
  }
  __shared__ double sh[8];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) tot += sh[w];
    db[co] += (float)tot;
  }
}

// ---------------------------------------------------------------------------
// pooling, upsampling + concatenation, and their adjoints (B samples)

__global__ void k_pool(const float* x, int cs, Dims f, Dims c, int B, float* y, const SolveCtl* skip) {
  if (skip && skip->done) return;
  const size_t total = (size_t)B * c.n * cs;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    const int ch = (int)(q % cs);
    const size_t pc = q / cs;
    const int b = (int)(pc / c.n), tc = (int)(pc % c.n);
    const int X = tc % c.X, Y = (tc / c.X) % c.Y, Z = tc / (c.X * c.Y);
    float s = 0.0f;
    for (int dz = 0; dz < 2; ++dz)
      for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx) {
          const int xx = 2 * X + dx, yy = 2 * Y + dy, zz = 2 * Z + dz;
          if (xx < f.X && yy < f.Y && zz < f.Z) s += x[((size_t)b * f.n + xx + f.X * (yy + f.Y * zz)) * cs + ch];
        }
    y[q] = s * 0.125f;
  }
}

// dx[child] += dy[parent] / 8
__global__ void k_pool_bwd(const float* dy, int cs, Dims f, Dims c, int B, float* dx) {
  const size_t total = (size_t)B * f.n * cs;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    const int ch = (int)(q % cs);
    const size_t pf = q / cs;
    const int b = (int)(pf / f.n), tf = (int)(pf % f.n);
    const int x = tf % f.X, y = (tf / f.X) % f.Y, z = tf / (f.X * f.Y);
    const size_t pc = (size_t)b * c.n + (x >> 1) + c.X * ((y >> 1) + c.Y * (z >> 1));
    dx[q] += dy[pc * cs + ch] * 0.125f;
  }
}

// out[p] = [coarse[parent(p)][0:cu], skip[p][0:csk]] with stride cu + csk
__global__ void k_up_concat(const float* coarse, int cu, Dims c, const float* skipt, int csk, Dims f, int B,
                            float* out, const SolveCtl* skip) {
  if (skip && skip->done) return;
  const int cs = cu + csk;
  const size_t total = (size_t)B * f.n * cs;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    const int ch = (int)(q % cs);
    const size_t pf = q / cs;
    float v;
    if (ch < cu) {
      const int b = (int)(pf / f.n), tf = (int)(pf % f.n);
      const int x = tf % f.X, y = (tf / f.X) % f.Y, z = tf / (f.X * f.Y);
      const size_t pc = (size_t)b * c.n + (x >> 1) + c.X * ((y >> 1) + c.Y * (z >> 1));
      v = coarse[pc * cu + ch];
    } else {
      v = skipt[pf * csk + (ch - cu)];
    }
    out[q] = v;
  }
}

// d_coarse[parent][ch] = sum over children of dout[child][ch] (ch < cu);
// d_skip[p][ch] = dout[p][cu + ch]
__global__ void k_up_concat_bwd(const float* dout, int cu, int csk, Dims c, Dims f, int B, float* dcoarse,
                                float* dskip) {
  const int cs = cu + csk;
  const size_t tc_total = (size_t)B * c.n * cu;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < tc_total; q += (size_t)gridDim.x * blockDim.x) {
    const int ch = (int)(q % cu);
    const size_t pc = q / cu;
    const int b = (int)(pc / c.n), tc = (int)(pc % c.n);
    const int X = tc % c.X, Y = (tc / c.X) % c.Y, Z = tc / (c.X * c.Y);
    float s = 0.0f;
    for (int dz = 0; dz < 2; ++dz)
      for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx) {
          const int xx = 2 * X + dx, yy = 2 * Y + dy, zz = 2 * Z + dz;
          if (xx < f.X && yy < f.Y && zz < f.Z) s += dout[((size_t)b * f.n + xx + f.X * (yy + f.Y * zz)) * cs + ch];
        }
    dcoarse[q] = s;
  }
  const size_t ts_total = (size_t)B * f.n * csk;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < ts_total; q += (size_t)gridDim.x * blockDim.x) {
    const size_t pf = q / csk;
    const int ch = (int)(q % csk);
    dskip[q] = dout[pf * cs + cu + ch];
  }
}

// ---------------------------------------------------------------------------
// features, scales, output mapping, loss

__device__ __forceinline__ bool live(const float* cop, int t, int c) {
  return cop[(size_t)t * kCopStride + kCopN + c] > 0.0f && cop[(size_t)t * kCopStride + kCopD + c] > 0.0f;
}

// sc[b] = max over live unknowns |rc_b| (b < B); sc[B] = d_ref
__global__ void __launch_bounds__(256) k_scales(const float* cop, const float* rc, int nt, int B, float* sc,
                                                const SolveCtl* skip) {
  if (skip && skip->done) return;
  const int b = blockIdx.x;
  float m = 0.0f, m1 = 0.0f;
  for (int t = threadIdx.x; t < nt; t += blockDim.x) {
    for (int c = 0; c < 2; ++c) {
      if (!live(cop, t, c)) continue;
      if (b < B) {
        if (rc) m = fmaxf(m, fabsf(rc[((size_t)b * nt + t) * 2 + c]));
      } else {
        const float d = cop[(size_t)t * kCopStride + kCopD + c];
        if (c == 0) m = fmaxf(m, d);
        else m1 = fmaxf(m1, d);
      }
    }
  }
  __shared__ float sh[2][8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    m1 = fmaxf(m1, __shfl_down_sync(0xffffffffu, m1, o));
  }
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = m;
    sh[1][threadIdx.x >> 5] = m1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float a = 0.0f, a1 = 0.0f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a = fmaxf(a, sh[0][w]);
      a1 = fmaxf(a1, sh[1][w]);
    }
    sc[b] = (b < B || a > 0.0f) ? a : a1;
  }
}

__global__ void k_features(const float* cop, const float* rc, Dims d, int B, const float* sc, float* F,
                           const SolveCtl* skip) {
  if (skip && skip->done) return;
  const size_t total = (size_t)B * d.n;
  const float inv_log = 1.0f / logf(1e4f);
  const float dref = sc[B];
  for (size_t p = blockIdx.x * (size_t)blockDim.x + threadIdx.x; p < total; p += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(p / d.n), t = (int)(p % d.n);
    const float s = sc[b];
    const float inv_s = s > 0.0f ? 1.0f / s : 0.0f;
    float f[kInCh];
#pragma unroll
    for (int c = 0; c < kInCh; ++c) f[c] = 0.0f;
    const float* R = cop + (size_t)t * kCopStride;
    const bool l0 = live(cop, t, 0), l1 = live(cop, t, 1);
    const bool lv[2] = {l0, l1};
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      if (!lv[c]) continue;
      f[c] = rc ? rc[((size_t)b * d.n + t) * 2 + c] * inv_s : 0.0f;
      f[2 + c] = 1.0f;
      f[4 + c] = dref > 0.0f ? logf(R[kCopD + c] / dref) * inv_log : 0.0f;
    }
    if (l0 && l1) f[6] = R[kCopE] / sqrtf(R[kCopD] * R[kCopD + 1]);
    const int x = t % d.X, y = (t / d.X) % d.Y, z = t / (d.X * d.Y);
    const int has[3] = {x > 0, y > 0, z > 0};
    const int step[3] = {1, d.X, d.X * d.Y};
    const int base[3] = {kCopX, kCopY, kCopZ};
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      if (!has[q]) continue;
      const int u = t - step[q];
      const float* Ru = cop + (size_t)u * kCopStride;
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int bb = 0; bb < 2; ++bb)
          if (lv[a] && live(cop, u, bb))
            f[7 + 4 * q + 2 * a + bb] = R[base[q] + 2 * a + bb] / sqrtf(R[kCopD + a] * Ru[kCopD + bb]);
    }
    float4* out = reinterpret_cast<float4*>(F + p * kInCh);
#pragma unroll
    for (int c = 0; c < kInCh / 4; ++c) out[c] = make_float4(f[4 * c], f[4 * c + 1], f[4 * c + 2], f[4 * c + 3]);
  }
}

// ---------------------------------------------------------------------------
// the G path: e = S G^T G S rc, S = diag(d_c^-1/2) on live unknowns

__device__ __forceinline__ float inv_sqrt_diag(const float* cop, int t, int c) {
  return live(cop, t, c) ? rsqrtf(cop[(size_t)t * kCopStride + kCopD + c]) : 0.0f;
}

// out[p][0:2] = S * in[p][0:2] (in: [B][nt][2] packed, or stride-16 when in_stride16), channels 2..15 = 0
__global__ void k_scale_in(const float* in, int in_stride16, const float* cop, int nt, int B, float* out,
                           const SolveCtl* skip) {
  if (skip && skip->done) return;
  const size_t total = (size_t)B * nt * kGS;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(q % kGS);
    const size_t p = q / kGS;
    float v = 0.0f;
    if (c < 2) {
      const int t = (int)(p % nt);
      v = inv_sqrt_diag(cop, t, c) * (in_stride16 ? in[p * kGS + c] : in[p * 2 + c]);
    }
    out[q] = v;
  }
}

// e[p][c] = S * w[p][c] for c < 2 (w has stride 16)
__global__ void k_scale_out(const float* w, const float* cop, int nt, int B, float* e, const SolveCtl* skip) {
  if (skip && skip->done) return;
  const size_t total = (size_t)B * nt * 2;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    const int c = (int)(q & 1);
    const size_t p = q >> 1;
    e[q] = inv_sqrt_diag(cop, (int)(p % nt), c) * w[p * kGS + c];
  }
}

// out = g * a, g shared by the B samples ([n][16])
__global__ void k_gmul(float* out, const float* g, const float* a, int n, int B, const SolveCtl* skip) {
  if (skip && skip->done) return;
  const size_t total = (size_t)B * n * kGS;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x)
    out[q] = g[q % ((size_t)n * kGS)] * a[q];
}

// b = h + P^T v (v on the coarser level: each child gets v[parent] / 8); t = g * b
__global__ void k_up_add_gate(const float* h, const float* v, const float* g, Dims f, Dims c, int B, float* b,
                              float* t, const SolveCtl* skip) {
  if (skip && skip->done) return;
  const size_t total = (size_t)B * f.n * kGS;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x) {
    const int ch = (int)(q % kGS);
    const size_t pf = q / kGS;
    const int bb = (int)(pf / f.n), tf = (int)(pf % f.n);
    const int x = tf % f.X, y = (tf / f.X) % f.Y, z = tf / (f.X * f.Y);
    const size_t pc = (size_t)bb * c.n + (x >> 1) + c.X * ((y >> 1) + c.Y * (z >> 1));
    const float bv = h[q] + v[pc * kGS + ch] * 0.125f;
    if (b) b[q] = bv;
    t[q] = g[(size_t)tf * kGS + ch] * bv;
  }
}

// dg[i] += sum_b u[b][i] v[b][i]  (i over n * 16)
__global__ void k_gate_grad(float* dg, const float* u, const float* v, int n, int B) {
  const size_t m = (size_t)n * kGS;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int b = 0; b < B; ++b) s += u[(size_t)b * m + i] * v[(size_t)b * m + i];
    dg[i] += s;
  }
}

// out += in (B samples, stride 16)
__global__ void k_add(float* out, const float* in, size_t total) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < total; q += (size_t)gridDim.x * blockDim.x)
    out[q] += in[q];
}

template <typename T>
__device__ __forceinline__ double capply(const float* cop, const Dims& d, const T* x, int t, int c) {
  const int tx = t % d.X, q = t / d.X, ty = q % d.Y, tz = q / d.Y;
  const float* R = cop + (size_t)t * kCopStride;
  double y = (double)R[kCopD + c] * (double)x[2 * t + c] - (double)R[kCopE] * (double)x[2 * t + 1 - c];
  const int step[3] = {1, d.X, d.X * d.Y};
  const int has_lo[3] = {tx > 0, ty > 0, tz > 0};
  const int has_hi[3] = {tx + 1 < d.X, ty + 1 < d.Y, tz + 1 < d.Z};
  const int base[3] = {kCopX, kCopY, kCopZ};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (has_lo[a]) {
      const int u = t - step[a];
      y -= (double)R[base[a] + 2 * c] * (double)x[2 * u] + (double)R[base[a] + 2 * c + 1] * (double)x[2 * u + 1];
    }
    if (has_hi[a]) {
      const int u = t + step[a];
      const float* Ru = cop + (size_t)u * kCopStride;
      y -= (double)Ru[base[a] + c] * (double)x[2 * u] + (double)Ru[base[a] + 2 + c] * (double)x[2 * u + 1];
    }
  }
  return y;
}

// v = e - target (live), per-sample den = target . rc (live)
__global__ void __launch_bounds__(256) k_loss_prep(const float* e, const float* tgt, const float* rc,
                                                   const float* cop, int nt, double* v, double* den) {
  const int b = blockIdx.x;
  double s = 0.0;
  for (int q = threadIdx.x; q < 2 * nt; q += blockDim.x) {
    const int t = q >> 1, c = q & 1;
    const size_t o = (size_t)b * 2 * nt + q;
    if (live(cop, t, c)) {
      v[o] = (double)e[o] - (double)tgt[o];
      s += (double)tgt[o] * (double)rc[o];
    } else {
      v[o] = 0.0;
    }
  }
  __shared__ double sh[8];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < 8; ++w) tot += sh[w];
    den[b] = tot;
  }
}

// per sample: loss_b = v.Av / den_b; de = live ? 2 Av / den_b / B : 0 (stride 16)
__global__ void __launch_bounds__(256) k_loss_grad(const double* v, const double* den, const float* cop, Dims d,
                                                   int B, float* dout, double* loss) {
  const int b = blockIdx.x;
  const int nt = d.n;
  const double dn = den[b];
  const double scale = 1.0;
  const bool ok = dn > 0.0;
  double s = 0.0;
  for (int q = threadIdx.x; q < 2 * nt; q += blockDim.x) {
    const int t = q >> 1, c = q & 1;
    const size_t o = (size_t)b * 2 * nt + q;
    double g = 0.0;
    if (live(cop, t, c)) {
      const double av = capply(cop, d, v + (size_t)b * 2 * nt, t, c);
      s += v[o] * av;
      if (ok) g = 2.0 * av / dn / B * scale;
    }
    dout[((size_t)b * nt + t) * 16 + c] = (float)g;
  }
  __shared__ double sh[8];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < 8; ++w) tot += sh[w];
    loss[b] = ok ? tot / dn : 0.0;
  }
}

// Global gradient-norm clipping of the training loop.  gs[0] = sum of g^2
// (accumulated by k_grad_sumsq), gs[1] = the step's gradient scale, gs[2] =
// running average of the clipped norm, gs[3] = steps seen.  A non-finite
// gradient skips the step (scale 0); a norm above twice the running average
// is scaled down to it, so that one outlier batch neither moves the weights
// far nor inflates Adam's second moment for thousands of steps.
__global__ void __launch_bounds__(256) k_grad_sumsq(const float* g, size_t n, double* gs) {
  double a = 0.0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const double v = g[q];
    a += v * v;
  }
  a = warp_sum(a);
  __shared__ double sh[8];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += sh[w];
    atomicAdd(gs, t);
  }
}

__global__ void k_grad_clip(double* gs) {
  const double norm = sqrt(gs[0]);
  double scale = 1.0;
  if (!isfinite(norm)) {
    scale = 0.0;
  } else {
    const double thr = gs[3] > 0.0 ? 2.0 * gs[2] : norm;
    if (norm > thr && norm > 0.0) scale = thr / norm;
    const double clipped = norm * scale;
    gs[2] = gs[3] > 0.0 ? 0.95 * gs[2] + 0.05 * clipped : clipped;
    gs[3] += 1.0;
  }
  gs[1] = scale;
  gs[0] = 0.0;
}

// Adam; `gscale` (optional) multiplies the gradient, and a zero scale leaves
// the parameters and moments unchanged.
__global__ void k_adam(float* p, const float* g, float* m, float* v, size_t n, float lr, float b1, float b2,
                       float c1, float c2, float eps, const double* gscale) {
  const float sc = gscale ? (float)*gscale : 1.0f;
  if (sc == 0.0f) return;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const float gq = g[q] * sc;
    const float mq = b1 * m[q] + (1.0f - b1) * gq;
    const float vq = b2 * v[q] + (1.0f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    p[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
  }
}

__global__ void k_zero_f(float* p, size_t n) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    p[q] = 0.0f;
}

// ---------------------------------------------------------------------------
// The G path of the solver's coarse correction (inference), 16 channels.
//
// The general brick kernel above spends its time on per-CTA latency: runtime
// channel counts make every staged element and every tap cost index
// arithmetic, and one warp per SM sub-partition exposes each instruction's
// latency.  This kernel fixes the channel counts (16 in, 16 or 8 out), reads
// its A fragments with ldmatrix at compile-time tap offsets, stages the weight
// fragments with cp.async, and absorbs the elementwise steps between the
// convolutions into its operand staging and epilogue, so that one application
// of e = S G^T G S r_c costs 2 NL launches:
//   forward, level 0:    x = S r_c                      h_0 = g_0 * (C_0 x),  q_1 = P h_0
//   forward, level l:    x = q_l                        h_l = g_l * (C_l x),  q_{l+1} = P h_l
//   transpose, level l:  x = g_l * (h_l + P^T v_{l+1})  v_l = C_l^T x
//   transpose, level 0:  as level l, then               e = S v_0 (two channels)
// P averages the 2x2x2 children that exist (sum / 8); P^T gives each child 1/8
// of its parent; at the deepest level x = g * h.
//
// A CTA computes an 8x4x2 brick of one sample.  Warp w owns y in
// {2(w&1), 2(w&1)+1} at z = w>>1; row r of its mma tile is x = r&7,
// y = 2(w&1) + (r>>3).  A halo row holds the 16 BF16 channels of one position
// with a 48-byte pitch: the 8 rows one ldmatrix matrix reads (8 consecutive x)
// then start in 8 distinct 16-byte bank groups.  Every brick origin is even,
// so the 2x2x2 children of each pooled output lie inside one CTA.

constexpr int kGBX = 8, kGBY = 4, kGBZ = 2;
constexpr int kGHX = kGBX + 2, kGHY = kGBY + 2, kGHZ = kGBZ + 2;
constexpr int kGHN = kGHX * kGHY * kGHZ;
constexpr int kGPitch = 24;  // BF16 per halo row

enum { GIN_SCALE = 0, GIN_PLAIN = 1, GIN_TGATE = 2 };
enum { GOUT_GATE = 0, GOUT_PLAIN = 1, GOUT_SCALE = 2 };

struct GConvArgs {
  const float* x;     // GIN_SCALE: r_c [B][n][2]; GIN_PLAIN: q_l; GIN_TGATE: h_l  ([B][n][16])
  const float* vpar;  // GIN_TGATE: v_{l+1} [B][nc][16], or null at the deepest level
  const float* gate;  // g_l [n][16] (GIN_TGATE, GOUT_GATE)
  const float* cop;   // coarse operator records (GIN_SCALE, GOUT_SCALE)
  const uint2* wf;    // B fragments: 27 taps x NT x 32 lanes
  float* y;           // GOUT_GATE: h_l; GOUT_PLAIN: v_l; GOUT_SCALE: e [B][n][2]
  float* pool;        // GOUT_GATE: q_{l+1} [B][nc][16], or null at the deepest level
  Dims d, dc;         // this level, the next coarser level
  int bx, by;         // bricks along x and y
  const SolveCtl* skip;
};

__host__ __device__ constexpr int gconv_tap_offset(int k) {
  return (k % 3) + kGHX * ((k / 3) % 3 + kGHY * (k / 9));
}

__device__ __forceinline__ void ldmatrix_x4(uint32_t* r, uint32_t addr) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(addr));
}

template <int IN, int OUT, int NT>
__global__ void __launch_bounds__(128) k_gconv(GConvArgs a) {
  __shared__ __align__(16) __nv_bfloat16 S[kGHN * kGPitch];
  __shared__ __align__(16) uint2 SW[27 * NT * 32];
  __shared__ float2 zx[OUT == GOUT_GATE ? 2 * 32 * NT : 1];
  const int tid = threadIdx.x, b = blockIdx.y;
  const int brick = blockIdx.x;
  const int X0 = (brick % a.bx) * kGBX, Y0 = ((brick / a.bx) % a.by) * kGBY, Z0 = (brick / (a.bx * a.by)) * kGBZ;
  const size_t nb = (size_t)b * a.d.n;

  // weight fragments: 16-byte asynchronous copies, waited for before the mma loop
  {
    constexpr int kChunks = 27 * NT * 32 * 8 / 16;
    const char* src = reinterpret_cast<const char*>(a.wf);
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(SW);
    for (int e = tid; e < kChunks; e += 128)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst + e * 16), "l"(src + (size_t)e * 16));
    asm volatile("cp.async.commit_group;\n" ::);
  }
  // the weights are fixed during a solve, so they are copied before the wait
  // for the previous kernel of the chain (programmatic dependent launch)
  pdl_wait();
  pdl_launch_dependents();
  if (a.skip && a.skip->done) {
    asm volatile("cp.async.wait_all;\n" ::);
    return;
  }

  // operand halo (10x6x4 positions), rounded to BF16
  if (IN == GIN_SCALE) {
    for (int hp = tid; hp < kGHN; hp += 128) {
      const int x = X0 + hp % kGHX - 1, y = Y0 + (hp / kGHX) % kGHY - 1, z = Z0 + hp / (kGHX * kGHY) - 1;
      float v0 = 0.0f, v1 = 0.0f;
      if (x >= 0 && y >= 0 && z >= 0 && x < a.d.X && y < a.d.Y && z < a.d.Z) {
        const int p = x + a.d.X * (y + a.d.Y * z);
        const float2 r = *reinterpret_cast<const float2*>(a.x + (nb + p) * 2);
        v0 = inv_sqrt_diag(a.cop, p, 0) * r.x;
        v1 = inv_sqrt_diag(a.cop, p, 1) * r.y;
      }
      uint4* row = reinterpret_cast<uint4*>(S + hp * kGPitch);
      row[0] = make_uint4(pack_bf16(v0, v1), 0u, 0u, 0u);
      row[1] = make_uint4(0u, 0u, 0u, 0u);
    }
  } else {
    constexpr int kItems = kGHN * 4;  // float4 per halo row
    constexpr int kIter = (kItems + 127) / 128;
    float4 v[kIter];
#pragma unroll
    for (int i = 0; i < kIter; ++i) {
      const int e = tid + i * 128;
      v[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      const int hp = e >> 2, c = (e & 3) * 4;
      const int x = X0 + hp % kGHX - 1, y = Y0 + (hp / kGHX) % kGHY - 1, z = Z0 + hp / (kGHX * kGHY) - 1;
      if (e < kItems && x >= 0 && y >= 0 && z >= 0 && x < a.d.X && y < a.d.Y && z < a.d.Z) {
        const int p = x + a.d.X * (y + a.d.Y * z);
        float4 h = __ldg(reinterpret_cast<const float4*>(a.x + (nb + p) * kGS + c));
        if (IN == GIN_TGATE) {
          if (a.vpar) {
            const int pp = (x >> 1) + a.dc.X * ((y >> 1) + a.dc.Y * (z >> 1));
            const float4 u =
                __ldg(reinterpret_cast<const float4*>(a.vpar + ((size_t)b * a.dc.n + pp) * kGS + c));
            h.x += u.x * 0.125f;
            h.y += u.y * 0.125f;
            h.z += u.z * 0.125f;
            h.w += u.w * 0.125f;
          }
          const float4 g = __ldg(reinterpret_cast<const float4*>(a.gate + (size_t)p * kGS + c));
          h.x *= g.x;
          h.y *= g.y;
          h.z *= g.z;
          h.w *= g.w;
        }
        v[i] = h;
      }
    }
#pragma unroll
    for (int i = 0; i < kIter; ++i) {
      const int e = tid + i * 128;
      if (e < kItems)
        *reinterpret_cast<uint2*>(S + (e >> 2) * kGPitch + (e & 3) * 4) =
            make_uint2(pack_bf16(v[i].x, v[i].y), pack_bf16(v[i].z, v[i].w));
    }
  }
  asm volatile("cp.async.wait_all;\n" ::);
  __syncthreads();

  // 27 taps, A fragments prefetched kPre taps ahead, two accumulator sets (even / odd taps)
  const int warp = tid >> 5, lane = tid & 31;
  const int yp = warp & 1, wz = warp >> 1;
  const int lm = lane >> 3;
  const uint32_t abase = (uint32_t)__cvta_generic_to_shared(S) +
                         (uint32_t)(((lane & 7) + kGHX * (2 * yp + (lm & 1) + kGHY * wz)) * kGPitch + (lm >> 1) * 8) * 2;
  constexpr int kPre = 4;
  uint32_t fa[kPre][4];
#pragma unroll
  for (int k = 0; k < kPre; ++k) ldmatrix_x4(fa[k], abase + gconv_tap_offset(k) * kGPitch * 2);
  float acc[2][NT][4];
#pragma unroll
  for (int s = 0; s < 2; ++s)
#pragma unroll
    for (int j = 0; j < NT; ++j) acc[s][j][0] = acc[s][j][1] = acc[s][j][2] = acc[s][j][3] = 0.0f;
#pragma unroll
  for (int k = 0; k < 27; ++k) {
    uint32_t* f = fa[k % kPre];
    const uint32_t a0 = f[0], a1 = f[1], a2 = f[2], a3 = f[3];
    if (k + kPre < 27) ldmatrix_x4(f, abase + gconv_tap_offset(k + kPre) * kGPitch * 2);
#pragma unroll
    for (int j = 0; j < NT; ++j) {
      const uint2 bw = SW[(k * NT + j) * 32 + lane];
      mma_bf16(acc[k & 1][j], a0, a1, a2, a3, bw.x, bw.y);
    }
  }

  // epilogue: lane (g, t) holds rows g (y = Y0 + 2yp) and g + 8 (y + 1), channels j*8 + 2t, +1
  const int g = lane >> 2, t = lane & 3;
  const int x = X0 + g, z = Z0 + wz;
  float r[NT][4];
#pragma unroll
  for (int j = 0; j < NT; ++j)
#pragma unroll
    for (int q = 0; q < 4; ++q) r[j][q] = acc[0][j][q] + acc[1][j][q];
  bool inr[2];
  int pos[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int y = Y0 + 2 * yp + h;
    inr[h] = x < a.d.X && y < a.d.Y && z < a.d.Z;
    pos[h] = x + a.d.X * (y + a.d.Y * z);
  }
  if (OUT == GOUT_SCALE) {
    if (t == 0) {
#pragma unroll
      for (int h = 0; h < 2; ++h)
        if (inr[h])
          *reinterpret_cast<float2*>(a.y + (nb + pos[h]) * 2) =
              make_float2(inv_sqrt_diag(a.cop, pos[h], 0) * r[0][2 * h], inv_sqrt_diag(a.cop, pos[h], 1) * r[0][2 * h + 1]);
    }
  } else if (OUT == GOUT_PLAIN) {
#pragma unroll
    for (int h = 0; h < 2; ++h)
      if (inr[h])
#pragma unroll
        for (int j = 0; j < NT; ++j)
          *reinterpret_cast<float2*>(a.y + (nb + pos[h]) * kGS + j * 8 + 2 * t) = make_float2(r[j][2 * h], r[j][2 * h + 1]);
  } else {
    float2 s[NT];
#pragma unroll
    for (int j = 0; j < NT; ++j) s[j] = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (!inr[h]) continue;
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        const int c0 = j * 8 + 2 * t;
        const float2 gv = __ldg(reinterpret_cast<const float2*>(a.gate + (size_t)pos[h] * kGS + c0));
        const float2 hv = make_float2(gv.x * r[j][2 * h], gv.y * r[j][2 * h + 1]);
        *reinterpret_cast<float2*>(a.y + (nb + pos[h]) * kGS + c0) = hv;
        s[j].x += hv.x;
        s[j].y += hv.y;
      }
    }
    if (a.pool) {  // uniform over the CTA
#pragma unroll
      for (int j = 0; j < NT; ++j) {  // x pairs: rows g and g ^ 1
        s[j].x += __shfl_xor_sync(0xffffffffu, s[j].x, 4);
        s[j].y += __shfl_xor_sync(0xffffffffu, s[j].y, 4);
      }
      if (wz == 1)
#pragma unroll
        for (int j = 0; j < NT; ++j) zx[(yp * 32 + lane) * NT + j] = s[j];
      __syncthreads();
      const int cx = x >> 1, cy = (Y0 >> 1) + yp, cz = Z0 >> 1;
      if (wz == 0 && (g & 1) == 0 && cx < a.dc.X && cy < a.dc.Y && cz < a.dc.Z) {
        float* q = a.pool + ((size_t)b * a.dc.n + cx + (size_t)a.dc.X * (cy + (size_t)a.dc.Y * cz)) * kGS;
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          const float2 o = zx[(yp * 32 + lane) * NT + j];
          *reinterpret_cast<float2*>(q + j * 8 + 2 * t) =
              make_float2((s[j].x + o.x) * 0.125f, (s[j].y + o.y) * 0.125f);
        }
      }
    }
  }
}

}  // namespace
}  // namespace pf
