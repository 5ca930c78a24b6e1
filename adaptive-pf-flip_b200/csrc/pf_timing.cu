// pf_timing.cu -- optional per-stage device timing with CUDA events recorded
// on the context stream (pf_set_timing / pf_get_timing).
#include "pf_ctx.h"

namespace pf {

void stage_begin(pf_ctx* ctx, int stage) {
  if (!ctx->timing_on || ctx->open_ev[stage]) return;
  cudaEvent_t a;
  if (cudaEventCreate(&a) != cudaSuccess) return;
  cudaEventRecord(a, ctx->stream);
  ctx->open_ev[stage] = a;
}

void stage_end(pf_ctx* ctx, int stage) {
  if (!ctx->timing_on || !ctx->open_ev[stage]) return;
  cudaEvent_t b;
  if (cudaEventCreate(&b) != cudaSuccess) return;
  cudaEventRecord(b, ctx->stream);
  ctx->timed.push_back({stage, ctx->open_ev[stage], b});
  ctx->open_ev[stage] = nullptr;
}

int get_timing(pf_ctx* ctx, pf_timing* out, int reset) {
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  for (const TimedStage& t : ctx->timed) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess) {
      ctx->acc_ms[t.stage] += ms;
      ctx->acc_n[t.stage] += 1;
    }
    cudaEventDestroy(t.a);
    cudaEventDestroy(t.b);
  }
  ctx->timed.clear();
  if (out) {
    for (int s = 0; s < PF_NSTAGES; ++s) {
      out->ms[s] = ctx->acc_ms[s];
      out->count[s] = ctx->acc_n[s];
    }
  }
  if (reset) {
    for (int s = 0; s < PF_NSTAGES; ++s) { ctx->acc_ms[s] = 0.0; ctx->acc_n[s] = 0; }
  }
  return PF_OK;
}

}  // namespace pf

extern "C" {

int pf_set_timing(pf_ctx* ctx, int enable) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (!enable) pf::get_timing(ctx, nullptr, 1);
  ctx->timing_on = enable != 0;
  return PF_OK;
}

long long pf_launch_count(const pf_ctx* ctx) { return ctx ? ctx->launches : -1; }

int pf_get_timing(pf_ctx* ctx, pf_timing* out, int reset) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  return pf::get_timing(ctx, out, reset);
}

}  // extern "C"
