// CountValidator on the device (plugin-Validation/count_to_validator.jl:18-84): the
// reference's per-event validation rule applied to every event of the last run.
#include <cstdio>
#include <vector>

#include "../../include/pxl.h"
#include "pxl_ctx.h"
#include "pxl_internal.cuh"

namespace pxl {

namespace {

// One block per event: N(track) = the TrackSOA's tuples with hits (the loop over
// stride_track with n_hits_track > 0, :50-55), then the five checks. status bits: 1 modules,
// 2 digis, 4 clusters (exact, :33-46), 8 tracks (relative difference >= 0.012, :56-63, in
// Float64 as the reference divides), 16 vertices (|difference| >= 1, :64-72).
__global__ void __launch_bounds__(256) k_validate_counts(Dev d, const uint32_t* __restrict__ expected,
                                                         uint32_t* __restrict__ status) {
  const int e = blockIdx.x;
  const EvInfo& E = d.ev[e];
  __shared__ uint32_t sh[33];
  const uint64_t tb = E.tuple_base;
  uint32_t cnt = 0;
  for (uint32_t t = threadIdx.x; t < E.n_tuples; t += blockDim.x) cnt += d.tuple_off[tb + t + 1] > d.tuple_off[tb + t];
  uint32_t n_tracks;
  block_excl_scan(cnt, sh, &n_tracks);
  if (threadIdx.x != 0) return;
  const uint32_t* x = expected + 5 * size_t(e);
  uint32_t bad = 0;
  if (E.n_modules != x[0]) bad |= 1u;
  if (E.n_words != x[1]) bad |= 2u;
  if (E.n_clusters != x[2]) bad |= 4u;
  const double rel = fabs((double(n_tracks) - double(x[3])) / double(x[3]));  // 0/0 gives NaN: passes
  if (rel >= double(0.012f)) bad |= 8u;
  const int64_t dv = int64_t(E.n_vtx) - int64_t(x[4]);
  if ((dv < 0 ? -dv : dv) >= 1) bad |= 16u;
  status[e] = bad | (n_tracks << 8);
}

}  // namespace

}  // namespace pxl

extern "C" int32_t pxl_validate_counts(PxlCtx* ctx, const uint32_t* expected, int32_t n_events, uint32_t* status) {
  using namespace pxl;
  if (!ctx || !expected || n_events <= 0) return PXL_ERR_ARG;
  if (n_events != ctx->last_E || !(ctx->done_mask & PXL_STAGE_VERTICES)) return PXL_ERR_STATE;
  if (cudaSetDevice(ctx->p.device) != cudaSuccess) return PXL_ERR_CUDA;
  if (!ctx->val_expected) {
    const size_t E = size_t(ctx->p.max_events);
    if (cudaMalloc(&ctx->val_expected, 5 * E * sizeof(uint32_t)) != cudaSuccess) return PXL_ERR_CUDA;
    ctx->allocs.push_back(ctx->val_expected);
    if (cudaMalloc(&ctx->val_status, E * sizeof(uint32_t)) != cudaSuccess) return PXL_ERR_CUDA;
    ctx->allocs.push_back(ctx->val_status);
  }
  cudaStream_t s = ctx->stream;
  std::vector<uint32_t> st(static_cast<size_t>(n_events));
  if (cudaStreamWaitEvent(s, ctx->last_done, 0) != cudaSuccess ||
      cudaMemcpyAsync(ctx->val_expected, expected, size_t(n_events) * 5 * sizeof(uint32_t), cudaMemcpyHostToDevice,
                      s) != cudaSuccess)
    return PXL_ERR_CUDA;
  Dev d = ctx->d;
  d.E = n_events;
  k_validate_counts<<<n_events, 256, 0, s>>>(d, ctx->val_expected, ctx->val_status);
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(st.data(), ctx->val_status, st.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return PXL_ERR_CUDA;
  int32_t good = 0;
  for (int32_t e = 0; e < n_events; ++e) {
    good += (st[size_t(e)] & 0xFFu) == 0;
    if (status) status[e] = st[size_t(e)];
  }
  return good;
}
