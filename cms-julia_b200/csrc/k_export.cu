// Batched, stream-ordered copy-out of the track and vertex collections (pxl_export_async).
//
// The reference hands each event's TrackSOA (CUDADataFormats/PixelTrackHeterogeneous.jl:10-62)
// and ZVertexSoA (z_vertex_soa.jl:4-26) to its consumers. For a batch, copying every event's
// fixed-stride views one by one costs one synchronous copy per product per event. Here the
// tracks of quality loose (the ones the vertex finder and downstream consumers take) and the
// vertices of all events are compacted on the device, event after event in tuple order, into
// one packed array per field, and each array goes to host memory in ONE asynchronous copy on
// a copy stream, with no host synchronisation. Two export buffer sets alternate, so the copy of
// one batch overlaps the chain of the next.
#include <algorithm>
#include <cstdio>

#include "../../include/pxl.h"
#include "pxl_ctx.h"
#include "pxl_internal.cuh"

namespace pxl {

namespace {

constexpr int kExpThreads = 256;

// loose tracks and vertices per event
__global__ void __launch_bounds__(kExpThreads) k_export_count(Dev d, ExportSet x) {
  const int e = blockIdx.x;
  const EvInfo& E = d.ev[e];
  __shared__ uint32_t sh[33];
  uint32_t cnt = 0;
  for (uint32_t t = threadIdx.x; t < E.n_tuples; t += blockDim.x) cnt += d.quality[uint64_t(E.tuple_base) + t] == 2;
  uint32_t tot;
  block_excl_scan(cnt, sh, &tot);
  if (threadIdx.x == 0) {
    x.index[4 * e + 1] = tot;
    x.index[4 * e + 3] = E.n_vtx;
  }
}

// first track and first vertex of each event (one block); row E holds the totals
__global__ void __launch_bounds__(1024) k_export_scan(Dev d, ExportSet x) {
  __shared__ uint32_t sh[33];
  uint32_t ct = 0, cv = 0;
  for (int b = 0; b < d.E; b += blockDim.x) {
    const int e = b + threadIdx.x;
    const uint32_t nt = e < d.E ? x.index[4 * e + 1] : 0u, nv = e < d.E ? x.index[4 * e + 3] : 0u;
    uint32_t tt, tv;
    const uint32_t et = block_excl_scan(nt, sh, &tt);
    const uint32_t ev = block_excl_scan(nv, sh, &tv);
    if (e < d.E) { x.index[4 * e] = ct + et; x.index[4 * e + 2] = cv + ev; }
    ct += tt;
    cv += tv;
  }
  if (threadIdx.x == 0) {
    x.index[4 * d.E] = ct; x.index[4 * d.E + 1] = ct; x.index[4 * d.E + 2] = cv; x.index[4 * d.E + 3] = cv;
  }
}

// the event's loose tracks in tuple order, and its vertices
__global__ void __launch_bounds__(kExpThreads) k_export_fill(Dev d, ExportSet x) {
  const int e = blockIdx.x;
  const EvInfo& E = d.ev[e];
  __shared__ uint32_t sh[33];
  const uint64_t tb = E.tuple_base;
  uint32_t base = x.index[4 * e];
  for (uint32_t b = 0; b < E.n_tuples; b += blockDim.x) {
    const uint32_t t = b + threadIdx.x;
    const bool loose = t < E.n_tuples && d.quality[tb + t] == 2;
    uint32_t tot;
    const uint32_t r = base + block_excl_scan(loose ? 1u : 0u, sh, &tot);
    if (loose && r < x.cap_tracks) {
      const uint64_t g = tb + t;
#pragma unroll
      for (int k = 0; k < 5; ++k) x.state[5 * size_t(r) + k] = d.t_state[5 * g + k];
#pragma unroll
      for (int k = 0; k < 15; ++k) x.cov[15 * size_t(r) + k] = d.t_cov[15 * g + k];
      x.pt[r] = d.t_pt[g];
      x.eta[r] = d.t_eta[g];
      x.chi2[r] = d.t_chi2[g];
      x.n_hits[r] = uint8_t(d.tuple_off[g + 1] - d.tuple_off[g]);
      x.vertex[r] = d.idv[g];
      x.tuple[r] = t + 1;
    }
    base += tot;
  }
  const uint32_t v0 = x.index[4 * e + 2], nv = E.n_vtx;
  const int32_t* nn = d.ndof + tb + size_t(e) * 1024;
  for (uint32_t v = threadIdx.x; v < nv; v += blockDim.x) {
    const uint32_t o = v0 + v;
    if (o >= x.cap_vertices) break;
    x.zv[o] = d.zv[size_t(e) * 1024 + v];
    x.wv[o] = d.wv[size_t(e) * 1024 + v];
    x.vchi2[o] = d.vchi2[size_t(e) * 1024 + v];
    x.ptv2[o] = d.ptv2[size_t(e) * 1024 + v];
    x.ndof[o] = nn[v];
  }
}

template <class T>
cudaError_t alloc_n(T** p, size_t n) {
  return cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T));
}

}  // namespace

int export_alloc(PxlCtx* ctx) {
  const Dev& d = ctx->d;
  const size_t nt = size_t(d.cap_tuples), nv = size_t(ctx->p.max_events) * 1024, ne = size_t(ctx->p.max_events) + 1;
  for (ExportSet& x : ctx->exp) {
    x.cap_tracks = uint32_t(nt);
    x.cap_vertices = uint32_t(nv);
    if (alloc_n(&x.index, 4 * ne) || alloc_n(&x.state, 5 * nt) || alloc_n(&x.cov, 15 * nt) || alloc_n(&x.pt, nt) ||
        alloc_n(&x.eta, nt) || alloc_n(&x.chi2, nt) || alloc_n(&x.n_hits, nt) || alloc_n(&x.vertex, nt) ||
        alloc_n(&x.tuple, nt) || alloc_n(&x.zv, nv) || alloc_n(&x.wv, nv) || alloc_n(&x.vchi2, nv) ||
        alloc_n(&x.ptv2, nv) || alloc_n(&x.ndof, nv))
      return PXL_ERR_CUDA;
    for (void* q : {(void*)x.index, (void*)x.state, (void*)x.cov, (void*)x.pt, (void*)x.eta, (void*)x.chi2,
                    (void*)x.n_hits, (void*)x.vertex, (void*)x.tuple, (void*)x.zv, (void*)x.wv, (void*)x.vchi2,
                    (void*)x.ptv2, (void*)x.ndof})
      ctx->allocs.push_back(q);
    if (cudaEventCreateWithFlags(&x.ready, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&x.copied, cudaEventDisableTiming) != cudaSuccess)
      return PXL_ERR_CUDA;
  }
  return 0;
}

int export_run(PxlCtx* ctx, const PxlExport* out, cudaStream_t s, cudaStream_t cs) {
  const Dev& d = ctx->d;
  if (!ctx->exp[0].index) {
    const int rc = export_alloc(ctx);
    if (rc) return rc;
  }
  ExportSet& x = ctx->exp[ctx->exp_next];
  ctx->exp_next ^= 1;
  const int E = ctx->last_E;
  // the set's previous copies must have left before its arrays are written again
  if (cudaStreamWaitEvent(s, ctx->last_done, 0) != cudaSuccess || cudaStreamWaitEvent(s, x.copied, 0) != cudaSuccess)
    return PXL_ERR_CUDA;
  Dev dd = d;
  dd.E = E;
  k_export_count<<<E, kExpThreads, 0, s>>>(dd, x);
  k_export_scan<<<1, 1024, 0, s>>>(dd, x);
  k_export_fill<<<E, kExpThreads, 0, s>>>(dd, x);
  if (cudaGetLastError() != cudaSuccess || cudaEventRecord(x.ready, s) != cudaSuccess ||
      cudaStreamWaitEvent(cs, x.ready, 0) != cudaSuccess)
    return PXL_ERR_CUDA;
  const size_t mt = size_t(std::min<int64_t>(out->max_tracks, x.cap_tracks));
  const size_t mv = size_t(std::min<int64_t>(out->max_vertices, x.cap_vertices));
  auto cp = [&](void* dst, const void* src, size_t bytes) {
    return !dst || bytes == 0 || cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, cs) == cudaSuccess;
  };
  const bool ok = cp(out->index, x.index, size_t(E + 1) * 16) && cp(out->state, x.state, mt * 20) &&
                  cp(out->cov, x.cov, mt * 60) && cp(out->pt, x.pt, mt * 4) && cp(out->eta, x.eta, mt * 4) &&
                  cp(out->chi2, x.chi2, mt * 4) && cp(out->n_hits, x.n_hits, mt) && cp(out->vertex, x.vertex, mt * 2) &&
                  cp(out->tuple, x.tuple, mt * 4) && cp(out->zv, x.zv, mv * 4) && cp(out->wv, x.wv, mv * 4) &&
                  cp(out->vchi2, x.vchi2, mv * 4) && cp(out->ptv2, x.ptv2, mv * 4) && cp(out->ndof, x.ndof, mv * 4);
  if (!ok || cudaEventRecord(x.copied, cs) != cudaSuccess) return PXL_ERR_CUDA;
  return 0;
}

int64_t export_bytes(const PxlExport* out, int32_t n_events) {
  const int64_t mt = out->max_tracks, mv = out->max_vertices;
  int64_t b = out->index ? int64_t(n_events + 1) * 16 : 0;
  b += (out->state ? 20 : 0) * mt + (out->cov ? 60 : 0) * mt + (out->pt ? 4 : 0) * mt + (out->eta ? 4 : 0) * mt +
       (out->chi2 ? 4 : 0) * mt + (out->n_hits ? 1 : 0) * mt + (out->vertex ? 2 : 0) * mt + (out->tuple ? 4 : 0) * mt;
  b += ((out->zv ? 4 : 0) + (out->wv ? 4 : 0) + (out->vchi2 ? 4 : 0) + (out->ptv2 ? 4 : 0) + (out->ndof ? 4 : 0)) * mv;
  return b;
}

}  // namespace pxl

extern "C" int32_t pxl_export_async(PxlCtx* ctx, const PxlExport* out, void* stream, void* copy_stream) {
  if (!ctx || !out || out->max_tracks < 0 || out->max_vertices < 0) return PXL_ERR_ARG;
  if (ctx->last_E <= 0 || (ctx->done_mask & PXL_STAGE_VERTICES) == 0) return PXL_ERR_STATE;
  if (cudaSetDevice(ctx->p.device) != cudaSuccess) return PXL_ERR_CUDA;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  cudaStream_t cs = copy_stream ? static_cast<cudaStream_t>(copy_stream) : s;
  const int rc = pxl::export_run(ctx, out, s, cs);
  return rc ? rc : 0;
}

extern "C" int64_t pxl_export_bytes(const PxlExport* out, int32_t n_events) {
  if (!out || n_events < 0) return PXL_ERR_ARG;
  return pxl::export_bytes(out, n_events);
}
