// Broken-line fits of the chain's tuples (launchBrokenLineKernelsOnCPU,
// broken_line_fit_on_gpu.jl:166-203: 3-hit and 4-hit tuples, 5-hit tuples fitted
// with their first 4 hits, at most 24576 per multiplicity) and the stand-alone
// fit entry point pxl_bl_fit (3..8 hits, FP64 or mixed precision).
#include <algorithm>
#include <mutex>

#include "../../include/pxl.h"
#include "bl_fit.cuh"
#include "pxl_internal.cuh"

namespace pxl {

namespace {

// Mixed precision keeps q/pT within 1e-5 of FP64 up to pT of about 100 GeV; the few stiffer
// tuples (about 1 % of a PU50 event's tuples are above 50 GeV) are fitted again in FP64.
constexpr double kRefitPt = 50.0;

// Returns false, writing nothing, for a mixed-precision fit that needs the FP64 refit.
template <int N, class T>
__device__ bool fit_tuple(const Dev& d, uint64_t g, uint32_t hb, const uint32_t* hits_of_tuple, double B) {
  double h[3][N];
  float ge[6][N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const uint32_t hit = hb + hits_of_tuple[i];
    const int det = d.detind[hit];
    const DetParamsD& dp = d.c.det[det];
    float gl[6];
    bl::to_global_cov(dp.R, d.xerr[hit], 0.0f, d.yerr[hit], gl);
#pragma unroll
    for (int k = 0; k < 6; ++k) ge[k][i] = gl[k];
    h[0][i] = d.xg[hit];
    h[1][i] = d.yg[hit];
    h[2][i] = d.zg[hit];
  }
  bl::TrackOut o;
  const bool ok = bl::fit_track<N, T>(h, ge, B, o);
  if (sizeof(T) == 4 && !(o.pt < kRefitPt)) return false;
  float* st = d.t_state + 5 * g;
  float* cv = d.t_cov + 15 * g;
#pragma unroll
  for (int k = 0; k < 5; ++k) st[k] = float(o.state[k]);
#pragma unroll
  for (int k = 0; k < 15; ++k) cv[k] = float(o.cov[k]);
  d.t_pt[g] = float(o.pt);
  d.t_eta[g] = float(o.eta);
  d.t_chi2[g] = float((o.chi2_line + o.chi2_circle) / double(2 * N - 5));
  d.t_fitted[g] = 1;
  (void)ok;
  return true;
}

// Which tuples are fitted, and with how many hits: 3-hit tuples with 3, 4- and
// 5-hit tuples with 4 (fit5as4), none flagged duplicate, at most fits_per_mult
// per multiplicity (the bin is read in decreasing id, so the largest ids win).
// One block per event: the fitted tuples go to the event's region of fit_list
// (3-hit from the front, 4-hit from the back) so that every warp of the fit
// kernel runs one hit count; the others get zero outputs here. The first pass
// sets t_fitted for every tuple (the fit kernel writes it again) and takes list
// slots one atomic per warp; the second zeroes the state and covariance words of
// the tuples left out, walking the packed arrays word by word so that the stores
// coalesce.
__global__ void __launch_bounds__(256) k_fit_list(Dev d) {
  const int e = blockIdx.x;
  EvInfo& E = d.ev[e];
  __shared__ uint32_t s_n3, s_n4;
  if (threadIdx.x == 0) { s_n3 = 0; s_n4 = 0; }
  __syncthreads();
  const uint64_t tb = E.tuple_base;
  const uint32_t nt = E.n_tuples;
  const unsigned lane = threadIdx.x & 31u;
  const uint32_t nt_pad = (nt + 31u) & ~31u;
  for (uint32_t t = threadIdx.x; t < nt_pad; t += blockDim.x) {
    const uint64_t g = tb + t;
    bool fit = false;
    uint32_t n = 0;
    if (t < nt) {
      n = d.tuple_off[g + 1] - d.tuple_off[g];
      fit = n >= 3 && n <= 5 && d.quality[g] != 1;
      if (fit) {
        const uint32_t cnt = E.tm_off[n] - E.tm_off[n - 1];
        if (cnt > d.fits_per_mult) {
          uint32_t larger = 0;
          for (uint32_t u = t + 1; u < nt; ++u) {
            const uint64_t gu = tb + u;
            if (d.tuple_off[gu + 1] - d.tuple_off[gu] == n && d.quality[gu] != 1) ++larger;
          }
          fit = larger < d.fits_per_mult;
        }
      }
    }
    const unsigned m3 = __ballot_sync(0xffffffffu, fit && n == 3);
    const unsigned m4 = __ballot_sync(0xffffffffu, fit && n != 3);
    uint32_t b3 = 0, b4 = 0;
    if (lane == 0) {
      if (m3) b3 = atomicAdd(&s_n3, uint32_t(__popc(m3)));
      if (m4) b4 = atomicAdd(&s_n4, uint32_t(__popc(m4)));
    }
    b3 = __shfl_sync(0xffffffffu, b3, 0);
    b4 = __shfl_sync(0xffffffffu, b4, 0);
    const unsigned below = (1u << lane) - 1u;
    if (t >= nt) continue;
    d.t_fitted[g] = fit ? 1 : 0;
    if (fit) {
      if (n == 3) d.fit_list[tb + b3 + __popc(m3 & below)] = t;
      else d.fit_list[tb + nt - 1 - (b4 + __popc(m4 & below))] = t;
      continue;
    }
    d.t_pt[g] = 0.f; d.t_eta[g] = 0.f; d.t_chi2[g] = 0.f;
  }
  __syncthreads();
  for (uint32_t w = threadIdx.x; w < 5 * nt; w += blockDim.x)
    if (!d.t_fitted[tb + w / 5]) d.t_state[5 * tb + w] = 0.f;
  for (uint32_t w = threadIdx.x; w < 15 * nt; w += blockDim.x)
    if (!d.t_fitted[tb + w / 15]) d.t_cov[15 * tb + w] = 0.f;
  if (threadIdx.x == 0) { E.n_fit3 = s_n3; E.n_fit4 = s_n4; E.n_refit3 = 0; E.n_refit4 = 0; }
}

// one hit count per launch, so that each instantiation keeps only its own registers.
// Capped at 128 registers (four blocks per SM): the 4-hit fit spills a few hundred
// bytes to L1 but runs twice the warps, which hides more of its FP64 latency.
template <int N, class T>
__global__ void __launch_bounds__(128, 4) k_fit_tuples(Dev d) {
  const int e = blockIdx.y;
  const EvInfo& E = d.ev[e];
  const uint64_t tb = E.tuple_base;
  const uint32_t hb = E.hit_base;
  const uint32_t nt = E.n_tuples, nfit = N == 3 ? E.n_fit3 : E.n_fit4;
  // B = Float64(Float32(bf)) as HelixFitOnGPU stores the field (ca_hit_ntuplet_generator.jl:83)
  const double B = double(d.c.b_field);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nfit; i += gridDim.x * blockDim.x) {
    const uint32_t t = d.fit_list[N == 3 ? tb + i : tb + nt - 1 - i];
    const uint64_t g = tb + t;
    if (!fit_tuple<N, T>(d, g, hb, d.tuple_hits + d.tuple_off[g], B)) {
      EvInfo& Ew = d.ev[e];
      const uint32_t k = atomicAdd(N == 3 ? &Ew.n_refit3 : &Ew.n_refit4, 1u);
      d.refit_list[N == 3 ? tb + k : tb + nt - 1 - k] = t;
    }
  }
}

// FP64 refits of the mixed-precision fits that asked for one (same list layout as fit_list)
template <int N>
__global__ void __launch_bounds__(128, 4) k_refit_tuples(Dev d) {
  const int e = blockIdx.y;
  const EvInfo& E = d.ev[e];
  const uint64_t tb = E.tuple_base;
  const uint32_t hb = E.hit_base;
  const uint32_t nt = E.n_tuples, nfit = N == 3 ? E.n_refit3 : E.n_refit4;
  const double B = double(d.c.b_field);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nfit; i += gridDim.x * blockDim.x) {
    const uint64_t g = tb + d.refit_list[N == 3 ? tb + i : tb + nt - 1 - i];
    fit_tuple<N, double>(d, g, hb, d.tuple_hits + d.tuple_off[g], B);
  }
}

template <int N, class T>
__device__ void standalone_fit(const double* hits, const float* hits_ge, int32_t first, double B, float* state,
                               float* cov, float* chi2, float* pt, float* eta, int32_t* status, int32_t t) {
  double h[3][N];
  float ge[6][N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
#pragma unroll
    for (int a = 0; a < 3; ++a) h[a][i] = hits[3 * (first + i) + a];
#pragma unroll
    for (int k = 0; k < 6; ++k) ge[k][i] = hits_ge[6 * (first + i) + k];
  }
  bl::TrackOut o;
  const bool ok = bl::fit_track<N, T>(h, ge, B, o);
#pragma unroll
  for (int k = 0; k < 5; ++k) state[5 * t + k] = float(o.state[k]);
#pragma unroll
  for (int k = 0; k < 15; ++k) cov[15 * t + k] = float(o.cov[k]);
  chi2[t] = float((o.chi2_line + o.chi2_circle) / double(2 * N - 5));
  pt[t] = float(o.pt);
  eta[t] = float(o.eta);
  status[t] = ok ? 0 : 1;
}

}  // namespace

// ------------------------------------------------------------ hit-count buckets
// Stand-alone fits take tracks of 3..8 hits in any order. A count and a scatter
// pass sort the track indices into one list per hit count in the caller's
// workspace, so that each per-N kernel holds only its own registers and every
// warp runs one N. Workspace: FitPlan header, then the lists.
__global__ void k_fit_plan_count(const int32_t* __restrict__ offs, int32_t n, FitPlan* plan, int32_t* status) {
  __shared__ uint32_t s_cnt[kFitMaxN + 1];
  if (threadIdx.x <= kFitMaxN) s_cnt[threadIdx.x] = 0;
  __syncthreads();
  for (int32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int32_t nh = offs[t + 1] - offs[t];
    if (nh >= 3 && nh <= kFitMaxN) atomicAdd(&s_cnt[nh], 1u);
    else if (status) status[t] = -1;
  }
  __syncthreads();
  if (threadIdx.x <= kFitMaxN && s_cnt[threadIdx.x]) atomicAdd(&plan->count[threadIdx.x], s_cnt[threadIdx.x]);
}

__global__ void k_fit_plan_fill(const int32_t* __restrict__ offs, int32_t n, FitPlan* plan) {
  __shared__ uint32_t s_base[kFitMaxN + 1];
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (int k = 0; k <= kFitMaxN; ++k) { s_base[k] = acc; acc += (k >= 3) ? plan->count[k] : 0u; }
  }
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x <= kFitMaxN) plan->base[threadIdx.x] = s_base[threadIdx.x];
  for (int32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const int32_t nh = offs[t + 1] - offs[t];
    if (nh < 3 || nh > kFitMaxN) continue;
    plan->list[s_base[nh] + atomicAdd(&plan->cursor[nh], 1u)] = t;
  }
}

namespace {

template <int N, class T>
__global__ void __launch_bounds__(128, 4) k_fit_bucket(const double* __restrict__ hits, const float* __restrict__ ge,
                                                    const int32_t* __restrict__ offs, const FitPlan* __restrict__ plan,
                                                    double B, float* state, float* cov, float* chi2, float* pt,
                                                    float* eta, int32_t* status) {
  const uint32_t cnt = plan->count[N];
  const int32_t* list = plan->list + plan->base_of(N);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const int32_t t = list[i];
    standalone_fit<N, T>(hits, ge, offs[t], B, state, cov, chi2, pt, eta, status, t);
  }
}

template <class T>
int launch_bucket_fits(const double* hits, const float* ge, const int32_t* offs, const FitPlan* plan, double B,
                       float* state, float* cov, float* chi2, float* pt, float* eta, int32_t* status, cudaStream_t s) {
  const int g = 148 * 4;
  return fan_out(s, 6, [&](int k, cudaStream_t st) {
    switch (k) {
      case 0: k_fit_bucket<3, T><<<g, 128, 0, st>>>(hits, ge, offs, plan, B, state, cov, chi2, pt, eta, status); break;
      case 1: k_fit_bucket<4, T><<<g, 128, 0, st>>>(hits, ge, offs, plan, B, state, cov, chi2, pt, eta, status); break;
      case 2: k_fit_bucket<5, T><<<g, 128, 0, st>>>(hits, ge, offs, plan, B, state, cov, chi2, pt, eta, status); break;
      case 3: k_fit_bucket<6, T><<<g, 128, 0, st>>>(hits, ge, offs, plan, B, state, cov, chi2, pt, eta, status); break;
      case 4: k_fit_bucket<7, T><<<g, 128, 0, st>>>(hits, ge, offs, plan, B, state, cov, chi2, pt, eta, status); break;
      default: k_fit_bucket<8, T><<<g, 128, 0, st>>>(hits, ge, offs, plan, B, state, cov, chi2, pt, eta, status); break;
    }
  });
}

}  // namespace

void launch_fit(const Dev& d, const Launch& L) {
  k_fit_list<<<d.E, 256, 0, L.s>>>(d);
  L.mark("fit_list");
  // about 7000 fits per PU50 event: enough CTAs for every SM with few events
  const int bx = (L.tune && L.tune[kTuneFitTuples] > 0) ? L.tune[kTuneFitTuples]
                                                         : std::max(2, std::min(64, (148 * 16) / std::max(1, int(d.E))));
  // FP64 as the reference fits (broken_line_fit_on_gpu.jl:28-30), or the mixed-precision fit
  if (d.fit_precision == 1) {
    k_fit_tuples<3, float><<<dim3(bx, d.E), 128, 0, L.s>>>(d);
    L.mark("broken_line_fit_3");
    k_fit_tuples<4, float><<<dim3(bx, d.E), 128, 0, L.s>>>(d);
    L.mark("broken_line_fit_4");
    // about 1 % of the fits: one block per event and hit count
    k_refit_tuples<3><<<dim3(1, d.E), 128, 0, L.s>>>(d);
    k_refit_tuples<4><<<dim3(1, d.E), 128, 0, L.s>>>(d);
    L.mark("broken_line_refit_fp64");
  } else {
    k_fit_tuples<3, double><<<dim3(bx, d.E), 128, 0, L.s>>>(d);
    L.mark("broken_line_fit_3");
    k_fit_tuples<4, double><<<dim3(bx, d.E), 128, 0, L.s>>>(d);
    L.mark("broken_line_fit_4");
  }
}

int64_t fit_plan_bytes(int32_t n_tracks) {
  return (int64_t(sizeof(FitPlan)) + 4 * int64_t(n_tracks > 0 ? n_tracks : 0) + 255) / 256 * 256;
}

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_side_mu;
SideStreams g_side[kMaxDevices];
bool g_side_made[kMaxDevices];
}  // namespace

SideStreams* side_streams_lock() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  g_side_mu.lock();
  if (!g_side_made[dev]) {
    SideStreams& ss = g_side[dev];
    bool ok = true;
    for (int j = 0; j < 2; ++j) {
      ok = ok && cudaStreamCreateWithFlags(&ss.st[j], cudaStreamNonBlocking) == cudaSuccess;
      ok = ok && cudaEventCreateWithFlags(&ss.join[j], cudaEventDisableTiming) == cudaSuccess;
    }
    ok = ok && cudaEventCreateWithFlags(&ss.fork, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      g_side_mu.unlock();
      return nullptr;
    }
    g_side_made[dev] = true;
  }
  return &g_side[dev];
}

void side_streams_unlock() { g_side_mu.unlock(); }

int fit_plan_build(const int32_t* offs, int32_t n, FitPlan* plan, int32_t* status, cudaStream_t s) {
  if (cudaMemsetAsync(plan, 0, sizeof(FitPlan) - sizeof(plan->list), s) != cudaSuccess) return PXL_ERR_CUDA;
  const int blocks = std::max(1, std::min(148 * 8, int((n + 255) / 256)));
  k_fit_plan_count<<<blocks, 256, 0, s>>>(offs, n, plan, status);
  k_fit_plan_fill<<<blocks, 256, 0, s>>>(offs, n, plan);
  return cudaGetLastError() == cudaSuccess ? 0 : PXL_ERR_CUDA;
}

}  // namespace pxl

extern "C" int64_t pxl_fit_workspace_bytes(int32_t n_tracks) { return pxl::fit_plan_bytes(n_tracks); }

extern "C" int32_t pxl_bl_fit(const double* hits, const float* hits_ge, const int32_t* offs, int32_t n, double b_field,
                              int32_t precision, float* state, float* cov, float* chi2, float* pt, float* eta,
                              int32_t* status, void* workspace, int64_t workspace_bytes, void* stream) {
  if (n < 0 || !hits || !hits_ge || !offs || !state || !cov || !chi2 || !pt || !eta || !status || !workspace)
    return PXL_ERR_ARG;
  if (precision != 0 && precision != 1) return PXL_ERR_ARG;
  if (workspace_bytes < pxl::fit_plan_bytes(n)) return PXL_ERR_CAPACITY;
  if (n == 0) return 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  auto* plan = static_cast<pxl::FitPlan*>(workspace);
  int rc = pxl::fit_plan_build(offs, n, plan, status, s);
  if (rc) return rc;
  rc = precision == 0
           ? pxl::launch_bucket_fits<double>(hits, hits_ge, offs, plan, b_field, state, cov, chi2, pt, eta, status, s)
           : pxl::launch_bucket_fits<float>(hits, hits_ge, offs, plan, b_field, state, cov, chi2, pt, eta, status, s);
  return rc == 0 ? 0 : PXL_ERR_CUDA;
}
