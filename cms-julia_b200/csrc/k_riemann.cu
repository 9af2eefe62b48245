// Stand-alone Riemann fits (C ABI pxl_riemann_fit): tracks grouped by hit count
// with the same workspace plan as pxl_bl_fit, one kernel per hit count.
#include <algorithm>

#include "../../include/pxl.h"
#include "pxl_internal.cuh"
#include "riemann.cuh"

namespace pxl {

namespace {

struct RmArgs {
  const double* hits;
  const float* ge;
  const int32_t* offs;
  const FitPlan* plan;
  double B;
  float* state;
  float* chi2;
  float* pt;
  int32_t* status;
};

template <int N, class T>
__global__ void __launch_bounds__(128) k_riemann(RmArgs A) {
  const uint32_t cnt = A.plan->count[N];
  const int32_t* list = A.plan->list + A.plan->base_of(N);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const int32_t t = list[i];
    const int32_t first = A.offs[t];
    double h[3][N];
    float ge[6][N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
#pragma unroll
      for (int a = 0; a < 3; ++a) h[a][k] = A.hits[3 * size_t(first + k) + a];
#pragma unroll
      for (int q = 0; q < 6; ++q) ge[q][k] = A.ge[6 * size_t(first + k) + q];
    }
    rm::RiemannOut o;
    const bool ok = rm::riemann_fit<N, T>(h, ge, A.B, o);
#pragma unroll
    for (int k = 0; k < 5; ++k) A.state[5 * size_t(t) + k] = float(o.state[k]);
    A.chi2[2 * size_t(t)] = float(o.chi2_circle);
    A.chi2[2 * size_t(t) + 1] = float(o.chi2_line);
    A.pt[t] = float(o.pt);
    A.status[t] = ok ? 0 : 1;
  }
}

template <class T>
int launch_riemann(const RmArgs& A, cudaStream_t s) {
  const int g = 148 * 4;
  return fan_out(s, 6, [&](int k, cudaStream_t st) {
    switch (k) {
      case 0: k_riemann<3, T><<<g, 128, 0, st>>>(A); break;
      case 1: k_riemann<4, T><<<g, 128, 0, st>>>(A); break;
      case 2: k_riemann<5, T><<<g, 128, 0, st>>>(A); break;
      case 3: k_riemann<6, T><<<g, 128, 0, st>>>(A); break;
      case 4: k_riemann<7, T><<<g, 128, 0, st>>>(A); break;
      default: k_riemann<8, T><<<g, 128, 0, st>>>(A); break;
    }
  });
}

}  // namespace

}  // namespace pxl

extern "C" int32_t pxl_riemann_fit(const double* hits, const float* hits_ge, const int32_t* offs, int32_t n,
                                   double b_field, int32_t precision, float* state, float* chi2, float* pt,
                                   int32_t* status, void* workspace, int64_t workspace_bytes, void* stream) {
  using namespace pxl;
  if (n < 0 || !hits || !hits_ge || !offs || !state || !chi2 || !pt || !status || !workspace) return PXL_ERR_ARG;
  if (precision != 0 && precision != 1) return PXL_ERR_ARG;
  if (workspace_bytes < fit_plan_bytes(n)) return PXL_ERR_CAPACITY;
  if (n == 0) return 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  auto* plan = static_cast<FitPlan*>(workspace);
  int rc = fit_plan_build(offs, n, plan, status, s);
  if (rc) return rc;
  RmArgs A{hits, hits_ge, offs, plan, b_field, state, chi2, pt, status};
  rc = precision == 0 ? launch_riemann<double>(A, s) : launch_riemann<float>(A, s);
  return rc == 0 ? 0 : PXL_ERR_CUDA;
}
