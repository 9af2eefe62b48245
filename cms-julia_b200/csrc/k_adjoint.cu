// Adjoint kernels of the broken-line fit (C ABI pxl_bl_fit_adjoint): per track the
// FP64 chi2 = chi2_line + chi2_circle and its gradient with respect to the hit
// coordinates (bl_adjoint.cuh), optionally with the hits first moved by per-module
// 6-DOF alignment corrections, whose gradients are accumulated per module.
//
// Alignment model (SOAFrame of SOARotation.jl:87-99 with a small correction): a hit
// h on module m with centre c_m moves to h + t_m + w_m x (h - c_m), t = translation,
// w = small rotation (first order). Then d chi2/d t_m = sum of the hits' gradients
// and d chi2/d w_m = sum of (h - c_m) x gradient over the module's hits.
#include <algorithm>

#include "../../include/pxl.h"
#include "bl_adjoint.cuh"
#include "pxl_internal.cuh"

namespace pxl {

namespace {

struct AdjArgs {
  const double* hits;
  const float* ge;
  const int32_t* offs;
  const FitPlan* plan;
  double B;
  const int16_t* hit_module;
  const double* module_pos;
  const float* align;
  int32_t n_modules;
  float* chi2;
  float* grad_hits;
  double* acc;  // [6 * n_modules] FP64 alignment gradient accumulators
};

template <int N>
__global__ void __launch_bounds__(128) k_bl_adjoint(AdjArgs A) {
  const uint32_t cnt = A.plan->count[N];
  const int32_t* list = A.plan->list + A.plan->base_of(N);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    const int32_t t = list[i];
    const int32_t first = A.offs[t];
    double h[3][N];
    float ge[6][N];
    int mod[N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const size_t j = size_t(first) + k;
      double x = A.hits[3 * j], y = A.hits[3 * j + 1], z = A.hits[3 * j + 2];
      mod[k] = A.hit_module ? int(A.hit_module[j]) : -1;
      if (mod[k] >= A.n_modules) mod[k] = -1;
      if (A.align && mod[k] >= 0) {
        const float* al = A.align + 6 * mod[k];
        const double* c = A.module_pos + 3 * mod[k];
        const double rx = x - c[0], ry = y - c[1], rz = z - c[2];
        const double wx = al[3], wy = al[4], wz = al[5];
        x += al[0] + (wy * rz - wz * ry);
        y += al[1] + (wz * rx - wx * rz);
        z += al[2] + (wx * ry - wy * rx);
      }
      h[0][k] = x; h[1][k] = y; h[2][k] = z;
#pragma unroll
      for (int q = 0; q < 6; ++q) ge[q][k] = A.ge[6 * j + q];
    }
    double g[3][N];
    const double c2 = bl::chi2_adjoint<N>(h, ge, A.B, g);
    if (A.chi2) A.chi2[t] = float(c2);
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const size_t j = size_t(first) + k;
      if (A.grad_hits) {
        A.grad_hits[3 * j] = float(g[0][k]);
        A.grad_hits[3 * j + 1] = float(g[1][k]);
        A.grad_hits[3 * j + 2] = float(g[2][k]);
      }
      if (A.acc && mod[k] >= 0) {
        // lever arm of the nominal hit about the module centre
        const double* c = A.module_pos + 3 * mod[k];
        const double rx = A.hits[3 * j] - c[0], ry = A.hits[3 * j + 1] - c[1], rz = A.hits[3 * j + 2] - c[2];
        double* a = A.acc + 6 * mod[k];
        atomicAdd(a + 0, g[0][k]);
        atomicAdd(a + 1, g[1][k]);
        atomicAdd(a + 2, g[2][k]);
        atomicAdd(a + 3, ry * g[2][k] - rz * g[1][k]);
        atomicAdd(a + 4, rz * g[0][k] - rx * g[2][k]);
        atomicAdd(a + 5, rx * g[1][k] - ry * g[0][k]);
      }
    }
  }
}

__global__ void k_align_out(const double* acc, int32_t n, float* out32, double* out64) {
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (out32) out32[i] = float(acc[i]);
    if (out64) out64[i] = acc[i];
  }
}

}  // namespace

}  // namespace pxl

extern "C" int64_t pxl_adjoint_workspace_bytes(int32_t n_tracks, int32_t n_modules) {
  return pxl::fit_plan_bytes(n_tracks) + (int64_t(6) * (n_modules > 0 ? n_modules : 0) * 8 + 255) / 256 * 256;
}

extern "C" int32_t pxl_bl_fit_adjoint(const double* hits, const float* hits_ge, const int32_t* offs, int32_t n,
                                      double b_field, const int16_t* hit_module, const double* module_pos,
                                      const float* align, int32_t n_modules, float* chi2, float* grad_hits,
                                      float* grad_align, double* grad_align64, void* workspace, int64_t ws_bytes,
                                      void* stream) {
  using namespace pxl;
  if (n < 0 || !hits || !hits_ge || !offs || !workspace || n_modules < 0) return PXL_ERR_ARG;
  const bool want_align = grad_align || grad_align64;
  if ((align || want_align) && (!hit_module || !module_pos || n_modules == 0)) return PXL_ERR_ARG;
  if (ws_bytes < pxl_adjoint_workspace_bytes(n, n_modules)) return PXL_ERR_CAPACITY;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  auto* plan = static_cast<FitPlan*>(workspace);
  double* acc = reinterpret_cast<double*>(static_cast<uint8_t*>(workspace) + fit_plan_bytes(n));
  if (want_align && cudaMemsetAsync(acc, 0, size_t(6) * n_modules * sizeof(double), s) != cudaSuccess)
    return PXL_ERR_CUDA;
  if (n > 0) {
    int rc = fit_plan_build(offs, n, plan, nullptr, s);
    if (rc) return rc;
    AdjArgs A{hits, hits_ge, offs, plan, b_field, hit_module, module_pos, align, n_modules, chi2, grad_hits,
              want_align ? acc : nullptr};
    const int g = 148 * 4;
    rc = fan_out(s, 6, [&](int k, cudaStream_t st) {
      switch (k) {
        case 0: k_bl_adjoint<3><<<g, 128, 0, st>>>(A); break;
        case 1: k_bl_adjoint<4><<<g, 128, 0, st>>>(A); break;
        case 2: k_bl_adjoint<5><<<g, 128, 0, st>>>(A); break;
        case 3: k_bl_adjoint<6><<<g, 128, 0, st>>>(A); break;
        case 4: k_bl_adjoint<7><<<g, 128, 0, st>>>(A); break;
        default: k_bl_adjoint<8><<<g, 128, 0, st>>>(A); break;
      }
    });
    if (rc) return PXL_ERR_CUDA;
  }
  if (want_align) k_align_out<<<std::max(1, (6 * n_modules + 255) / 256), 256, 0, s>>>(acc, 6 * n_modules, grad_align, grad_align64);
  return cudaGetLastError() == cudaSuccess ? 0 : PXL_ERR_CUDA;
}
