// Broken-line helix fit, one thread per track with every matrix in registers.
// Restates plugin-PixelTriplets/broken_line.jl:46-528 (BL_Fast_fit,
// prepare_broken_line_data, mult_scatt, matrixc_u, BL_Line_fit, BL_Circle_fit,
// translate_karimaki) and cholesky_inversion.jl (symmetric inverse).
//
// Scalar policy: T is the working type of the bulk arithmetic. The symmetric
// band-system inverse, the solve u = C^-1 r and every covariance propagation
// are always FP64. T = double gives the reference's all-FP64 fit; T = float
// gives the mixed-precision fit (FP32 arithmetic, FP64 Cholesky and covariance).
#pragma once
#include <cstdint>

namespace pxl {
namespace bl {

template <class T> __device__ __forceinline__ T s_sqrt(T x);
template <> __device__ __forceinline__ double s_sqrt<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float s_sqrt<float>(float x) { return sqrtf(x); }
template <class T> __device__ __forceinline__ T s_atan(T x);
template <> __device__ __forceinline__ double s_atan<double>(double x) { return atan(x); }
template <> __device__ __forceinline__ float s_atan<float>(float x) { return atanf(x); }
template <class T> __device__ __forceinline__ T s_log(T x);
template <> __device__ __forceinline__ double s_log<double>(double x) { return log(x); }
template <> __device__ __forceinline__ float s_log<float>(float x) { return logf(x); }
template <class T> __device__ __forceinline__ T s_sin(T x);
template <> __device__ __forceinline__ double s_sin<double>(double x) { return sin(x); }
template <> __device__ __forceinline__ float s_sin<float>(float x) { return sinf(x); }
template <class T> __device__ __forceinline__ T s_cos(T x);
template <> __device__ __forceinline__ double s_cos<double>(double x) { return cos(x); }
template <> __device__ __forceinline__ float s_cos<float>(float x) { return cosf(x); }
template <class T> __device__ __forceinline__ T s_abs(T x) { return x < T(0) ? -x : x; }

constexpr double kPi = 3.141592653589793;

// custom atan2 of broken_line.jl:256-268: range (-pi/2, 3pi/2)
template <class T>
__device__ __forceinline__ T bl_atan2(T y, T x) {
  if (x > T(0)) return s_atan<T>(y / x);
  if (x < T(0)) return s_atan<T>(y / x) + T(kPi);
  if (y > T(0) && x == T(0)) return T(kPi / 2);
  if (y < T(0) && x == T(0)) return T(-kPi / 2);
  return T(__longlong_as_double(0x7ff8000000000000ll));
}

template <class T>
__device__ __forceinline__ T mult_scatt(T length, T B, T R, T slope) {
  T pt2 = B * R;
  pt2 = pt2 < T(20.0) ? pt2 : T(20.0);
  pt2 = pt2 * pt2;
  const T XXI_0 = T(0.06 / 16.0);
  const T fact = T(0.7 * ((13.6 / 1000) * (13.6 / 1000)));
  const T slope_term = T(1) + slope * slope;
  const T abs_len = s_abs(length) * XXI_0;
  const T lt = s_log<T>(abs_len);
  const T sq = (T(1) + T(0.038) * lt) * (T(1) + T(0.038) * lt);
  return fact / (pt2 * slope_term) * abs_len * sq;
}

template <class T>
__device__ __forceinline__ void rotation_matrix(T slope, T R[2][2]) {
  const T a = T(1) / s_sqrt<T>(T(1) + slope * slope);
  const T b = slope * a;
  R[0][0] = a; R[0][1] = b; R[1][0] = -b; R[1][1] = a;
}

// symmetric positive-definite inverse by LDL^T, FP64, reading the lower triangle
template <int M>
__device__ __forceinline__ void invert_sym(const double A[M][M], double Inv[M][M]) {
  double L[M][M], D[M], Li[M][M];
#pragma unroll
  for (int j = 0; j < M; ++j) {
    double dd = A[j][j];
#pragma unroll
    for (int k = 0; k < j; ++k) dd -= L[j][k] * L[j][k] * D[k];
    D[j] = dd;
    L[j][j] = 1.0;
#pragma unroll
    for (int i = j + 1; i < M; ++i) {
      double v = A[i][j];
#pragma unroll
      for (int k = 0; k < j; ++k) v -= L[i][k] * L[j][k] * D[k];
      L[i][j] = v / dd;
    }
  }
#pragma unroll
  for (int i = 0; i < M; ++i) {
    Li[i][i] = 1.0;
#pragma unroll
    for (int j = 0; j < i; ++j) {
      double v = 0;
#pragma unroll
      for (int k = j; k < i; ++k) v -= L[i][k] * Li[k][j];
      Li[i][j] = v;
    }
  }
#pragma unroll
  for (int i = 0; i < M; ++i)
#pragma unroll
    for (int j = 0; j <= i; ++j) {
      double v = 0;
#pragma unroll
      for (int k = i; k < M; ++k) v += Li[k][i] * Li[k][j] / D[k];
      Inv[i][j] = v;
      Inv[j][i] = v;
    }
}

template <int N, class T>
struct Prepared {
  int q;
  T radii[2][N];
  T s[N], S[N], Z[N], VarBeta[N];
};

// BL_Fast_fit; h[3][N] hit coordinates (columns are hits)
template <int N, class T>
__device__ __forceinline__ void fast_fit(const T h[3][N], T r[4]) {
  constexpr int mid = N >> 1;
  const T h11 = h[0][0], h21 = h[1][0], h1m = h[0][mid], h2m = h[1][mid], h1n = h[0][N - 1], h2n = h[1][N - 1];
  const T a1 = h1m - h11, a2 = h2m - h21, b1 = h1n - h1m, b2 = h2n - h2m, c1 = h11 - h1n, c2 = h21 - h2n;
  const T ca = c1 * a2 - c2 * a1, ba = b1 * a2 - b2 * a1;
  const T nc = c1 * c1 + c2 * c2, na = a1 * a1 + a2 * a2, nb = b1 * b1 + b2 * b2;
  const T tmp = T(0.5) / ca;
  r[0] = h11 - (a2 * nc + c2 * na) * tmp;
  r[1] = h21 + (a1 * nc + c1 * na) * tmp;
  r[2] = s_sqrt<T>(na * nb * nc) / (T(2.0) * s_abs(ba));
  const T cx = r[0], cy = r[1];
  const T d1 = h11 - cx, d2 = h21 - cy, e1 = h1n - cx, e2 = h2n - cy;
  const T de = d1 * e2 - d2 * e1, dotde = d1 * e1 + d2 * e2;
  const T dz = h[2][N - 1] - h[2][0];
  r[3] = r[2] * bl_atan2<T>(de, dotde) / dz;
}

template <int N, class T>
__device__ __forceinline__ void prepare(const T h[3][N], const T f[4], T B, Prepared<N, T>& d) {
  const T x1 = h[0][1] - h[0][0], y1 = h[1][1] - h[1][0];
  const T xn = h[0][N - 1] - h[0][N - 2], yn = h[1][N - 1] - h[1][N - 2];
  d.q = (x1 * yn - y1 * xn) > T(0) ? -1 : 1;
  const T slope = -T(d.q) / f[3];
  T R[2][2];
  rotation_matrix<T>(slope, R);
#pragma unroll
  for (int j = 0; j < N; ++j) { d.radii[0][j] = h[0][j] - f[0]; d.radii[1][j] = h[1][j] - f[1]; }
  const T rr = s_sqrt<T>(f[0] * f[0] + f[1] * f[1]);
  const T sc = -f[2] / rr;
  const T e1 = sc * f[0], e2 = sc * f[1];
  const T fac = T(d.q) * f[2];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const T xi = d.radii[0][i], yi = d.radii[1][i];
    d.s[i] = fac * bl_atan2<T>(xi * e2 - yi * e1, xi * e1 + yi * e2);
  }
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const T xi = d.s[i], yi = h[2][i];
    d.S[i] = R[0][0] * xi + R[0][1] * yi;
    d.Z[i] = R[1][0] * xi + R[1][1] * yi;
  }
  d.VarBeta[0] = 0;
  d.VarBeta[N - 1] = 0;
#pragma unroll
  for (int i = 1; i < N - 1; ++i)
    d.VarBeta[i] = mult_scatt<T>(d.S[i + 1] - d.S[i], B, f[2], slope) + mult_scatt<T>(d.S[i] - d.S[i - 1], B, f[2], slope);
}

// matrixc_u (broken_line.jl:217-250) into the top-left N x N block of C (M >= N)
template <int N, int M, class T>
__device__ __forceinline__ void matrixc_u(const T w[N], const T S[N], const T VB[N], double C[M][M]) {
  T Tm[N][N + 2];
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N + 2; ++j) Tm[i][j] = T(0);
#pragma unroll
  for (int i = 0; i < N; ++i) {
    Tm[i][i] = w[i];
    if (i > 1) Tm[i][i] += T(1) / (VB[i - 1] * ((S[i] - S[i - 1]) * (S[i] - S[i - 1])));
    if (i > 0 && i < N - 1) {
      const T q = (S[i + 1] - S[i - 1]) / ((S[i + 1] - S[i]) * (S[i] - S[i - 1]));
      Tm[i][i] += (T(1) / VB[i]) * (q * q);
    }
    if (i < N - 2) Tm[i][i] += T(1) / (VB[i + 1] * ((S[i + 1] - S[i]) * (S[i + 1] - S[i])));
    if (i > 0 && i < N - 1)
      Tm[i][i + 1] = T(1) / (VB[i] * (S[i + 1] - S[i])) * (-(S[i + 1] - S[i - 1]) / ((S[i + 1] - S[i]) * (S[i] - S[i - 1])));
    if (i < N - 2)
      Tm[i][i + 1] += T(1) / (VB[i + 1] * (S[i + 1] - S[i])) * (-(S[i + 2] - S[i]) / ((S[i + 2] - S[i + 1]) * (S[i + 1] - S[i])));
    if (i < N - 2) Tm[i][i + 2] = T(1) / (VB[i + 1] * (S[i + 2] - S[i + 1]) * (S[i + 1] - S[i]));
    Tm[i][i] *= T(0.5);
  }
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) C[i][j] = double(Tm[i][j] + Tm[j][i]);
}

__device__ __forceinline__ void sandwich2(const double J[2][2], double C[2][2]) {
  double Tm[2][2], O[2][2];
  for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) Tm[a][b] = J[a][0] * C[0][b] + J[a][1] * C[1][b];
  for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) O[a][b] = Tm[a][0] * J[b][0] + Tm[a][1] * J[b][1];
  for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) C[a][b] = O[a][b];
}

__device__ __forceinline__ void sandwich3(const double J[3][3], double C[3][3]) {
  double Tm[3][3], O[3][3];
  for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) Tm[a][b] = J[a][0] * C[0][b] + J[a][1] * C[1][b] + J[a][2] * C[2][b];
  for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) O[a][b] = Tm[a][0] * J[b][0] + Tm[a][1] * J[b][1] + Tm[a][2] * J[b][2];
  for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) C[a][b] = O[a][b];
}

struct LineOut { double par[2]; double cov[2][2]; double chi2; };
struct CircleOut { double par[3]; double cov[3][3]; int q; double chi2; };

// BL_Line_fit, broken_line.jl:546-696; ge[6][N] as Float32
template <int N, class T>
__device__ __forceinline__ void line_fit(const float ge[6][N], const T f[4], T B, const Prepared<N, T>& d, LineOut& L) {
  const T slope = -T(d.q) / f[3];
  T R[2][2];
  rotation_matrix<T>(slope, R);
  const double tol = 1e-12;
  T w[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    auto z = [&](float v) { return fabs(double(v)) < tol ? T(0) : T(v); };
    const T V[3][3] = {{T(ge[0][i]), z(ge[1][i]), z(ge[3][i])}, {z(ge[1][i]), T(ge[2][i]), z(ge[4][i])},
                       {z(ge[3][i]), z(ge[4][i]), T(ge[5][i])}};
    const T tmp = T(1) / s_sqrt<T>(d.radii[0][i] * d.radii[0][i] + d.radii[1][i] * d.radii[1][i]);
    const T J[2][3] = {{d.radii[1][i] * tmp, -d.radii[0][i] * tmp, T(0)}, {T(0), T(0), T(1)}};
    T M1[2][3], M2[2][3], M3[2][2];
    for (int a = 0; a < 2; ++a) for (int b = 0; b < 3; ++b) M1[a][b] = R[a][0] * J[0][b] + R[a][1] * J[1][b];
    for (int a = 0; a < 2; ++a) for (int b = 0; b < 3; ++b) M2[a][b] = M1[a][0] * V[0][b] + M1[a][1] * V[1][b] + M1[a][2] * V[2][b];
    for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) M3[a][b] = M2[a][0] * J[b][0] + M2[a][1] * J[b][1] + M2[a][2] * J[b][2];
    const T m22 = M3[1][0] * R[1][0] + M3[1][1] * R[1][1];
    w[i] = T(1) / m22;
  }
  double C[N][N], I[N][N];
  matrixc_u<N, N, T>(w, d.S, d.VarBeta, C);
  invert_sym<N>(C, I);
  double u[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    double v = 0;
#pragma unroll
    for (int k = 0; k < N; ++k) v += I[i][k] * double(w[k] * d.Z[k]);
    u[i] = v;
  }
  T par0 = (T(u[1]) - T(u[0])) / (d.S[1] - d.S[0]);
  T par1 = T(u[0]);
  const double idiff = 1.0 / double(d.S[1] - d.S[0]);
  double cov[2][2] = {{(I[0][0] - 2 * I[0][1] + I[1][1]) * (idiff * idiff) + double(mult_scatt<T>(d.S[1] - d.S[0], B, f[2], slope)),
                       (I[0][1] - I[0][0]) * idiff},
                      {(I[0][1] - I[0][0]) * idiff, I[0][0]}};
  double jac[2][2] = {{1, 0}, {-double(d.S[0]), 1}};
  par1 = par1 - par0 * d.S[0];
  sandwich2(jac, cov);
  const T tmp = R[0][0] - par0 * R[0][1];
  const T j22 = T(1) / tmp;
  jac[1][1] = double(j22);
  jac[0][0] = double(j22 * j22);
  jac[0][1] = 0;
  jac[1][0] = double(par1 * R[0][1] * (j22 * j22));
  par1 = par1 * j22;
  par0 = (R[0][1] + par0 * R[0][0]) * j22;
  sandwich2(jac, cov);
  L.par[0] = double(par0);
  L.par[1] = double(par1);
  for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) L.cov[a][b] = cov[a][b];
  T chi2 = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const T diff = d.Z[i] - T(u[i]);
    chi2 += w[i] * (diff * diff);
    if (i > 0 && i < N - 1) {
      const T den1 = d.S[i] - d.S[i - 1], den2 = d.S[i + 1] - d.S[i], den3 = d.S[i] - d.S[i - 1], den4 = d.S[i + 1] - d.S[i - 1];
      const T t = (T(u[i - 1]) / den1) - (T(u[i]) * (den4 / (den2 * den3))) + (T(u[i + 1]) / (d.S[i + 1] - d.S[i]));
      chi2 += (t * t) / d.VarBeta[i];
    }
  }
  L.chi2 = double(chi2);
}

template <class T>
__device__ __forceinline__ void translate_karimaki(CircleOut& c, T x0, T y0) {
  const T p1 = T(c.par[0]), p2 = T(c.par[1]), p3 = T(c.par[2]);
  const T cs = s_cos<T>(p1), sn = s_sin<T>(p1);
  const T DP = x0 * cs + y0 * sn;
  const T DO = x0 * sn - y0 * cs + p2;
  const T uu = T(1) + p3 * p2;
  const T C = -p3 * y0 + uu * cs;
  const T BB = p3 * x0 + uu * sn;
  const T A = T(2.0) * DO + p3 * (DO * DO + DP * DP);
  const T U = s_sqrt<T>(T(1.0) + p3 * A);
  const T xi = T(1.0) / (BB * BB + C * C);
  const T v = T(1.0) + p3 * DO;
  const T lambda = (T(0.5) * A) / (U * ((T(1.0) + U) * (T(1.0) + U)));
  const T mu = T(1.0) / (U * (T(1.0) + U)) + p3 * lambda;
  const T zeta = DO * DO + DP * DP;
  const double J[3][3] = {{double(xi * uu * v), double(-xi * (p3 * p3) * DP), double(xi * DP)},
                          {double(T(2.0) * mu * uu * DP), double(T(2.0) * mu * v), double(mu * zeta - lambda * A)},
                          {0.0, 0.0, 1.0}};
  c.par[0] = double(bl_atan2<T>(BB, C));
  c.par[1] = double(A / (T(1.0) + U));
  sandwich3(J, c.cov);
}

// BL_Circle_fit, broken_line.jl:330-528; returns false where the reference raises
template <int N, class T>
__device__ __forceinline__ bool circle_fit(const T h[3][N], const float ge[6][N], const T f[4], T B, Prepared<N, T>& d,
                                           CircleOut& c) {
  bool ok = true;
  c.q = d.q;
  const T slope = -T(c.q) / f[3];
  T VB[N];
#pragma unroll
  for (int i = 0; i < N; ++i) VB[i] = d.VarBeta[i] * (T(1.0) + slope * slope);
#pragma unroll
  for (int i = 0; i < N; ++i) d.Z[i] = s_sqrt<T>(d.radii[0][i] * d.radii[0][i] + d.radii[1][i] * d.radii[1][i]) - f[2];
  const double tol = 1e-12;
  T w[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    auto z = [&](float v) { return fabs(double(v)) < tol ? T(0) : T(v); };
    const T V[2][2] = {{z(ge[0][i]), z(ge[1][i])}, {z(ge[1][i]), z(ge[2][i])}};
    T RR[2][2];
    rotation_matrix<T>(-d.radii[0][i] / d.radii[1][i], RR);
    const T t0 = RR[1][0] * V[0][0] + RR[1][1] * V[1][0];
    const T t1 = RR[1][0] * V[0][1] + RR[1][1] * V[1][1];
    w[i] = T(1.0) / (t0 * RR[1][0] + t1 * RR[1][1]);
  }
  constexpr int M = N + 1;
  double C[M][M];
#pragma unroll
  for (int i = 0; i < M; ++i)
#pragma unroll
    for (int j = 0; j < M; ++j) C[i][j] = 0.0;
  matrixc_u<N, M, T>(w, d.s, VB, C);
  const T* s = d.s;
  T cnn = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    T v = 0;
    if (i > 0 && i < N - 1) v += -(s[i + 1] - s[i - 1]) * (s[i + 1] - s[i - 1]) / (T(2.0) * VB[i] * (s[i + 1] - s[i]) * (s[i] - s[i - 1]));
    if (i > 1) v += (s[i] - s[i - 2]) / (T(2.0) * VB[i - 1] * (s[i] - s[i - 1]));
    if (i < N - 2) v += (s[i + 2] - s[i]) / (T(2.0) * VB[i + 1] * (s[i + 1] - s[i]));
    C[i][N] = double(v);
    C[N][i] = double(v);
    if (i > 0 && i < N - 1) cnn += ((s[i + 1] - s[i - 1]) * (s[i + 1] - s[i - 1])) / (T(4.0) * VB[i]);
  }
  C[N][N] = double(cnn);
  double I[M][M];
  invert_sym<M>(C, I);
  double u[M];
#pragma unroll
  for (int i = 0; i < M; ++i) {
    double v = 0;
#pragma unroll
    for (int k = 0; k < N; ++k) v += I[i][k] * double(w[k] * d.Z[k]);
    u[i] = v;
  }
#pragma unroll
  for (int col = 0; col < 2; ++col) {
    const T t = s_sqrt<T>(d.radii[0][col] * d.radii[0][col] + d.radii[1][col] * d.radii[1][col]);
    d.radii[0][col] /= t;
    d.radii[1][col] /= t;
  }
  const T tmp1 = -d.Z[0] + T(u[0]);
  const T dv0 = h[0][0] + tmp1 * d.radii[0][0], dv1 = h[1][0] + tmp1 * d.radii[1][0];
  const T tmp2 = -d.Z[1] + T(u[1]);
  const T ev0 = h[0][1] + tmp2 * d.radii[0][1], ev1 = h[1][1] + tmp2 * d.radii[1][1];
  const T emd0 = ev0 - dv0, emd1 = ev1 - dv1;
  const T nrm = s_sqrt<T>(emd0 * emd0 + emd1 * emd1);
  c.par[0] = double(bl_atan2<T>(emd1, emd0));
  const T inner = f[2] * f[2] - T(0.25) * (nrm * nrm);
  if (inner < T(0)) ok = false;
  c.par[1] = double(-T(c.q) * (f[2] - s_sqrt<T>(inner)));
  c.par[2] = double(T(c.q) * (T(1.0) / f[2] + T(u[N])));
  if (!(double(c.q) * c.par[1] <= 0)) ok = false;
  const T t1 = nrm * nrm;
  const T fl = T(floor(double(c.q) / 2));
  const T den = s_sqrt<T>((T(2) * f[2]) * (T(2) * f[2]) - t1);
  const double J[3][3] = {
      {double((d.radii[1][0] * emd0 - emd1 * d.radii[0][0]) / t1), double((d.radii[1][1] * emd0 - emd1 * d.radii[0][1]) / t1), 0},
      {double(fl * (emd0 * d.radii[0][0] + emd1 * d.radii[1][0]) / den), double(fl * (emd0 * d.radii[0][1] + emd1 * d.radii[1][1]) / den), 0},
      {0, 0, double(c.q)}};
  c.cov[0][0] = I[0][0]; c.cov[0][1] = I[0][1]; c.cov[0][2] = I[0][N];
  c.cov[1][0] = I[1][0]; c.cov[1][1] = I[1][1]; c.cov[1][2] = I[1][N];
  c.cov[2][0] = I[N][0]; c.cov[2][1] = I[N][1]; c.cov[2][2] = I[N][N];
  sandwich3(J, c.cov);
  translate_karimaki<T>(c, T(0.5) * emd0, T(0.5) * emd1);
  c.cov[0][0] += double((T(1) + slope * slope) * mult_scatt<T>(d.S[1] - d.S[0], B, f[2], slope));
  translate_karimaki<T>(c, dv0, dv1);
  T chi2 = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const T diff = d.Z[i] - T(u[i]);
    chi2 += w[i] * (diff * diff);
    if (i > 0 && i < N - 1) {
      const T d1 = s[i] - s[i - 1], d2 = s[i + 1] - s[i], d3 = s[i + 1] - s[i - 1];
      const T t = T(u[i - 1]) / d1 - (T(u[i]) * d3) / (d1 * d2) + T(u[i + 1]) / d2 + (d3 * T(u[N])) / T(2.0);
      chi2 += (t * t) / VB[i];
    }
  }
  c.chi2 = double(chi2);
  return ok;
}

struct TrackOut {
  double state[5];
  double cov[15];
  double chi2_line, chi2_circle, pt, eta;
};

// full fit of one track of N hits: hits[3][N] (FP64 inputs), ge[6][N] (Float32)
template <int N, class T>
__device__ __forceinline__ bool fit_track(const double hits[3][N], const float ge[6][N], double Bd, TrackOut& o) {
  T h[3][N];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int i = 0; i < N; ++i) h[a][i] = T(hits[a][i]);
  const T B = T(Bd);
  T f[4];
  fast_fit<N, T>(h, f);
  Prepared<N, T> d;
  prepare<N, T>(h, f, B, d);
  LineOut L;
  line_fit<N, T>(ge, f, B, d, L);
  CircleOut C;
  const bool ok = circle_fit<N, T>(h, ge, f, B, d, C);
  const double b = 1.0 / Bd;
  o.state[0] = C.par[0]; o.state[1] = C.par[1]; o.state[2] = C.par[2] * b; o.state[3] = L.par[0]; o.state[4] = L.par[1];
  const double cv[15] = {C.cov[0][0], C.cov[0][1], b * C.cov[0][2], 0.0, 0.0, C.cov[1][1], b * C.cov[1][2], 0.0, 0.0,
                         (b * b) * C.cov[2][2], 0.0, 0.0, L.cov[0][0], L.cov[0][1], L.cov[1][1]};
#pragma unroll
  for (int k = 0; k < 15; ++k) o.cov[k] = cv[k];
  o.chi2_line = L.chi2;
  o.chi2_circle = C.chi2;
  o.pt = Bd / fabs(C.par[2]);
  o.eta = asinh(L.par[0]);
  return ok;
}

// toGlobal of (cxx, 0, cyy), SOARotation.jl:139-147, Float32 as the reference
__device__ __forceinline__ void to_global_cov(const float* R, float cxx, float cxy, float cyy, float* gl) {
  const float xx = R[0], xy = R[1], xz = R[2], yx = R[3], yy = R[4], yz = R[5];
  gl[0] = __fadd_rn(__fmul_rn(xx, __fadd_rn(__fmul_rn(xx, cxx), __fmul_rn(yx, cxy))), __fmul_rn(yx, __fadd_rn(__fmul_rn(xx, cxy), __fmul_rn(yx, cyy))));
  gl[1] = __fadd_rn(__fmul_rn(xx, __fadd_rn(__fmul_rn(xy, cxx), __fmul_rn(yy, cxy))), __fmul_rn(yx, __fadd_rn(__fmul_rn(xy, cxy), __fmul_rn(yy, cyy))));
  gl[2] = __fadd_rn(__fmul_rn(xy, __fadd_rn(__fmul_rn(xy, cxx), __fmul_rn(yy, cxy))), __fmul_rn(yy, __fadd_rn(__fmul_rn(xy, cxy), __fmul_rn(yy, cyy))));
  gl[3] = __fadd_rn(__fmul_rn(xx, __fadd_rn(__fmul_rn(xz, cxx), __fmul_rn(yz, cxy))), __fmul_rn(yx, __fadd_rn(__fmul_rn(xz, cxy), __fmul_rn(yz, cyy))));
  gl[4] = __fadd_rn(__fmul_rn(xy, __fadd_rn(__fmul_rn(xz, cxx), __fmul_rn(yz, cxy))), __fmul_rn(yy, __fadd_rn(__fmul_rn(xz, cxy), __fmul_rn(yz, cyy))));
  gl[5] = __fadd_rn(__fmul_rn(xz, __fadd_rn(__fmul_rn(xz, cxx), __fmul_rn(yz, cxy))), __fmul_rn(yz, __fadd_rn(__fmul_rn(xz, cxy), __fmul_rn(yz, cyy))));
}

}  // namespace bl
}  // namespace pxl
