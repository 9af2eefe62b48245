// Test infrastructure (CPU oracle): the broken-line helix fit in FP64 and the
// fit driver over tuples, restated from the reference
// (plugin-PixelTriplets/broken_line.jl:46-528, :546-696,
// broken_line_fit_on_gpu.jl:24-203, cholesky_inversion.jl:3-256,
// SOARotation.jl:139-147, CUDADataFormats/TrajectoryStateSOA.jl:85-109).
// The symmetric inverse is a generic LDL^T inverse written from the
// factorisation; for N <= 5 it is the same algebra as the reference's unrolled
// invert22..invert55 (results agree to rounding). Transcendentals come from
// the C library (the reference uses Julia's own libm), so FP64 results agree
// with the reference to a few ulp, not bit for bit.
#include <algorithm>
#include <cmath>

#include "oracle.h"

namespace orc {

namespace {

constexpr int kMaxN = 8;

// custom atan2 of broken_line.jl:256-268: range (-pi/2, 3pi/2)
inline double bl_atan2(double y, double x) {
  if (x > 0) return std::atan(y / x);
  if (x < 0) return std::atan(y / x) + M_PI;
  if (y > 0 && x == 0) return M_PI / 2;
  if (y < 0 && x == 0) return -M_PI / 2;
  return NAN;
}

inline double sqr(double x) { return x * x; }

// mult_scatt, broken_line.jl:46-79
inline double mult_scatt(double length, double B, double R, double slope) {
  double pt2 = std::min(20.0, B * R);
  pt2 = pt2 * pt2;
  const double XXI_0 = 0.06 / 16.0;
  const double geometry_factor = 0.7;
  const double fact = geometry_factor * ((13.6 / 1000) * (13.6 / 1000));
  double slope_term = 1 + slope * slope;
  double abs_len = std::fabs(length) * XXI_0;
  double log_term = std::log(abs_len);
  double sq = (1 + 0.038 * log_term) * (1 + 0.038 * log_term);
  return fact / (pt2 * slope_term) * abs_len * sq;
}

// symmetric positive-definite inverse by LDL^T (reads the lower triangle only)
bool invert_sym(const double* A, int n, int lda, double* Inv) {
  double L[10][10] = {}, D[10], Li[10][10] = {};
  for (int j = 0; j < n; ++j) {
    double d = A[j * lda + j];
    for (int k = 0; k < j; ++k) d -= L[j][k] * L[j][k] * D[k];
    D[j] = d;
    L[j][j] = 1.0;
    for (int i = j + 1; i < n; ++i) {
      double v = A[i * lda + j];
      for (int k = 0; k < j; ++k) v -= L[i][k] * L[j][k] * D[k];
      L[i][j] = v / d;
    }
  }
  // Li = L^{-1} (unit lower)
  for (int i = 0; i < n; ++i) {
    Li[i][i] = 1.0;
    for (int j = 0; j < i; ++j) {
      double v = 0;
      for (int k = j; k < i; ++k) v -= L[i][k] * Li[k][j];
      Li[i][j] = v;
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      double v = 0;
      for (int k = i; k < n; ++k) v += Li[k][i] * Li[k][j] / D[k];
      Inv[i * n + j] = v;
      Inv[j * n + i] = v;
    }
  return true;
}

struct Prepared {
  int q;
  double radii[2][kMaxN];
  double s[kMaxN], S[kMaxN], Z[kMaxN], VarBeta[kMaxN];
};

struct CircleFit { double par[3]; double cov[3][3]; int32_t q; double chi2; };
struct LineFit { double par[2]; double cov[2][2]; double chi2; };

inline void rotation_matrix(double slope, double R[2][2]) {
  double a = 1.0 / std::sqrt(1.0 + slope * slope);
  double b = slope * a;
  R[0][0] = a; R[0][1] = b; R[1][0] = -b; R[1][1] = a;
}

// BL_Fast_fit, broken_line.jl:275-313; hits column-major 3xN
void fast_fit(const double* h, int n, double* r) {
  int mid = (n >> 1);
  double h11 = h[0], h21 = h[1], h1m = h[3 * mid], h2m = h[3 * mid + 1], h1n = h[3 * (n - 1)], h2n = h[3 * (n - 1) + 1];
  double a1 = h1m - h11, a2 = h2m - h21, b1 = h1n - h1m, b2 = h2n - h2m, c1 = h11 - h1n, c2 = h21 - h2n;
  double ca = c1 * a2 - c2 * a1, ba = b1 * a2 - b2 * a1;
  double nc = c1 * c1 + c2 * c2, na = a1 * a1 + a2 * a2, nb = b1 * b1 + b2 * b2;
  double tmp = 0.5 / ca;
  r[0] = h11 - (a2 * nc + c2 * na) * tmp;
  r[1] = h21 + (a1 * nc + c1 * na) * tmp;
  r[2] = std::sqrt(na * nb * nc) / (2.0 * std::fabs(ba));
  double cx = r[0], cy = r[1];
  double d1 = h11 - cx, d2 = h21 - cy, e1 = h1n - cx, e2 = h2n - cy;
  double de = d1 * e2 - d2 * e1, dotde = d1 * e1 + d2 * e2;
  double dz = h[3 * (n - 1) + 2] - h[2];
  r[3] = r[2] * bl_atan2(de, dotde) / dz;
}

// prepare_broken_line_data, broken_line.jl:150-207
void prepare(const double* h, int n, const double* f, double B, Prepared& d) {
  double x1 = h[3] - h[0], y1 = h[4] - h[1];
  double xn = h[3 * (n - 1)] - h[3 * (n - 2)], yn = h[3 * (n - 1) + 1] - h[3 * (n - 2) + 1];
  d.q = (x1 * yn - y1 * xn) > 0 ? -1 : 1;
  double slope = -double(d.q) / f[3];
  double R[2][2];
  rotation_matrix(slope, R);
  for (int j = 0; j < n; ++j) { d.radii[0][j] = h[3 * j] - f[0]; d.radii[1][j] = h[3 * j + 1] - f[1]; }
  double rr = std::sqrt(f[0] * f[0] + f[1] * f[1]);
  double sc = -f[2] / rr;
  double e1 = sc * f[0], e2 = sc * f[1];
  double fac = d.q * f[2];
  for (int i = 0; i < n; ++i) {
    double xi = d.radii[0][i], yi = d.radii[1][i];
    double c = xi * e2 - yi * e1, dd = xi * e1 + yi * e2;
    d.s[i] = fac * bl_atan2(c, dd);
  }
  for (int i = 0; i < n; ++i) {
    double xi = d.s[i], yi = h[3 * i + 2];
    d.S[i] = R[0][0] * xi + R[0][1] * yi;
    d.Z[i] = R[1][0] * xi + R[1][1] * yi;
  }
  d.VarBeta[0] = 0; d.VarBeta[n - 1] = 0;
  for (int i = 1; i < n - 1; ++i) {
    double d1 = d.S[i + 1] - d.S[i], d2 = d.S[i] - d.S[i - 1];
    d.VarBeta[i] = mult_scatt(d1, B, f[2], slope) + mult_scatt(d2, B, f[2], slope);
  }
}

// matrixc_u, broken_line.jl:217-250 (0-based i); returns the symmetric n x n matrix (ld = ldc)
void matrixc_u(const double* w, const double* S, const double* VB, int n, double* C, int ldc) {
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) C[i * ldc + j] = 0;
  double T[kMaxN + 2][kMaxN + 2] = {};
  for (int i = 0; i < n; ++i) {
    T[i][i] = w[i];
    if (i > 1) T[i][i] += 1.0 / (VB[i - 1] * sqr(S[i] - S[i - 1]));
    if (i > 0 && i < n - 1)
      T[i][i] += (1.0 / VB[i]) * sqr((S[i + 1] - S[i - 1]) / ((S[i + 1] - S[i]) * (S[i] - S[i - 1])));
    if (i < n - 2) T[i][i] += 1.0 / (VB[i + 1] * sqr(S[i + 1] - S[i]));
    if (i > 0 && i < n - 1)
      T[i][i + 1] = 1.0 / (VB[i] * (S[i + 1] - S[i])) * (-(S[i + 1] - S[i - 1]) / ((S[i + 1] - S[i]) * (S[i] - S[i - 1])));
    if (i < n - 2)
      T[i][i + 1] += 1.0 / (VB[i + 1] * (S[i + 1] - S[i])) * (-(S[i + 2] - S[i]) / ((S[i + 2] - S[i + 1]) * (S[i + 1] - S[i])));
    if (i < n - 2) T[i][i + 2] = 1.0 / (VB[i + 1] * (S[i + 2] - S[i + 1]) * (S[i + 1] - S[i]));
    T[i][i] *= 0.5;
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) C[i * ldc + j] = T[i][j] + T[j][i];
}

// BL_Line_fit, broken_line.jl:546-696; ge column-major 6xN (Float32 values)
void line_fit(const float* ge, int n, const double* f, double B, const Prepared& d, LineFit& L) {
  double slope = -double(d.q) / f[3];
  double R[2][2];
  rotation_matrix(slope, R);
  const double tol = 1e-12;
  double w[kMaxN];
  for (int i = 0; i < n; ++i) {
    const float* g = ge + 6 * i;
    auto z = [&](float v) { return std::fabs(double(v)) < tol ? 0.0 : double(v); };
    double V[3][3] = {{double(g[0]), z(g[1]), z(g[3])}, {z(g[1]), double(g[2]), z(g[4])}, {z(g[3]), z(g[4]), double(g[5])}};
    double tmp = 1 / std::sqrt(d.radii[0][i] * d.radii[0][i] + d.radii[1][i] * d.radii[1][i]);
    double J[2][3] = {{d.radii[1][i] * tmp, -d.radii[0][i] * tmp, 0}, {0, 0, 1.0}};
    double M1[2][3], M2[2][3], M3[2][2], M4[2][2];
    for (int a = 0; a < 2; ++a) for (int b = 0; b < 3; ++b) M1[a][b] = R[a][0] * J[0][b] + R[a][1] * J[1][b];
    for (int a = 0; a < 2; ++a) for (int b = 0; b < 3; ++b) M2[a][b] = M1[a][0] * V[0][b] + M1[a][1] * V[1][b] + M1[a][2] * V[2][b];
    for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) M3[a][b] = M2[a][0] * J[b][0] + M2[a][1] * J[b][1] + M2[a][2] * J[b][2];
    for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) M4[a][b] = M3[a][0] * R[b][0] + M3[a][1] * R[b][1];
    w[i] = 1.0 / M4[1][1];
  }
  double r_u[kMaxN];
  for (int i = 0; i < n; ++i) r_u[i] = w[i] * d.Z[i];
  double C[kMaxN * kMaxN], I[kMaxN * kMaxN];
  matrixc_u(w, d.S, d.VarBeta, n, C, n);
  invert_sym(C, n, n, I);
  double u[kMaxN];
  for (int i = 0; i < n; ++i) { double v = 0; for (int k = 0; k < n; ++k) v += I[i * n + k] * r_u[k]; u[i] = v; }
  L.par[0] = (u[1] - u[0]) / (d.S[1] - d.S[0]);
  L.par[1] = u[0];
  double idiff = 1.0 / (d.S[1] - d.S[0]);
  double I11 = I[0], I12 = I[1], I22 = I[n + 1];
  double cov[2][2] = {{(I11 - 2 * I12 + I22) * sqr(idiff) + mult_scatt(d.S[1] - d.S[0], B, f[2], slope), (I12 - I11) * idiff},
                      {(I12 - I11) * idiff, I11}};
  double jac[2][2] = {{1, 0}, {-d.S[0], 1}};
  L.par[1] = L.par[1] - L.par[0] * d.S[0];
  auto sandwich2 = [](double J[2][2], double Cv[2][2]) {
    double T[2][2], O[2][2];
    for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) T[a][b] = J[a][0] * Cv[0][b] + J[a][1] * Cv[1][b];
    for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) O[a][b] = T[a][0] * J[b][0] + T[a][1] * J[b][1];
    for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) Cv[a][b] = O[a][b];
  };
  sandwich2(jac, cov);
  double tmp = R[0][0] - L.par[0] * R[0][1];
  jac[1][1] = 1 / tmp;
  jac[0][0] = jac[1][1] * jac[1][1];
  jac[0][1] = 0;
  jac[1][0] = L.par[1] * R[0][1] * jac[0][0];
  L.par[1] = L.par[1] * jac[1][1];
  L.par[0] = (R[0][1] + L.par[0] * R[0][0]) * jac[1][1];
  sandwich2(jac, cov);
  for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) L.cov[a][b] = cov[a][b];
  double chi2 = 0;
  for (int i = 0; i < n; ++i) {
    double diff = d.Z[i] - u[i];
    chi2 += w[i] * (diff * diff);
    if (i > 0 && i < n - 1) {
      double den1 = d.S[i] - d.S[i - 1], den2 = d.S[i + 1] - d.S[i], den3 = d.S[i] - d.S[i - 1], den4 = d.S[i + 1] - d.S[i - 1];
      double t = (u[i - 1] / den1) - (u[i] * (den4 / (den2 * den3))) + (u[i + 1] / (d.S[i + 1] - d.S[i]));
      chi2 += (t * t) / d.VarBeta[i];
    }
  }
  L.chi2 = chi2;
}

void sandwich3(const double J[3][3], double C[3][3]) {
  double T[3][3], O[3][3];
  for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) T[a][b] = J[a][0] * C[0][b] + J[a][1] * C[1][b] + J[a][2] * C[2][b];
  for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) O[a][b] = T[a][0] * J[b][0] + T[a][1] * J[b][1] + T[a][2] * J[b][2];
  for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) C[a][b] = O[a][b];
}

// translate_karimaki, broken_line.jl:103-132
void translate_karimaki(CircleFit& c, double x0, double y0) {
  double p1 = c.par[0], p2 = c.par[1], p3 = c.par[2];
  double DP = x0 * std::cos(p1) + y0 * std::sin(p1);
  double DO = x0 * std::sin(p1) - y0 * std::cos(p1) + p2;
  double uu = 1 + p3 * p2;
  double C = -p3 * y0 + uu * std::cos(p1);
  double BB = p3 * x0 + uu * std::sin(p1);
  double A = 2.0 * DO + p3 * (DO * DO + DP * DP);
  double U = std::sqrt(1.0 + p3 * A);
  double xi = 1.0 / (BB * BB + C * C);
  double v = 1.0 + p3 * DO;
  double lambda = (0.5 * A) / (U * ((1.0 + U) * (1.0 + U)));
  double mu = 1.0 / (U * (1.0 + U)) + p3 * lambda;
  double zeta = DO * DO + DP * DP;
  double J[3][3] = {{xi * uu * v, -xi * (p3 * p3) * DP, xi * DP},
                    {2.0 * mu * uu * DP, 2.0 * mu * v, mu * zeta - lambda * A},
                    {0.0, 0.0, 1.0}};
  c.par[0] = bl_atan2(BB, C);
  c.par[1] = A / (1.0 + U);
  sandwich3(J, c.cov);
}

// BL_Circle_fit, broken_line.jl:330-528
bool circle_fit(const double* h, const float* ge, int n, const double* f, double B, Prepared& d, CircleFit& c) {
  bool domain_ok = true;
  c.q = d.q;
  double slope = -double(c.q) / f[3];
  double VB[kMaxN];
  for (int i = 0; i < n; ++i) VB[i] = d.VarBeta[i] * (1.0 + slope * slope);
  for (int i = 0; i < n; ++i) d.Z[i] = std::sqrt(d.radii[0][i] * d.radii[0][i] + d.radii[1][i] * d.radii[1][i]) - f[2];
  const double tol = 1e-12;
  double w[kMaxN];
  for (int i = 0; i < n; ++i) {
    const float* g = ge + 6 * i;
    auto z = [&](float v) { return std::fabs(double(v)) < tol ? 0.0 : double(v); };
    double V[2][2] = {{z(g[0]), z(g[1])}, {z(g[1]), z(g[2])}};
    double RR[2][2];
    rotation_matrix(-d.radii[0][i] / d.radii[1][i], RR);
    double T[2][2];
    for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) T[a][b] = RR[a][0] * V[0][b] + RR[a][1] * V[1][b];
    double m22 = T[1][0] * RR[1][0] + T[1][1] * RR[1][1];
    w[i] = 1.0 / m22;
  }
  const int m = n + 1;
  double r_u[kMaxN + 1];
  for (int i = 0; i < n; ++i) r_u[i] = w[i] * d.Z[i];
  r_u[n] = 0;
  double C[(kMaxN + 1) * (kMaxN + 1)] = {};
  matrixc_u(w, d.s, VB, n, C, m);
  C[n * m + n] = 0.0;
  const double* s = d.s;
  for (int i = 0; i < n; ++i) {
    double v = 0.0;
    if (i > 0 && i < n - 1) v += -(s[i + 1] - s[i - 1]) * (s[i + 1] - s[i - 1]) / (2.0 * VB[i] * (s[i + 1] - s[i]) * (s[i] - s[i - 1]));
    if (i > 1) v += (s[i] - s[i - 2]) / (2.0 * VB[i - 1] * (s[i] - s[i - 1]));
    if (i < n - 2) v += (s[i + 2] - s[i]) / (2.0 * VB[i + 1] * (s[i + 1] - s[i]));
    C[i * m + n] = v;
    C[n * m + i] = v;
    if (i > 0 && i < n - 1) C[n * m + n] += sqr(s[i + 1] - s[i - 1]) / (4.0 * VB[i]);
  }
  double I[(kMaxN + 1) * (kMaxN + 1)];
  invert_sym(C, m, m, I);
  double u[kMaxN + 1];
  for (int i = 0; i < m; ++i) { double v = 0; for (int k = 0; k < m; ++k) v += I[i * m + k] * r_u[k]; u[i] = v; }
  for (int col = 0; col < 2; ++col) {
    double t = std::sqrt(d.radii[0][col] * d.radii[0][col] + d.radii[1][col] * d.radii[1][col]);
    d.radii[0][col] /= t;
    d.radii[1][col] /= t;
  }
  double tmp1 = -d.Z[0] + u[0];
  double dv[2] = {h[0] + tmp1 * d.radii[0][0], h[1] + tmp1 * d.radii[1][0]};
  double tmp2 = -d.Z[1] + u[1];
  double ev[2] = {h[3] + tmp2 * d.radii[0][1], h[4] + tmp2 * d.radii[1][1]};
  double emd[2] = {ev[0] - dv[0], ev[1] - dv[1]};
  double nrm = std::sqrt(emd[0] * emd[0] + emd[1] * emd[1]);
  c.par[0] = bl_atan2(emd[1], emd[0]);
  double inner = sqr(f[2]) - 0.25 * (nrm * nrm);
  if (inner < 0) domain_ok = false;
  c.par[1] = -c.q * (f[2] - std::sqrt(inner));
  c.par[2] = c.q * (1.0 / f[2] + u[n]);
  if (!(c.q * c.par[1] <= 0)) domain_ok = false;
  double t1 = nrm * nrm;
  double fl = std::floor(double(c.q) / 2);
  double den = std::sqrt(sqr(2 * f[2]) - t1);
  double J[3][3] = {{(d.radii[1][0] * emd[0] - emd[1] * d.radii[0][0]) / t1, (d.radii[1][1] * emd[0] - emd[1] * d.radii[0][1]) / t1, 0},
                    {fl * (emd[0] * d.radii[0][0] + emd[1] * d.radii[1][0]) / den, fl * (emd[0] * d.radii[0][1] + emd[1] * d.radii[1][1]) / den, 0},
                    {0, 0, double(c.q)}};
  c.cov[0][0] = I[0]; c.cov[0][1] = I[1]; c.cov[0][2] = I[n];
  c.cov[1][0] = I[m]; c.cov[1][1] = I[m + 1]; c.cov[1][2] = I[m + n];
  c.cov[2][0] = I[n * m]; c.cov[2][1] = I[n * m + 1]; c.cov[2][2] = I[n * m + n];
  sandwich3(J, c.cov);
  translate_karimaki(c, 0.5 * emd[0], 0.5 * emd[1]);
  c.cov[0][0] += (1 + slope * slope) * mult_scatt(d.S[1] - d.S[0], B, f[2], slope);
  translate_karimaki(c, dv[0], dv[1]);
  double chi2 = 0.0;
  for (int i = 0; i < n; ++i) {
    double diff = d.Z[i] - u[i];
    chi2 += w[i] * (diff * diff);
    if (i > 0 && i < n - 1) {
      double d1 = s[i] - s[i - 1], d2 = s[i + 1] - s[i], d3 = s[i + 1] - s[i - 1];
      double t = u[i - 1] / d1 - (u[i] * d3) / (d1 * d2) + u[i + 1] / d2 + (d3 * u[n]) / 2.0;
      chi2 += (t * t) / VB[i];
    }
  }
  c.chi2 = chi2;
  return domain_ok;
}

// toGlobal of a local (cxx, cxy, cyy) covariance, SOARotation.jl:139-147 (Float32)
void to_global_cov(const float* R, float cxx, float cxy, float cyy, float* gl) {
  float xx = R[0], xy = R[1], xz = R[2], yx = R[3], yy = R[4], yz = R[5];
  gl[0] = xx * (xx * cxx + yx * cxy) + yx * (xx * cxy + yx * cyy);
  gl[1] = xx * (xy * cxx + yy * cxy) + yx * (xy * cxy + yy * cyy);
  gl[2] = xy * (xy * cxx + yy * cxy) + yy * (xy * cxy + yy * cyy);
  gl[3] = xx * (xz * cxx + yz * cxy) + yx * (xz * cxy + yz * cyy);
  gl[4] = xy * (xz * cxx + yz * cxy) + yy * (xz * cxy + yz * cyy);
  gl[5] = xz * (xz * cxx + yz * cxy) + yz * (xz * cxy + yz * cyy);
}

}  // namespace

int bl_fit_track(const double* hits, const float* ge, int n, double B, double* state5, double* cov15, double* chi2_line,
                 double* chi2_circle, double* pt, double* eta, double* fast4) {
  if (n < 3 || n > kMaxN) return -1;
  double f[4];
  fast_fit(hits, n, f);
  if (fast4) for (int k = 0; k < 4; ++k) fast4[k] = f[k];
  Prepared d;
  prepare(hits, n, f, B, d);
  LineFit L;
  line_fit(ge, n, f, B, d, L);
  CircleFit C;
  bool ok = circle_fit(hits, ge, n, f, B, d, C);
  double b = 1.0 / B;  // copyFromCircle!(…, 1.0f0 / B, …)
  state5[0] = C.par[0]; state5[1] = C.par[1]; state5[2] = C.par[2] * b; state5[3] = L.par[0]; state5[4] = L.par[1];
  double cv[15] = {C.cov[0][0], C.cov[0][1], b * C.cov[0][2], 0.0, 0.0, C.cov[1][1], b * C.cov[1][2], 0.0, 0.0,
                   (b * b) * C.cov[2][2], 0.0, 0.0, L.cov[0][0], L.cov[0][1], L.cov[1][1]};
  for (int k = 0; k < 15; ++k) cov15[k] = cv[k];
  *chi2_line = L.chi2;
  *chi2_circle = C.chi2;
  *pt = B / std::fabs(C.par[2]);
  *eta = std::asinh(L.par[0]);
  return ok ? 0 : 1;
}

// launchBrokenLineKernelsOnCPU, broken_line_fit_on_gpu.jl:166-203
void fit_tuples(const Conditions& cond, EventOut& ev) {
  const double B = double(float(0.0114256972711507));
  const uint32_t nb = ev.caps.tuples;
  ev.pt.assign(nb, 0.f); ev.eta.assign(nb, 0.f); ev.chi2.assign(nb, 0.f);
  ev.state.assign(size_t(nb) * 5, 0.f); ev.cov.assign(size_t(nb) * 15, 0.f);
  ev.fitted.assign(nb, 0);
  const int passes[3][2] = {{3, 3}, {4, 4}, {4, 5}};  // (hits in fit, multiplicity bin); fit5as4
  for (auto& ps : passes) {
    int N = ps[0], nb = ps[1];
    uint32_t b0 = ev.tm_off[nb - 1], b1 = ev.tm_off[nb];
    uint32_t cnt = b1 - b0;
    if (cnt > ev.caps.fits_per_mult) { ev.flags |= kFlagFitsCapped; cnt = ev.caps.fits_per_mult; }
    for (uint32_t t = 0; t < cnt; ++t) {
      uint32_t tk = ev.tm_bins[b0 + t];
      uint32_t hs = ev.tuple_off[tk - 1];  // 1-based start
      double h[3 * kMaxN];
      float g[6 * kMaxN];
      for (int i = 0; i < N; ++i) {
        uint32_t hit = ev.tuple_hits[hs - 1 + i];
        int det = ev.det_ind[hit - 1];
        const DetParams& dp = cond.cpe.det[det];
        to_global_cov(dp.R, float(ev.xerr[hit - 1]), 0.0f, ev.yerr[hit - 1], g + 6 * i);
        h[3 * i] = ev.xg[hit - 1]; h[3 * i + 1] = ev.yg[hit - 1]; h[3 * i + 2] = ev.zg[hit - 1];
      }
      double st[5], cv[15], cl, cc, pt, eta;
      int rc = bl_fit_track(h, g, N, B, st, cv, &cl, &cc, &pt, &eta, nullptr);
      if (rc) ev.flags |= kFlagFitDomain;
      for (int k = 0; k < 5; ++k) ev.state[size_t(tk - 1) * 5 + k] = float(st[k]);
      for (int k = 0; k < 15; ++k) ev.cov[size_t(tk - 1) * 15 + k] = float(cv[k]);
      ev.pt[tk - 1] = float(pt);
      ev.eta[tk - 1] = float(eta);
      ev.chi2[tk - 1] = float((cl + cc) / double(2 * N - 5));
      ev.fitted[tk - 1] = 1;
    }
  }
}

}  // namespace orc
