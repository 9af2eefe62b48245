// Test infrastructure (CPU oracle): forward-mode derivatives of the broken-line
// fit's chi2 (chi2_line + chi2_circle) with respect to the hit coordinates.
//
// The chi2 path of the reference fit (broken_line.jl:150-250 prepare_broken_line_data
// and matrixc_u, :275-313 BL_Fast_fit, :330-528 BL_Circle_fit, :546-696 BL_Line_fit,
// with the dense symmetric inverse of cholesky_inversion.jl) is restated here on a
// dual-number scalar (value, derivative): one pass per seeded hit coordinate gives
// one column of the gradient. It follows the reference's own formulation (radius
// from the chord lengths, s measured from the direction of the origin, dense
// inverse), independent of the GPU kernels' reformulated evaluation, so it is a
// second reference for the hand-written adjoint besides finite differences.
#include <algorithm>
#include <cmath>

#include "oracle.h"

namespace orc {

namespace {

struct Dual {
  double v = 0.0, d = 0.0;
  Dual() = default;
  Dual(double x) : v(x), d(0.0) {}  // NOLINT: constants promote implicitly
  Dual(double x, double dx) : v(x), d(dx) {}
};
inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
inline Dual operator-(Dual a) { return {-a.v, -a.d}; }
inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
inline Dual& operator+=(Dual& a, Dual b) { return a = a + b; }
inline Dual& operator-=(Dual& a, Dual b) { return a = a - b; }
inline Dual& operator*=(Dual& a, Dual b) { return a = a * b; }
inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
inline bool operator==(Dual a, Dual b) { return a.v == b.v; }
inline Dual dsqrt(Dual a) { const double s = std::sqrt(a.v); return {s, a.d / (2.0 * s)}; }
inline Dual datan(Dual a) { return {std::atan(a.v), a.d / (1.0 + a.v * a.v)}; }
inline Dual dlog(Dual a) { return {std::log(a.v), a.d / a.v}; }
inline Dual dfabs(Dual a) { return a.v < 0 ? -a : a; }

constexpr int kMaxN = 8;

// custom atan2 of broken_line.jl:256-268
Dual bl_atan2(Dual y, Dual x) {
  if (x.v > 0) return datan(y / x);
  if (x.v < 0) return datan(y / x) + Dual(M_PI);
  if (y.v > 0) return Dual(M_PI / 2);
  if (y.v < 0) return Dual(-M_PI / 2);
  return Dual(NAN);
}

// mult_scatt, broken_line.jl:46-79
Dual mult_scatt(Dual length, double B, Dual R, Dual slope) {
  Dual pt2 = (B * R.v < 20.0) ? Dual(B) * R : Dual(20.0);
  pt2 = pt2 * pt2;
  const double XXI_0 = 0.06 / 16.0;
  const double fact = 0.7 * ((13.6 / 1000) * (13.6 / 1000));
  Dual abs_len = dfabs(length) * Dual(XXI_0);
  Dual lt = Dual(1.0) + Dual(0.038) * dlog(abs_len);
  return Dual(fact) / (pt2 * (Dual(1.0) + slope * slope)) * abs_len * (lt * lt);
}

void rotation_matrix(Dual slope, Dual R[2][2]) {
  Dual a = Dual(1.0) / dsqrt(Dual(1.0) + slope * slope);
  Dual b = slope * a;
  R[0][0] = a; R[0][1] = b; R[1][0] = -b; R[1][1] = a;
}

// dense symmetric inverse by L D L^T
void invert_sym(const Dual* A, int n, Dual* Inv) {
  Dual L[10][10], D[10], Li[10][10];
  for (int j = 0; j < n; ++j) {
    Dual d = A[j * n + j];
    for (int k = 0; k < j; ++k) d -= L[j][k] * L[j][k] * D[k];
    D[j] = d;
    L[j][j] = Dual(1.0);
    for (int i = j + 1; i < n; ++i) {
      Dual v = A[i * n + j];
      for (int k = 0; k < j; ++k) v -= L[i][k] * L[j][k] * D[k];
      L[i][j] = v / d;
    }
  }
  for (int i = 0; i < n; ++i) {
    Li[i][i] = Dual(1.0);
    for (int j = 0; j < i; ++j) {
      Dual v;
      for (int k = j; k < i; ++k) v -= L[i][k] * Li[k][j];
      Li[i][j] = v;
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      Dual v;
      for (int k = i; k < n; ++k) v += Li[k][i] * Li[k][j] / D[k];
      Inv[i * n + j] = v;
      Inv[j * n + i] = v;
    }
}

// matrixc_u into the top-left n x n of C (ld m)
void matrixc_u(const Dual* w, const Dual* S, const Dual* VB, int n, Dual* C, int m) {
  Dual T[kMaxN + 2][kMaxN + 2];
  for (int i = 0; i < n; ++i) {
    T[i][i] = w[i];
    if (i > 1) T[i][i] += Dual(1.0) / (VB[i - 1] * ((S[i] - S[i - 1]) * (S[i] - S[i - 1])));
    if (i > 0 && i < n - 1) {
      Dual q = (S[i + 1] - S[i - 1]) / ((S[i + 1] - S[i]) * (S[i] - S[i - 1]));
      T[i][i] += (Dual(1.0) / VB[i]) * (q * q);
    }
    if (i < n - 2) T[i][i] += Dual(1.0) / (VB[i + 1] * ((S[i + 1] - S[i]) * (S[i + 1] - S[i])));
    if (i > 0 && i < n - 1)
      T[i][i + 1] = Dual(1.0) / (VB[i] * (S[i + 1] - S[i])) * (-(S[i + 1] - S[i - 1]) / ((S[i + 1] - S[i]) * (S[i] - S[i - 1])));
    if (i < n - 2)
      T[i][i + 1] += Dual(1.0) / (VB[i + 1] * (S[i + 1] - S[i])) * (-(S[i + 2] - S[i]) / ((S[i + 2] - S[i + 1]) * (S[i + 1] - S[i])));
    if (i < n - 2) T[i][i + 2] = Dual(1.0) / (VB[i + 1] * (S[i + 2] - S[i + 1]) * (S[i + 1] - S[i]));
    T[i][i] *= Dual(0.5);
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) C[i * m + j] = T[i][j] + T[j][i];
}

// chi2_line + chi2_circle of one track; h row-major per hit (x, y, z), ge per hit (6)
Dual chi2_of(const Dual* h, const float* ge, int n, double B) {
  // BL_Fast_fit
  const int mid = n >> 1;
  const Dual h11 = h[0], h21 = h[1], h1m = h[3 * mid], h2m = h[3 * mid + 1], h1n = h[3 * (n - 1)], h2n = h[3 * (n - 1) + 1];
  const Dual a1 = h1m - h11, a2 = h2m - h21, b1 = h1n - h1m, b2 = h2n - h2m, c1 = h11 - h1n, c2 = h21 - h2n;
  const Dual ca = c1 * a2 - c2 * a1, ba = b1 * a2 - b2 * a1;
  const Dual nc = c1 * c1 + c2 * c2, na = a1 * a1 + a2 * a2, nb = b1 * b1 + b2 * b2;
  const Dual tmp = Dual(0.5) / ca;
  Dual f[4];
  f[0] = h11 - (a2 * nc + c2 * na) * tmp;
  f[1] = h21 + (a1 * nc + c1 * na) * tmp;
  f[2] = dsqrt(na * nb * nc) / (Dual(2.0) * dfabs(ba));
  {
    const Dual d1 = h11 - f[0], d2 = h21 - f[1], e1 = h1n - f[0], e2 = h2n - f[1];
    f[3] = f[2] * bl_atan2(d1 * e2 - d2 * e1, d1 * e1 + d2 * e2) / (h[3 * (n - 1) + 2] - h[2]);
  }
  // prepare_broken_line_data
  const Dual x1 = h[3] - h[0], y1 = h[4] - h[1];
  const Dual xn = h[3 * (n - 1)] - h[3 * (n - 2)], yn = h[3 * (n - 1) + 1] - h[3 * (n - 2) + 1];
  const int q = (x1 * yn - y1 * xn).v > 0 ? -1 : 1;
  const Dual slope = Dual(-double(q)) / f[3];
  Dual R[2][2];
  rotation_matrix(slope, R);
  Dual rx[kMaxN], ry[kMaxN], s[kMaxN], S[kMaxN], Z[kMaxN], VB[kMaxN];
  for (int j = 0; j < n; ++j) { rx[j] = h[3 * j] - f[0]; ry[j] = h[3 * j + 1] - f[1]; }
  const Dual rr = dsqrt(f[0] * f[0] + f[1] * f[1]);
  const Dual sc = -f[2] / rr;
  const Dual e1 = sc * f[0], e2 = sc * f[1];
  const Dual fac = Dual(double(q)) * f[2];
  for (int i = 0; i < n; ++i) s[i] = fac * bl_atan2(rx[i] * e2 - ry[i] * e1, rx[i] * e1 + ry[i] * e2);
  for (int i = 0; i < n; ++i) {
    S[i] = R[0][0] * s[i] + R[0][1] * h[3 * i + 2];
    Z[i] = R[1][0] * s[i] + R[1][1] * h[3 * i + 2];
  }
  VB[0] = Dual(0.0);
  VB[n - 1] = Dual(0.0);
  for (int i = 1; i < n - 1; ++i)
    VB[i] = mult_scatt(S[i + 1] - S[i], B, f[2], slope) + mult_scatt(S[i] - S[i - 1], B, f[2], slope);
  const double tol = 1e-12;
  auto z = [&](float v) { return std::fabs(double(v)) < tol ? Dual(0.0) : Dual(double(v)); };
  // BL_Line_fit chi2
  Dual chi2;
  {
    Dual w[kMaxN];
    for (int i = 0; i < n; ++i) {
      const float* g = ge + 6 * i;
      const Dual V[3][3] = {{Dual(double(g[0])), z(g[1]), z(g[3])}, {z(g[1]), Dual(double(g[2])), z(g[4])},
                            {z(g[3]), z(g[4]), Dual(double(g[5]))}};
      const Dual t = Dual(1.0) / dsqrt(rx[i] * rx[i] + ry[i] * ry[i]);
      const Dual J[2][3] = {{ry[i] * t, -rx[i] * t, Dual(0.0)}, {Dual(0.0), Dual(0.0), Dual(1.0)}};
      Dual rj[3];
      for (int b = 0; b < 3; ++b) rj[b] = R[1][0] * J[0][b] + R[1][1] * J[1][b];
      Dual m22;
      for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) m22 += rj[a] * V[a][b] * rj[b];
      w[i] = Dual(1.0) / m22;
    }
    Dual C[kMaxN * kMaxN], I[kMaxN * kMaxN], u[kMaxN];
    matrixc_u(w, S, VB, n, C, n);
    invert_sym(C, n, I);
    for (int i = 0; i < n; ++i) {
      Dual v;
      for (int k = 0; k < n; ++k) v += I[i * n + k] * (w[k] * Z[k]);
      u[i] = v;
    }
    for (int i = 0; i < n; ++i) {
      const Dual diff = Z[i] - u[i];
      chi2 += w[i] * (diff * diff);
      if (i > 0 && i < n - 1) {
        const Dual d1 = S[i] - S[i - 1], d2 = S[i + 1] - S[i];
        const Dual t = u[i - 1] / d1 - u[i] * ((S[i + 1] - S[i - 1]) / (d2 * d1)) + u[i + 1] / d2;
        chi2 += (t * t) / VB[i];
      }
    }
  }
  // BL_Circle_fit chi2
  {
    Dual VBc[kMaxN], Zc[kMaxN], w[kMaxN];
    for (int i = 0; i < n; ++i) VBc[i] = VB[i] * (Dual(1.0) + slope * slope);
    for (int i = 0; i < n; ++i) Zc[i] = dsqrt(rx[i] * rx[i] + ry[i] * ry[i]) - f[2];
    for (int i = 0; i < n; ++i) {
      const float* g = ge + 6 * i;
      const Dual V[2][2] = {{z(g[0]), z(g[1])}, {z(g[1]), z(g[2])}};
      Dual RR[2][2];
      rotation_matrix(-rx[i] / ry[i], RR);
      const Dual t0 = RR[1][0] * V[0][0] + RR[1][1] * V[1][0];
      const Dual t1 = RR[1][0] * V[0][1] + RR[1][1] * V[1][1];
      w[i] = Dual(1.0) / (t0 * RR[1][0] + t1 * RR[1][1]);
    }
    const int m = n + 1;
    Dual C[(kMaxN + 1) * (kMaxN + 1)], I[(kMaxN + 1) * (kMaxN + 1)], u[kMaxN + 1];
    matrixc_u(w, s, VBc, n, C, m);
    for (int i = 0; i < n; ++i) {
      Dual v;
      if (i > 0 && i < n - 1) v += -(s[i + 1] - s[i - 1]) * (s[i + 1] - s[i - 1]) / (Dual(2.0) * VBc[i] * (s[i + 1] - s[i]) * (s[i] - s[i - 1]));
      if (i > 1) v += (s[i] - s[i - 2]) / (Dual(2.0) * VBc[i - 1] * (s[i] - s[i - 1]));
      if (i < n - 2) v += (s[i + 2] - s[i]) / (Dual(2.0) * VBc[i + 1] * (s[i + 1] - s[i]));
      C[i * m + n] = v;
      C[n * m + i] = v;
      if (i > 0 && i < n - 1) C[n * m + n] += ((s[i + 1] - s[i - 1]) * (s[i + 1] - s[i - 1])) / (Dual(4.0) * VBc[i]);
    }
    invert_sym(C, m, I);
    for (int i = 0; i < m; ++i) {
      Dual v;
      for (int k = 0; k < n; ++k) v += I[i * m + k] * (w[k] * Zc[k]);
      u[i] = v;
    }
    for (int i = 0; i < n; ++i) {
      const Dual diff = Zc[i] - u[i];
      chi2 += w[i] * (diff * diff);
      if (i > 0 && i < n - 1) {
        const Dual d1 = s[i] - s[i - 1], d2 = s[i + 1] - s[i], d3 = s[i + 1] - s[i - 1];
        const Dual t = u[i - 1] / d1 - (u[i] * d3) / (d1 * d2) + u[i + 1] / d2 + (d3 * u[n]) / Dual(2.0);
        chi2 += (t * t) / VBc[i];
      }
    }
  }
  return chi2;
}

}  // namespace

double bl_chi2_grad_fwd(const double* hits, const float* ge, int n, double B, double* grad) {
  if (n < 3 || n > kMaxN) return NAN;
  Dual h[3 * kMaxN];
  double chi2 = 0.0;
  for (int k = 0; k < 3 * n; ++k) {
    for (int j = 0; j < 3 * n; ++j) h[j] = Dual(hits[j], j == k ? 1.0 : 0.0);
    const Dual c = chi2_of(h, ge, n, B);
    grad[k] = c.d;
    chi2 = c.v;
  }
  return chi2;
}

}  // namespace orc
