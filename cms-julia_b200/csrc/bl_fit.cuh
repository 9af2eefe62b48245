// Broken-line helix fit, one thread per track with every array in registers.
// Restates plugin-PixelTriplets/broken_line.jl:46-696 (BL_Fast_fit,
// prepare_broken_line_data, mult_scatt, matrixc_u, BL_Line_fit, BL_Circle_fit,
// translate_karimaki); the reference inverts the band systems with the dense
// Cholesky of cholesky_inversion.jl.
//
// B200 formulation (same mathematics, different evaluation):
//  * Band solve. The line system is pentadiagonal (matrixc_u) and the circle
//    system adds one dense border row for the curvature correction. Both are
//    factorised as L D L^T in O(N), eliminating the hits in reverse order and
//    the border last, so that the covariance entries the fit needs (hits 0, 1
//    and the border) come from the trailing 3x3 block of the inverse alone.
//    The factorisation, the solve and everything downstream of the solution
//    (parameters, Jacobians, Karimaki translations, covariances) are FP64.
//  * Local frame. Hit coordinates are taken relative to hit 0 (subtracted in
//    FP64 on load). Arc lengths and radial residuals are formed from
//    cancellation-free identities: the angle between two radius vectors
//    r0 and r0 + p is atan2(r0 x p, |r0|^2 + r0.p), and |r0 + p| - |r0| =
//    (2 r0.p + |p|^2) / (|r0 + p| + |r0|), with the fast-fit radius taken as
//    |r0| so that the linearisation circle passes exactly through hit 0.
//    The line fit works on (S, Z) relative to hit 0 and moves the intercept
//    back in FP64.
// T is the working type of the hit geometry, the weights, the multiple-
// scattering variances, the band-matrix entries and the chi2: T = double is the
// FP64 fit, T = float the mixed-precision fit.
#pragma once
#include <cmath>
#include <cstdint>

// the fit is host-callable too, so that the formulation can be checked on the CPU
#define BL_HD __host__ __device__ __forceinline__

namespace pxl {
namespace bl {

template <class T> BL_HD T s_sqrt(T x);
template <> BL_HD double s_sqrt<double>(double x) { return sqrt(x); }
template <> BL_HD float s_sqrt<float>(float x) { return sqrtf(x); }
template <class T> BL_HD T s_atan(T x);
template <> BL_HD double s_atan<double>(double x) { return atan(x); }
template <> BL_HD float s_atan<float>(float x) { return atanf(x); }
template <class T> BL_HD T s_log(T x);
template <> BL_HD double s_log<double>(double x) { return log(x); }
template <> BL_HD float s_log<float>(float x) { return logf(x); }
template <class T> BL_HD T s_abs(T x) { return x < T(0) ? -x : x; }

constexpr double kPi = 3.141592653589793;

// custom atan2 of broken_line.jl:256-268: range (-pi/2, 3pi/2)
template <class T>
BL_HD T bl_atan2(T y, T x) {
  if (x > T(0)) return s_atan<T>(y / x);
  if (x < T(0)) return s_atan<T>(y / x) + T(kPi);
  if (y > T(0) && x == T(0)) return T(kPi / 2);
  if (y < T(0) && x == T(0)) return T(-kPi / 2);
  return T(NAN);
}

// multiple-scattering variance of one segment (broken_line.jl:46-57)
template <class T>
BL_HD T mult_scatt(T length, T B, T R, T slope) {
  T pt2 = B * R;
  pt2 = pt2 < T(20.0) ? pt2 : T(20.0);
  pt2 = pt2 * pt2;
  const T XXI_0 = T(0.06 / 16.0);
  const T fact = T(0.7 * ((13.6 / 1000) * (13.6 / 1000)));
  const T abs_len = s_abs(length) * XXI_0;
  const T lt = T(1) + T(0.038) * s_log<T>(abs_len);
  return fact / (pt2 * (T(1) + slope * slope)) * abs_len * (lt * lt);
}

template <class T>
BL_HD void rotation_matrix(T slope, T R[2][2]) {
  const T a = T(1) / s_sqrt<T>(T(1) + slope * slope);
  const T b = slope * a;
  R[0][0] = a; R[0][1] = b; R[1][0] = -b; R[1][1] = a;
}

// Power of the point p with respect to the circle through the local origin whose
// centre is -u: |u + p|^2 - |u|^2 = 2 u.p + |p|^2. For a hit near the circle the two
// terms cancel (u is a radius long, p a chord), so in FP32 the products and sums are
// carried with their exact rounding errors (fma two-product and two-sum, the Dot2
// scheme of Ogita, Rump and Oishi): the result is as accurate as the inputs allow.
template <class T>
BL_HD T power_of_point(T ux, T uy, T px, T py) {
  if constexpr (sizeof(T) == 8) {
    return T(2) * (ux * px + uy * py) + (px * px + py * py);
  } else {
    auto two_sum = [](T a, T b, T& e) { const T s = a + b; const T z = s - a; e = (a - (s - z)) + (b - z); return s; };
    const T p1 = ux * px, e1 = fmaf(ux, px, -p1);
    const T p2 = uy * py, e2 = fmaf(uy, py, -p2);
    const T q1 = px * px, f1 = fmaf(px, px, -q1);
    const T q2 = py * py, f2 = fmaf(py, py, -q2);
    T es, et, eh;
    const T sp = two_sum(p1, p2, es);
    const T sq = two_sum(q1, q2, et);
    const T h = two_sum(T(2) * sp, sq, eh);
    return h + (eh + T(2) * (e1 + e2 + es) + (f1 + f2 + et));
  }
}

// a*d - b*c with the rounding of both products compensated in FP32 (Kahan's
// fma-based difference of products); exact enough for nearly parallel chords
template <class T>
BL_HD T diff_of_products(T a, T d, T b, T c) {
  if constexpr (sizeof(T) == 8) {
    return a * d - b * c;
  } else {
    const T w = b * c;
    const T e = fmaf(-b, c, w);
    const T f = fmaf(a, d, -w);
    return f + e;
  }
}

// --------------------------------------------------------------- band solver
// Symmetric positive-definite system of N hit unknowns (pentadiagonal block)
// and, when Border, one extra unknown coupled to every hit. Arrays are in
// elimination order k = 0..N-1, which is hit N-1-k; the border is eliminated last.
template <int N, bool Border>
struct Band {
  static constexpr int M = N + (Border ? 1 : 0);
  double D[M];   // pivots
  double l1[N];  // L[k][k-1]
  double l2[N];  // L[k][k-2]
  double g[N];   // L[border][k]
};

// d: diagonal, e1[k]: entry (k, k+1), e2[k]: entry (k, k+2), b[k]: (border, k), c: (border, border)
template <int N, bool Border>
BL_HD void band_factor(const double d[N], const double e1[N], const double e2[N],
                                            const double b[N], double c, Band<N, Border>& f) {
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double l2 = 0.0, l1 = 0.0;
    if (k >= 2) l2 = e2[k - 2] / f.D[k - 2];
    if (k >= 1) l1 = (e1[k - 1] - (k >= 2 ? l2 * f.D[k - 2] * f.l1[k - 1] : 0.0)) / f.D[k - 1];
    f.l1[k] = l1;
    f.l2[k] = l2;
    double dk = d[k];
    if (k >= 1) dk -= l1 * l1 * f.D[k - 1];
    if (k >= 2) dk -= l2 * l2 * f.D[k - 2];
    f.D[k] = dk;
    if constexpr (Border) {
      double gk = b[k];
      if (k >= 1) gk -= f.g[k - 1] * f.D[k - 1] * l1;
      if (k >= 2) gk -= f.g[k - 2] * f.D[k - 2] * l2;
      f.g[k] = gk / dk;
    }
  }
  if constexpr (Border) {
    double dn = c;
#pragma unroll
    for (int k = 0; k < N; ++k) dn -= f.g[k] * f.g[k] * f.D[k];
    f.D[N] = dn;
  }
}

// solves the system for a right-hand side that is zero on the border; x[M]
template <int N, bool Border>
BL_HD void band_solve(const Band<N, Border>& f, const double r[N], double x[Band<N, Border>::M]) {
  constexpr int M = Band<N, Border>::M;
  double y[M];
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double v = r[k];
    if (k >= 1) v -= f.l1[k] * y[k - 1];
    if (k >= 2) v -= f.l2[k] * y[k - 2];
    y[k] = v;
  }
  if constexpr (Border) {
    double v = 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) v -= f.g[k] * y[k];
    y[N] = v;
  }
#pragma unroll
  for (int k = 0; k < M; ++k) y[k] /= f.D[k];
  if constexpr (Border) x[N] = y[N];
#pragma unroll
  for (int k = N - 1; k >= 0; --k) {
    double v = y[k];
    if (k + 1 < N) v -= f.l1[k + 1] * x[k + 1];
    if (k + 2 < N) v -= f.l2[k + 2] * x[k + 2];
    if constexpr (Border) v -= f.g[k] * x[N];
    x[k] = v;
  }
}

// trailing block of the inverse: entries among hit 1 (elimination N-2), hit 0
// (elimination N-1) and the border. Inv[a][b] with a, b in {hit0, hit1, border} = {0, 1, 2}.
template <int N, bool Border>
BL_HD void band_trailing_inverse(const Band<N, Border>& f, double inv[3][3]) {
  // L block rows (hit1, hit0, border): [[1,0,0],[a,1,0],[gb,gc,1]]; its inverse is
  // [[1,0,0],[-a,1,0],[a*gc-gb,-gc,1]]
  const double a = f.l1[N - 1];
  double gb = 0.0, gc = 0.0, idn = 0.0;
  if constexpr (Border) {
    gb = f.g[N - 2];
    gc = f.g[N - 1];
    idn = 1.0 / f.D[N];
  }
  const double Mi[3][3] = {{1.0, 0.0, 0.0}, {-a, 1.0, 0.0}, {a * gc - gb, -gc, 1.0}};
  const double iD[3] = {1.0 / f.D[N - 2], 1.0 / f.D[N - 1], idn};
  double blk[3][3];
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      double v = 0.0;
#pragma unroll
      for (int m = 0; m < 3; ++m) v += Mi[m][p] * Mi[m][q] * iD[m];
      blk[p][q] = v;
    }
  // reorder (hit1, hit0, border) -> (hit0, hit1, border)
  const int o[3] = {1, 0, 2};
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int q = 0; q < 3; ++q) inv[p][q] = blk[o[p]][o[q]];
}

// band entries of matrixc_u (broken_line.jl:217-250) for weights w, abscissae S and
// scattering variances VB, in elimination order (k = hit N-1-k)
template <int N, class T>
BL_HD void band_entries(const T w[N], const T S[N], const T VB[N], double d[N], double e1[N],
                                             double e2[N]) {
  T dS[N];  // dS[i] = S[i+1] - S[i]
#pragma unroll
  for (int i = 0; i + 1 < N; ++i) dS[i] = S[i + 1] - S[i];
  dS[N - 1] = T(1);
  T iv[N];  // 1 / VB at the interior hits
#pragma unroll
  for (int i = 0; i < N; ++i) iv[i] = (i > 0 && i < N - 1) ? T(1) / VB[i] : T(0);
#pragma unroll
  for (int i = 0; i < N; ++i) {
    T dg = w[i];
    if (i > 1) dg += iv[i - 1] / (dS[i - 1] * dS[i - 1]);
    if (i > 0 && i < N - 1) {
      const T q = (dS[i] + dS[i - 1]) / (dS[i] * dS[i - 1]);
      dg += iv[i] * (q * q);
    }
    if (i < N - 2) dg += iv[i + 1] / (dS[i] * dS[i]);
    T o1 = T(0), o2 = T(0);
    if (i > 0 && i < N - 1) o1 = -iv[i] / dS[i] * ((dS[i] + dS[i - 1]) / (dS[i] * dS[i - 1]));
    if (i < N - 2) {
      o1 += -iv[i + 1] / dS[i] * ((dS[i + 1] + dS[i]) / (dS[i + 1] * dS[i]));
      o2 = iv[i + 1] / (dS[i + 1] * dS[i]);
    }
    const int k = N - 1 - i;
    d[k] = double(dg);
    // entry (i, i+1) is (k-1, k) in elimination order, (i, i+2) is (k-2, k)
    if (i + 1 < N) e1[k - 1] = double(o1);
    if (i + 2 < N) e2[k - 2] = double(o2);
  }
  e1[N - 1] = 0.0;
  e2[N - 2] = 0.0;
  e2[N - 1] = 0.0;
}

// --------------------------------------------------------------- fit state
template <int N, class T>
struct Geo {
  T p[3][N];     // hit - hit 0
  double h0[3];  // hit 0
};

template <int N, class T>
struct Prep {
  int q;
  T R, f3, slope;
  T cx, cy;       // fast-fit centre relative to hit 0
  T rx[N], ry[N]; // hit - centre
  T s[N];         // arc length relative to hit 0
  double s0;      // arc length of hit 0
  T S[N], Z[N];   // line-fit coordinates relative to hit 0
  T VB[N];
  T Rl[2][2];     // line-fit rotation
};

// BL_Fast_fit (broken_line.jl:275-313) in the frame of hit 0
template <int N, class T>
BL_HD void fast_fit(const Geo<N, T>& G, Prep<N, T>& P) {
  constexpr int mid = N >> 1;
  const T a1 = G.p[0][mid], a2 = G.p[1][mid];
  const T b1 = G.p[0][N - 1] - G.p[0][mid], b2 = G.p[1][N - 1] - G.p[1][mid];
  const T c1 = -G.p[0][N - 1], c2 = -G.p[1][N - 1];
  const T ca = diff_of_products<T>(c1, a2, c2, a1);
  const T nc = c1 * c1 + c2 * c2, na = a1 * a1 + a2 * a2;
  const T tmp = T(0.5) / ca;
  P.cx = -(a2 * nc + c2 * na) * tmp;
  P.cy = (a1 * nc + c1 * na) * tmp;
  P.R = s_sqrt<T>(P.cx * P.cx + P.cy * P.cy);
  // angle from (hit0 - centre) to (hit N-1 - centre)
  const T d1 = -P.cx, d2 = -P.cy;
  const T de = d1 * G.p[1][N - 1] - d2 * G.p[0][N - 1];
  const T dotde = d1 * d1 + d2 * d2 + d1 * G.p[0][N - 1] + d2 * G.p[1][N - 1];
  P.f3 = P.R * bl_atan2<T>(de, dotde) / G.p[2][N - 1];
}

// prepare_broken_line_data (broken_line.jl:150-207)
template <int N, class T>
BL_HD void prepare(const Geo<N, T>& G, T B, Prep<N, T>& P) {
  const T x1 = G.p[0][1], y1 = G.p[1][1];
  const T xn = G.p[0][N - 1] - G.p[0][N - 2], yn = G.p[1][N - 1] - G.p[1][N - 2];
  P.q = (x1 * yn - y1 * xn) > T(0) ? -1 : 1;
  P.slope = -T(P.q) / P.f3;
  rotation_matrix<T>(P.slope, P.Rl);
#pragma unroll
  for (int i = 0; i < N; ++i) { P.rx[i] = G.p[0][i] - P.cx; P.ry[i] = G.p[1][i] - P.cy; }
  const T ux = -P.cx, uy = -P.cy, uu = ux * ux + uy * uy;
  const T fac = T(P.q) * P.R;
  // the reference measures s from the direction centre -> origin: e ~ u - hit0
  const T hx = T(G.h0[0]), hy = T(G.h0[1]);
  P.s0 = double(fac * bl_atan2<T>(-(ux * hy - uy * hx), uu - (ux * hx + uy * hy)));
  P.s[0] = T(0);
#pragma unroll
  for (int i = 1; i < N; ++i)
    P.s[i] = -fac * bl_atan2<T>(ux * G.p[1][i] - uy * G.p[0][i], uu + ux * G.p[0][i] + uy * G.p[1][i]);
#pragma unroll
  for (int i = 0; i < N; ++i) {
    P.S[i] = P.Rl[0][0] * P.s[i] + P.Rl[0][1] * G.p[2][i];
    P.Z[i] = P.Rl[1][0] * P.s[i] + P.Rl[1][1] * G.p[2][i];
  }
  P.VB[0] = T(0);
  P.VB[N - 1] = T(0);
#pragma unroll
  for (int i = 1; i < N - 1; ++i)
    P.VB[i] = mult_scatt<T>(P.S[i + 1] - P.S[i], B, P.R, P.slope) + mult_scatt<T>(P.S[i] - P.S[i - 1], B, P.R, P.slope);
}

BL_HD void sandwich2(const double J[2][2], double C[2][2]) {
  double Tm[2][2], O[2][2];
  for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) Tm[a][b] = J[a][0] * C[0][b] + J[a][1] * C[1][b];
  for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) O[a][b] = Tm[a][0] * J[b][0] + Tm[a][1] * J[b][1];
  for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) C[a][b] = O[a][b];
}

BL_HD void sandwich3(const double J[3][3], double C[3][3]) {
  double Tm[3][3], O[3][3];
  for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) Tm[a][b] = J[a][0] * C[0][b] + J[a][1] * C[1][b] + J[a][2] * C[2][b];
  for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) O[a][b] = Tm[a][0] * J[b][0] + Tm[a][1] * J[b][1] + Tm[a][2] * J[b][2];
  for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) C[a][b] = O[a][b];
}

struct LineOut { double par[2]; double cov[2][2]; double chi2; };
struct CircleOut { double par[3]; double cov[3][3]; int q; double chi2; };

// line-fit weights: 1 / variance of the hit along Z after the rotation (broken_line.jl:560-590)
template <int N, class T>
BL_HD void line_weights(const float ge[6][N], const Prep<N, T>& P, T w[N]) {
  const double tol = 1e-12;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    auto z = [&](float v) { return fabs(double(v)) < tol ? T(0) : T(v); };
    const T V[3][3] = {{T(ge[0][i]), z(ge[1][i]), z(ge[3][i])}, {z(ge[1][i]), T(ge[2][i]), z(ge[4][i])},
                       {z(ge[3][i]), z(ge[4][i]), T(ge[5][i])}};
    const T tmp = T(1) / s_sqrt<T>(P.rx[i] * P.rx[i] + P.ry[i] * P.ry[i]);
    const T J[2][3] = {{P.ry[i] * tmp, -P.rx[i] * tmp, T(0)}, {T(0), T(0), T(1)}};
    // second row of R J V J^T R^T
    T rj[3];
#pragma unroll
    for (int b = 0; b < 3; ++b) rj[b] = P.Rl[1][0] * J[0][b] + P.Rl[1][1] * J[1][b];
    T m22 = T(0);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      T v = T(0);
#pragma unroll
      for (int b = 0; b < 3; ++b) v += V[a][b] * rj[b];
      m22 += rj[a] * v;
    }
    w[i] = T(1) / m22;
  }
}

// line-fit system: weights, band factorisation and solution u (hit order)
template <int N, class T>
BL_HD void line_system(const float ge[6][N], const Prep<N, T>& P, T w[N], Band<N, false>& f, double u[N]) {
  line_weights<N, T>(ge, P, w);
  // assembled in FP64, as the circle system (circle_system)
  double wd[N], Sd[N], VBd[N];
#pragma unroll
  for (int i = 0; i < N; ++i) { wd[i] = double(w[i]); Sd[i] = double(P.S[i]); VBd[i] = double(P.VB[i]); }
  double d[N], e1[N], e2[N], r[N];
  band_entries<N, double>(wd, Sd, VBd, d, e1, e2);
#pragma unroll
  for (int i = 0; i < N; ++i) r[N - 1 - i] = wd[i] * double(P.Z[i]);
  band_factor<N, false>(d, e1, e2, nullptr, 0.0, f);
  double ue[N];
  band_solve<N, false>(f, r, ue);
#pragma unroll
  for (int i = 0; i < N; ++i) u[i] = ue[N - 1 - i];
}

// BL_Line_fit (broken_line.jl:546-696)
template <int N, class T>
BL_HD void line_fit(const float ge[6][N], const Geo<N, T>& G, T B, const Prep<N, T>& P, LineOut& L) {
  T w[N];
  Band<N, false> f;
  double u[N];
  line_system<N, T>(ge, P, w, f, u);
  double I[3][3];
  band_trailing_inverse<N, false>(f, I);
  // absolute position of hit 0 in the rotated (S, Z) frame
  const double Sc = double(P.Rl[0][0]) * P.s0 + double(P.Rl[0][1]) * G.h0[2];
  const double Zc = double(P.Rl[1][0]) * P.s0 + double(P.Rl[1][1]) * G.h0[2];
  const double dS0 = double(P.S[1]) - double(P.S[0]);
  double par0 = (u[1] - u[0]) / dS0;
  double par1 = (u[0] + Zc) - par0 * (double(P.S[0]) + Sc);
  const double idiff = 1.0 / dS0;
  double cov[2][2] = {{(I[0][0] - 2 * I[0][1] + I[1][1]) * (idiff * idiff) +
                           double(mult_scatt<T>(P.S[1] - P.S[0], B, P.R, P.slope)),
                       (I[0][1] - I[0][0]) * idiff},
                      {(I[0][1] - I[0][0]) * idiff, I[0][0]}};
  double jac[2][2] = {{1, 0}, {-(double(P.S[0]) + Sc), 1}};
  sandwich2(jac, cov);
  const double R00 = double(P.Rl[0][0]), R01 = double(P.Rl[0][1]);
  const double j22 = 1.0 / (R00 - par0 * R01);
  jac[0][0] = j22 * j22;
  jac[0][1] = 0;
  jac[1][0] = par1 * R01 * (j22 * j22);
  jac[1][1] = j22;
  par1 = par1 * j22;
  par0 = (R01 + par0 * R00) * j22;
  sandwich2(jac, cov);
  L.par[0] = par0;
  L.par[1] = par1;
  for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) L.cov[a][b] = cov[a][b];
  T chi2 = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const T diff = P.Z[i] - T(u[i]);
    chi2 += w[i] * (diff * diff);
    if (i > 0 && i < N - 1) {
      const T d1 = P.S[i] - P.S[i - 1], d2 = P.S[i + 1] - P.S[i];
      const T t = T(u[i - 1]) / d1 - T(u[i]) * ((d1 + d2) / (d2 * d1)) + T(u[i + 1]) / d2;
      chi2 += (t * t) / P.VB[i];
    }
  }
  L.chi2 = double(chi2);
}

// Karimaki translation of (phi, d, rho) and its covariance to a point (x0, y0) (broken_line.jl:85-127).
// With rot, the fit ran in a frame rotated by -theta (cos, sin = cr, sr): the direction vector
// (C, BB) is turned back by theta before phi is taken, so phi comes out in the global frame and
// on the reference's atan2 branch; d, rho and the covariance do not depend on the frame.
BL_HD void translate_karimaki(CircleOut& c, double x0, double y0, bool rot = false, double cr = 1.0,
                              double sr = 0.0) {
  const double p1 = c.par[0], p2 = c.par[1], p3 = c.par[2];
  double sn, cs;
  sincos(p1, &sn, &cs);
  const double DP = x0 * cs + y0 * sn;
  const double DO = x0 * sn - y0 * cs + p2;
  const double uu = 1.0 + p3 * p2;
  const double C = -p3 * y0 + uu * cs;
  const double BB = p3 * x0 + uu * sn;
  const double A = 2.0 * DO + p3 * (DO * DO + DP * DP);
  const double U = sqrt(1.0 + p3 * A);
  const double xi = 1.0 / (BB * BB + C * C);
  const double v = 1.0 + p3 * DO;
  const double lambda = (0.5 * A) / (U * ((1.0 + U) * (1.0 + U)));
  const double mu = 1.0 / (U * (1.0 + U)) + p3 * lambda;
  const double zeta = DO * DO + DP * DP;
  const double J[3][3] = {{xi * uu * v, -xi * (p3 * p3) * DP, xi * DP},
                          {2.0 * mu * uu * DP, 2.0 * mu * v, mu * zeta - lambda * A},
                          {0.0, 0.0, 1.0}};
  if (rot) c.par[0] = bl_atan2<double>(C * sr + BB * cr, C * cr - BB * sr);
  else c.par[0] = bl_atan2<double>(BB, C);
  c.par[1] = A / (1.0 + U);
  sandwich3(J, c.cov);
}

// circle-fit system: scaled scattering variances, radial residuals, weights, band
// factorisation (border = curvature correction) and solution u[N+1] (hit order)
template <int N, class T>
BL_HD void circle_system(const float ge[6][N], const Geo<N, T>& G, const Prep<N, T>& P, T VB[N], T Z[N], T rn[N],
                         T w[N], Band<N, true>& f, double u[N + 1]) {
  const T ms_scale = T(1.0) + P.slope * P.slope;
#pragma unroll
  for (int i = 0; i < N; ++i) VB[i] = P.VB[i] * ms_scale;
  // radial residuals of the hits to the fast-fit circle, which passes through hit 0
  const T ux = -P.cx, uy = -P.cy;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    rn[i] = s_sqrt<T>(P.rx[i] * P.rx[i] + P.ry[i] * P.ry[i]);
    const T px = G.p[0][i], py = G.p[1][i];
    Z[i] = power_of_point<T>(ux, uy, px, py) / (rn[i] + P.R);
  }
  const double tol = 1e-12;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    auto z = [&](float v) { return fabs(double(v)) < tol ? T(0) : T(v); };
    const T V[2][2] = {{z(ge[0][i]), z(ge[1][i])}, {z(ge[1][i]), z(ge[2][i])}};
    T RR[2][2];
    rotation_matrix<T>(-P.rx[i] / P.ry[i], RR);
    const T t0 = RR[1][0] * V[0][0] + RR[1][1] * V[1][0];
    const T t1 = RR[1][0] * V[0][1] + RR[1][1] * V[1][1];
    w[i] = T(1.0) / (t0 * RR[1][0] + t1 * RR[1][1]);
  }
  // The system is assembled in FP64 from the FP32 weights, arc lengths, scattering variances
  // and residuals: for a stiff track the scattering terms are large and nearly cancel against
  // each other in the elimination, and FP32 entries would cost the curvature correction digits
  // (which the fast-fit curvature then cancels further when the fast fit is far off).
  double wd[N], sd[N], VBd[N];
#pragma unroll
  for (int i = 0; i < N; ++i) { wd[i] = double(w[i]); sd[i] = double(P.s[i]); VBd[i] = double(VB[i]); }
  double d[N], e1[N], e2[N], b[N], r[N];
  band_entries<N, double>(wd, sd, VBd, d, e1, e2);
  const double* s = sd;
  double cnn = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    double v = 0;
    if (i > 0 && i < N - 1) v += -(s[i + 1] - s[i - 1]) * (s[i + 1] - s[i - 1]) / (2.0 * VBd[i] * (s[i + 1] - s[i]) * (s[i] - s[i - 1]));
    if (i > 1) v += (s[i] - s[i - 2]) / (2.0 * VBd[i - 1] * (s[i] - s[i - 1]));
    if (i < N - 2) v += (s[i + 2] - s[i]) / (2.0 * VBd[i + 1] * (s[i + 1] - s[i]));
    b[N - 1 - i] = v;
    r[N - 1 - i] = wd[i] * double(Z[i]);
    if (i > 0 && i < N - 1) cnn += ((s[i + 1] - s[i - 1]) * (s[i + 1] - s[i - 1])) / (4.0 * VBd[i]);
  }
  band_factor<N, true>(d, e1, e2, b, cnn, f);
  double ue[N + 1];
  band_solve<N, true>(f, r, ue);
#pragma unroll
  for (int i = 0; i < N; ++i) u[i] = ue[N - 1 - i];
  u[N] = ue[N];
}

// BL_Circle_fit (broken_line.jl:330-528); returns false where the reference raises. rot, cr,
// sr: the frame rotation of the hits (fit_track), undone on phi.
template <int N, class T>
BL_HD bool circle_fit(const float ge[6][N], const Geo<N, T>& G, T B, const Prep<N, T>& P,
                                           CircleOut& c, bool rot = false, double cr = 1.0, double sr = 0.0) {
  bool ok = true;
  c.q = P.q;
  const T ms_scale = T(1.0) + P.slope * P.slope;
  T VB[N], Z[N], rn[N], w[N];
  Band<N, true> f;
  double u[N + 1];
  circle_system<N, T>(ge, G, P, VB, Z, rn, w, f, u);
  const T* s = P.s;
  double I[3][3];
  band_trailing_inverse<N, true>(f, I);
  // fitted points 0 and 1 (hit-0 frame), FP64 from here on
  const double R = double(P.R);
  const double n0 = double(rn[0]), n1 = double(rn[1]);
  const double r0x = double(P.rx[0]) / n0, r0y = double(P.ry[0]) / n0;
  const double r1x = double(P.rx[1]) / n1, r1y = double(P.ry[1]) / n1;
  const double tmp1 = u[0] - double(Z[0]);
  const double dv0 = tmp1 * r0x, dv1 = tmp1 * r0y;
  const double tmp2 = u[1] - double(Z[1]);
  const double ev0 = double(G.p[0][1]) + tmp2 * r1x, ev1 = double(G.p[1][1]) + tmp2 * r1y;
  const double emd0 = ev0 - dv0, emd1 = ev1 - dv1;
  const double t1 = emd0 * emd0 + emd1 * emd1;
  c.par[0] = bl_atan2<double>(emd1, emd0);
  const double inner = R * R - 0.25 * t1;
  if (inner < 0) ok = false;
  c.par[1] = -double(c.q) * (0.25 * t1) / (R + sqrt(inner));
  c.par[2] = double(c.q) * (1.0 / R + u[N]);
  if (!(double(c.q) * c.par[1] <= 0)) ok = false;
  const double fl = floor(double(c.q) / 2);
  const double den = sqrt((2 * R) * (2 * R) - t1);
  const double J[3][3] = {
      {(r0y * emd0 - emd1 * r0x) / t1, (r1y * emd0 - emd1 * r1x) / t1, 0},
      {fl * (emd0 * r0x + emd1 * r0y) / den, fl * (emd0 * r1x + emd1 * r1y) / den, 0},
      {0, 0, double(c.q)}};
  c.cov[0][0] = I[0][0]; c.cov[0][1] = I[0][1]; c.cov[0][2] = I[0][2];
  c.cov[1][0] = I[1][0]; c.cov[1][1] = I[1][1]; c.cov[1][2] = I[1][2];
  c.cov[2][0] = I[2][0]; c.cov[2][1] = I[2][1]; c.cov[2][2] = I[2][2];
  sandwich3(J, c.cov);
  translate_karimaki(c, 0.5 * emd0, 0.5 * emd1);
  c.cov[0][0] += double(ms_scale * mult_scatt<T>(P.S[1] - P.S[0], B, P.R, P.slope));
  translate_karimaki(c, G.h0[0] + dv0, G.h0[1] + dv1, rot, cr, sr);
  T chi2 = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const T diff = Z[i] - T(u[i]);
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

// The hits and their global covariances turned about the origin by -theta, the angle of the
// chord from the first to the last hit in the transverse plane (cos, sin -> cr, sr), in FP64.
// zero_tiny: global covariance entries below 1e-12 are zeroed first, as the broken-line fit
// of the reference zeroes them.
template <int N>
BL_HD void chord_frame(const double hits[3][N], const float ge_in[6][N], bool zero_tiny, double hr[3][N],
                       float ge[6][N], double& cr, double& sr) {
  const double dx = hits[0][N - 1] - hits[0][0], dy = hits[1][N - 1] - hits[1][0];
  const double l = sqrt(dx * dx + dy * dy);
  cr = 1.0;
  sr = 0.0;
  if (l > 0) { cr = dx / l; sr = dy / l; }
#pragma unroll
  for (int i = 0; i < N; ++i) {
    hr[0][i] = cr * hits[0][i] + sr * hits[1][i];
    hr[1][i] = cr * hits[1][i] - sr * hits[0][i];
    hr[2][i] = hits[2][i];
    auto z = [&](float v) { return zero_tiny && fabs(double(v)) < 1e-12 ? 0.0 : double(v); };
    const double xx = z(ge_in[0][i]), xy = z(ge_in[1][i]), yy = z(ge_in[2][i]);
    const double xz = z(ge_in[3][i]), yz = z(ge_in[4][i]);
    ge[0][i] = float(cr * cr * xx + 2 * cr * sr * xy + sr * sr * yy);
    ge[1][i] = float((cr * cr - sr * sr) * xy + cr * sr * (yy - xx));
    ge[2][i] = float(sr * sr * xx - 2 * cr * sr * xy + cr * cr * yy);
    ge[3][i] = float(cr * xz + sr * yz);
    ge[4][i] = float(cr * yz - sr * xz);
    ge[5][i] = ge_in[5][i];
  }
}

// full fit of one track of N hits: hits[3][N] (FP64 inputs), ge[6][N] (Float32).
// The FP32 fit (T = float) works in the chord frame: the transverse plane turned about the
// origin so that the chord from the first to the last hit lies along x. A hit's offset from
// hit 0 then has a large component along the chord but a small one across it, of the order of
// the sagitta; rounding the offsets to FP32 costs the across component, which carries the
// curvature, almost nothing (in the global frame a 30 cm offset rounds by 2e-6 cm, 3e-5 of a
// 10 GeV track's sagitta). The rotation, the offsets and the hit covariances are turned in FP64
// (global entries below 1e-12 zeroed first, as the reference zeroes them) and phi is turned back
// in the last Karimaki translation; everything else is invariant under the rotation.
template <int N, class T>
BL_HD bool fit_track(const double hits[3][N], const float ge_in[6][N], double Bd, TrackOut& o) {
  Geo<N, T> G;
  constexpr bool rot = sizeof(T) == 4;
  double cr = 1.0, sr = 0.0;
  float ge[6][N];
  if constexpr (rot) {
    double hr[3][N];
    chord_frame<N>(hits, ge_in, true, hr, ge, cr, sr);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      G.h0[a] = hr[a][0];
#pragma unroll
      for (int i = 0; i < N; ++i) G.p[a][i] = T(hr[a][i] - hr[a][0]);
    }
  } else {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      G.h0[a] = hits[a][0];
#pragma unroll
      for (int i = 0; i < N; ++i) G.p[a][i] = T(hits[a][i] - hits[a][0]);
    }
#pragma unroll
    for (int k = 0; k < 6; ++k)
#pragma unroll
      for (int i = 0; i < N; ++i) ge[k][i] = ge_in[k][i];
  }
  const T B = T(Bd);
  Prep<N, T> P;
  fast_fit<N, T>(G, P);
  prepare<N, T>(G, B, P);
  LineOut L;
  line_fit<N, T>(ge, G, B, P, L);
  CircleOut C;
  const bool ok = circle_fit<N, T>(ge, G, B, P, C, rot, cr, sr);
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
