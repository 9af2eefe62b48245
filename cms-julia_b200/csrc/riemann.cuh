// Riemann helix fit, one thread per track (plugin-PixelTriplets/riemann_fit.jl:
// fast_fit :378-420, circle_fit :445-590 without the covariance propagation,
// line_fit :841-988 and the helpers :31-298). The algorithm is the
// Riemann-Chernov circle fit (hits mapped onto the paraboloid z = x^2 + y^2, the
// circle is the plane through their weighted centre of gravity normal to the
// smallest eigenvector of the weighted scatter matrix) followed by a
// least-squares line fit in the (s, z) plane rotated by the fast-fit angle, both
// with multiple-scattering covariances. Where the Julia port is unfinished the
// ported algorithm is followed: the plane offset c = -v . r0, the fast-fit radius
// and tan(theta) in the line's scattering term, and (phi, d0, pT) from the circle
// geometry (pT = R B).
//
// Precision: T is the type of the per-hit geometry and the circle's scattering model;
// the per-hit projected variances, the line's arc lengths and scattering covariance, the
// inverses of the N x N covariance matrices (Cholesky), the scatter matrix, its 3x3
// eigenproblem and the final parameters are FP64.
#pragma once
#include "bl_fit.cuh"

namespace pxl {
namespace rm {

using bl::s_sqrt;
using bl::s_log;
using bl::s_abs;
using bl::bl_atan2;

// inverse of a symmetric positive-definite N x N matrix via Cholesky (A = L L^T)
template <int N>
BL_HD void chol_inverse(const double A[N][N], double Inv[N][N]) {
  double L[N][N];
#pragma unroll
  for (int j = 0; j < N; ++j) {
    double d = A[j][j];
#pragma unroll
    for (int k = 0; k < j; ++k) d -= L[j][k] * L[j][k];
    const double ljj = sqrt(d), il = 1.0 / ljj;
    L[j][j] = ljj;
#pragma unroll
    for (int i = j + 1; i < N; ++i) {
      double v = A[i][j];
#pragma unroll
      for (int k = 0; k < j; ++k) v -= L[i][k] * L[j][k];
      L[i][j] = v * il;
    }
  }
  // M = L^-1 (lower), Inv = M^T M
  double M[N][N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    M[i][i] = 1.0 / L[i][i];
#pragma unroll
    for (int j = 0; j < i; ++j) {
      double v = 0.0;
#pragma unroll
      for (int k = j; k < i; ++k) v -= L[i][k] * M[k][j];
      M[i][j] = v * M[i][i];
    }
  }
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j <= i; ++j) {
      double v = 0.0;
#pragma unroll
      for (int k = i; k < N; ++k) v += M[k][i] * M[k][j];
      Inv[i][j] = v;
      Inv[j][i] = v;
    }
}

// eigenvector of the smallest eigenvalue of a symmetric 3x3 matrix (cyclic Jacobi, FP64)
BL_HD void min_eigen3(const double Ain[3][3], double v[3], double& lambda) {
  double A[3][3], V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) A[i][j] = Ain[i][j];
  for (int sweep = 0; sweep < 12; ++sweep) {
    const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
    const double dia = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
    if (!(off > 1e-32 * dia)) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (A[p][q] == 0.0) continue;
        const double th = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
        const double t = (th >= 0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 3; ++k) {
          const double akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq;
          A[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k) {
          const double apk = A[p][k], aqk = A[q][k];
          A[p][k] = c * apk - s * aqk;
          A[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < 3; ++k) {
          const double vkp = V[k][p], vkq = V[k][q];
          V[k][p] = c * vkp - s * vkq;
          V[k][q] = s * vkp + c * vkq;
        }
      }
  }
  int m = 0;
  if (A[1][1] < A[m][m]) m = 1;
  if (A[2][2] < A[m][m]) m = 2;
  lambda = A[m][m];
  v[0] = V[0][m]; v[1] = V[1][m]; v[2] = V[2][m];
}

struct RiemannOut {
  double state[5];  // phi, d0, q/pT, cot(theta), zip
  double chi2_circle, chi2_line, pt;
};

// The fit in a frame turned by -theta about the origin (rot; cos, sin = cr, sr): phi is taken
// from the circle centre turned back. ge: the hits' covariances in that frame; ge_glob: in the
// global frame, which cov_carttorad_prefit's projection reads (it takes the direction (1, tan a)
// of a frame-independent angle a against the global axes, so it depends on the frame).
template <int N, class T>
BL_HD bool riemann_fit_frame(const double hits[3][N], const float ge[6][N], const float ge_glob[6][N], double Bd,
                             RiemannOut& o, bool rot, double cr, double sr) {
  // hits relative to hit 0 (FP64 subtraction), absolute hit 0 kept for the radii
  T px[N], py[N], pz[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    px[i] = T(hits[0][i] - hits[0][0]);
    py[i] = T(hits[1][i] - hits[1][0]);
    pz[i] = T(hits[2][i] - hits[2][0]);
  }
  const T B = T(Bd);
  // ---------------------------------------------------------------- fast fit
  constexpr int mid = N / 2;
  T fx, fy, fR, ftan;  // centre relative to hit 0, radius, tan(theta)
  {
    const T b0 = px[mid], b1 = py[mid], c0 = px[N - 1], c1 = py[N - 1];
    const T b2 = b0 * b0 + b1 * b1, c2 = c0 * c0 + c1 * c1;
    const bool flip = s_abs(b0) < s_abs(b1);
    const T bx = flip ? b1 : b0, by = flip ? b0 : b1, cx = flip ? c1 : c0, cy = flip ? c0 : c1;
    const T div = T(2) * bl::diff_of_products<T>(cx, by, bx, cy);
    const T Y0 = (cx * b2 - bx * c2) / div;
    const T X0 = (T(0.5) * b2 - Y0 * by) / bx;
    fx = flip ? Y0 : X0;
    fy = flip ? X0 : Y0;
    fR = s_sqrt<T>(X0 * X0 + Y0 * Y0);
    const T d0 = -fx, d1 = -fy;
    const T cr = d0 * py[N - 1] - d1 * px[N - 1];
    const T dt = d0 * d0 + d1 * d1 + d0 * px[N - 1] + d1 * py[N - 1];
    ftan = fR * bl_atan2<T>(cr, dt) / pz[N - 1];
  }
  // radii from the beam line (absolute coordinates)
  T rad[N];
#pragma unroll
  for (int i = 0; i < N; ++i) rad[i] = T(sqrt(hits[0][i] * hits[0][i] + hits[1][i] * hits[1][i]));
  // centre in absolute coordinates, for the angles seen from the origin
  const T gcx = T(hits[0][0]) + fx, gcy = T(hits[1][0]) + fy;
  // ---------------------------------------------------------------- circle weights
  double Cr[N][N];
  {
    const T p_t = fR * B < T(20) ? fR * B : T(20);
    const T p_2 = p_t * p_t * (T(1) + T(1) / (ftan * ftan));
    T theta = T(atan(double(ftan)));
    if (theta < T(0)) theta += T(bl::kPi);
    const T k3 = s_sqrt<T>(T(1) + T(1) / (ftan * ftan));
    const T x0inv = T(0.06 / 16.0);
    T sv[N], sig2[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
      // angle at the centre between the origin and hit i: -o x p, -o . p with o the centre
      const T qx = T(hits[0][i]) - gcx, qy = T(hits[1][i]) - gcy;
      // the cross product of two vectors a radius long is small against its terms: its two
      // products are compensated in FP32
      sv[i] = s_abs(bl_atan2<T>(bl::diff_of_products<T>(gcy, qx, gcx, qy), -gcx * qx - gcy * qy) * fR);
    }
    const T st = T(sin(double(theta)));
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const T rl = (i == 0 ? sv[0] * k3 : s_abs(sv[i] * k3 - sv[i - 1] * k3)) * x0inv;
      // (1 + 0.038 ln x)^2 x -> 0 as x -> 0: the continuous value where a length rounds to 0
      const T l = rl > T(0) ? T(1) + T(0.038) * s_log<T>(rl) : T(0);
      sig2[i] = l * l * rl * T(0.000225) / (p_2 * st * st);
    }
#pragma unroll
    for (int k = 0; k < N; ++k)
#pragma unroll
      for (int l = k; l < N; ++l) {
        T v = T(0);
#pragma unroll
        for (int i = 0; i <= (k < l ? k : l); ++i) v += (rad[k] - rad[i]) * (rad[l] - rad[i]) * sig2[i];
        Cr[k][l] = double(v);
        Cr[l][k] = double(v);
      }
#pragma unroll
    for (int i = 0; i < N; ++i) {
      // projected variance (cov_carttorad_prefit): its three terms cancel almost exactly
      // for hits near the coordinate axes, so it is evaluated in FP64 in both modes
      const double vxx = ge_glob[0][i], vxy = ge_glob[1][i], vyy = ge_glob[2][i];
      double d;
      if (rad[i] < T(1e-4)) {
        d = vxx;
      } else {
        const double ax = hits[0][i], ay = hits[1][i];
        const double bx = ax - double(gcx), by = ay - double(gcy);
        const double x2 = ax * bx + ay * by, y2 = ax * by - ay * bx;
        const double tc = -y2 / x2, tc2 = tc * tc;
        d = 1.0 / (1.0 + tc2) * (vxx + vyy * tc2 + 2.0 * vxy * tc);
      }
      Cr[i][i] += d;
    }
  }
  double G[N][N];
  chol_inverse<N>(Cr, G);
  double renorm = 0.0;
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) renorm += G[i][j];
  double wgt[N];
#pragma unroll
  for (int j = 0; j < N; ++j) {
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < N; ++i) s += G[i][j];
    wgt[j] = s / renorm;
  }
  // ---------------------------------------------------------------- Riemann-Chernov circle (FP64)
  double hmx = 0.0, hmy = 0.0;
#pragma unroll
  for (int i = 0; i < N; ++i) { hmx += double(px[i]); hmy += double(py[i]); }
  hmx /= N;
  hmy /= N;
  double p3[3][N], q2 = 0.0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    p3[0][i] = double(px[i]) - hmx;
    p3[1][i] = double(py[i]) - hmy;
    q2 += p3[0][i] * p3[0][i] + p3[1][i] * p3[1][i];
  }
  const double s = sqrt(double(N) / q2);
#pragma unroll
  for (int i = 0; i < N; ++i) {
    p3[0][i] *= s;
    p3[1][i] *= s;
    p3[2][i] = p3[0][i] * p3[0][i] + p3[1][i] * p3[1][i];
  }
  double r0[3] = {0, 0, 0};
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int i = 0; i < N; ++i) r0[k] += p3[k][i] * wgt[i];
  double A[3][3];
  {
    double Xm[3][N];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
      for (int i = 0; i < N; ++i) Xm[k][i] = p3[k][i] - r0[k];
    // A = X (G / renorm) X^T
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b) {
        double v = 0.0;
#pragma unroll
        for (int i = 0; i < N; ++i) {
          double gi = 0.0;
#pragma unroll
          for (int j = 0; j < N; ++j) gi += G[i][j] * Xm[b][j];
          v += Xm[a][i] * gi;
        }
        A[a][b] = v / renorm;
        A[b][a] = v / renorm;
      }
  }
  double v[3], lam;
  min_eigen3(A, v, lam);
  if (!(v[2] > 0)) { v[0] = -v[0]; v[1] = -v[1]; v[2] = -v[2]; }
  const double c = -(v[0] * r0[0] + v[1] * r0[1] + v[2] * r0[2]);
  const double hh = sqrt(1.0 - v[2] * v[2] - 4.0 * c * v[2]);
  const double v2x2_inv = 1.0 / (2.0 * v[2]);
  const double uvr2 = hh * v2x2_inv;
  // circle centre relative to hit 0, radius
  const double cx = -v[0] * v2x2_inv / s + hmx, cy = -v[1] * v2x2_inv / s + hmy, R = uvr2 / s;
  const int q = (double(px[1]) * (cy - double(py[0])) - double(py[1]) * (cx - double(px[0]))) > 0 ? -1 : 1;
  o.chi2_circle = fabs(lam) * renorm / ((2.0 * v[2] * uvr2 * s) * (2.0 * v[2] * uvr2 * s));
  // ---------------------------------------------------------------- line fit in the rotated (s, z) plane
  double theta = -q * atan(double(ftan));
  if (theta < 0) theta += bl::kPi;
  double sn, cs;
  sincos(theta, &sn, &cs);
  const T ox = T(cx), oy = T(cy);  // centre relative to hit 0
  const T gox = T(hits[0][0] + cx), goy = T(hits[1][0] + cy);
  T sarc[N], cov_zz[N];
  const T Rt = T(R);
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const T qx = px[i] - ox, qy = py[i] - oy;  // hit - centre
    const T cr = bl::diff_of_products<T>(goy, qx, gox, qy), dt = -gox * qx - goy * qy;
    if constexpr (sizeof(T) == 4) {
      // the arc lengths in FP64: the line of a nearly flat track (cot(theta) ~ 1e-3) with a
      // large chi2 moves with them by more than their FP32 rounding allows
      const double hx = double(px[i]) - cx, hy = double(py[i]) - cy;
      const double gx = hits[0][0] + cx, gy = hits[1][0] + cy;
      sarc[i] = T(-double(q) * atan2(gy * hx - gx * hy, -gx * hx - gy * hy) * R);
    } else {
      const T at = -T(q) * bl_atan2<T>(cr, dt);
      sarc[i] = at * Rt;
    }
    const T temp0 = -T(q) * Rt / (dt * dt + cr * cr);
    const T d_x = temp0 * (goy * dt + gox * cr), d_y = temp0 * (-gox * dt + goy * cr);
    // Jx (V) Jx^T for the (s, z) pair, then the Z' variance after the rotation
    const T vxx = T(ge[0][i]), vxy = T(ge[1][i]), vyy = T(ge[2][i]), vxz = T(ge[3][i]), vyz = T(ge[4][i]),
            vzz = T(ge[5][i]);
    const T t00 = d_x * (vxx * d_x + vxy * d_y) + d_y * (vxy * d_x + vyy * d_y);
    const T t01 = d_x * vxz + d_y * vyz;
    const T t11 = vzz;
    const T r10 = T(-cs), r11 = T(sn);
    cov_zz[i] = r10 * (r10 * t00 + r11 * t01) + r11 * (r10 * t01 + r11 * t11);
  }
  double Cz[N][N];
  {
    // The line's scattering covariance is built in FP64 in both modes: its path lengths S3
    // run from the origin with the absolute z (the reference's choice), so they are large
    // against their differences, and a nearly flat line (cot(theta) ~ 1e-3) through hits with
    // a large chi2 moves with the relative weights by more than the FP32 rounding allows.
    const double ft = double(ftan);
    const double p_t = double(fR * B < T(20) ? fR * B : T(20));
    const double p_2 = p_t * p_t * (1.0 + 1.0 / (ft * ft));
    double S3[N], sig2[N];
    const double x0inv = 0.06 / 16.0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const double si = double(sarc[i]), zi = hits[2][i];
      S3[i] = sqrt(si * si + zi * zi);
    }
#pragma unroll
    for (int i = 0; i < N; ++i) {
      const double rl = (i == 0 ? S3[0] : fabs(S3[i] - S3[i - 1])) * x0inv;
      const double l = rl > 0.0 ? 1.0 + 0.038 * log(rl) : 0.0;
      sig2[i] = 0.000225 / p_2 * (l * l) * rl;
    }
#pragma unroll
    for (int k = 0; k < N; ++k)
#pragma unroll
      for (int l = k; l < N; ++l) {
        double v2 = 0.0;
#pragma unroll
        for (int i = 0; i <= (k < l ? k : l); ++i) v2 += fabs(S3[k] - S3[i]) * fabs(S3[l] - S3[i]) * sig2[i];
        Cz[k][l] = v2 + (k == l ? double(cov_zz[k]) : 0.0);
        Cz[l][k] = Cz[k][l];
      }
  }
  double Vi[N][N];
  chol_inverse<N>(Cz, Vi);
  double xr[N], yr[N];
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const double si = double(sarc[i]), zi = hits[2][i];
    xr[i] = sn * si + cs * zi;
    yr[i] = -cs * si + sn * zi;
  }
  double M00 = 0, M01 = 0, M11 = 0, r0l = 0, r1l = 0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    double wi = 0, wxi = 0, wyi = 0;
#pragma unroll
    for (int j = 0; j < N; ++j) { wi += Vi[i][j]; wxi += Vi[i][j] * xr[j]; wyi += Vi[i][j] * yr[j]; }
    M00 += wi;
    M01 += wxi;
    M11 += xr[i] * wxi;
    r0l += wyi;
    r1l += xr[i] * wyi;
  }
  const double det = M00 * M11 - M01 * M01;
  const double sol0 = (M11 * r0l - M01 * r1l) / det, sol1 = (M00 * r1l - M01 * r0l) / det;
  const double cf = 1.0 / (sn - sol1 * cs);
  double chi2l = 0.0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    double acc = 0;
#pragma unroll
    for (int j = 0; j < N; ++j) acc += Vi[i][j] * (yr[j] - sol0 - sol1 * xr[j]);
    chi2l += (yr[i] - sol0 - sol1 * xr[i]) * acc;
  }
  o.chi2_line = chi2l;
  // ---------------------------------------------------------------- (phi, d0, q/pT, cot(theta), zip)
  double gx = hits[0][0] + cx, gy = hits[1][0] + cy;
  const double rc = sqrt(gx * gx + gy * gy);
  if (rot) {
    const double tx = cr * gx - sr * gy;
    gy = sr * gx + cr * gy;
    gx = tx;
  }
  o.state[0] = atan2(q * gx, -q * gy);
  o.state[1] = q * (rc - R);
  o.pt = R * Bd;
  o.state[2] = q / o.pt;
  o.state[3] = cf * (sol1 * sn + cs);
  o.state[4] = cf * sol0;
  return isfinite(o.state[0]) && isfinite(o.state[2]);
}

// The FP32 fit (T = float) runs in the chord frame of the hits (bl::chord_frame): their
// offsets from hit 0, rounded to FP32, then keep the small component across the chord, which
// carries the curvature, almost exactly. Every quantity but phi is invariant under the turn.
template <int N, class T>
BL_HD bool riemann_fit(const double hits[3][N], const float ge[6][N], double Bd, RiemannOut& o) {
  if constexpr (sizeof(T) == 4) {
    double hr[3][N], cr, sr;
    float gr[6][N];
    bl::chord_frame<N>(hits, ge, false, hr, gr, cr, sr);
    return riemann_fit_frame<N, T>(hr, gr, ge, Bd, o, true, cr, sr);
  } else {
    return riemann_fit_frame<N, T>(hits, ge, ge, Bd, o, false, 1.0, 0.0);
  }
}

}  // namespace rm
}  // namespace pxl
