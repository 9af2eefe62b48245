// Test infrastructure (CPU oracle): the Riemann helix fit in FP64, restated from
// plugin-PixelTriplets/riemann_fit.jl (fast_fit :378-420, circle_fit :445-590
// without the covariance propagation, line_fit :841-988, with the helpers
// compute_rad_len_uniform_material :31-39, scatter_cov_line :59-103,
// scatter_cov_rad :112-150, cov_carttorad_prefit :226-256, weight_circle
// :264-266, Charge :275-277, min_eigen3D :292-298).
//
// The Julia file is an unfinished port that is not compiled into the module; the
// restatement follows the algorithm it ports (the Riemann-Chernov circle fit and
// the rotated s-z least-squares line fit) where the port is broken:
//  * circle offset c = -v . r0 (the port sets c = 0, riemann_fit.jl:505-506);
//  * scatter_cov_line reads the fast-fit radius and tan(theta) (the port indexes
//    fast_fit[2] and fast_fit[3], the centre's y and the radius, :66-67);
//  * the (phi, d0, pT) conversion the port calls but never defines (par_urvtopak,
//    :1011) is written from the circle geometry: the track direction at the point
//    of closest approach is the centre direction turned by -q*90 degrees,
//    d0 = q (|centre| - R), pT = R B.
// The symmetric inverses use the same LDL^T inverse as the broken-line oracle, the
// 3x3 eigenproblem a cyclic Jacobi iteration.
#include <algorithm>
#include <cmath>

#include "oracle.h"

namespace orc {

namespace {

constexpr int kMaxN = 8;

double atan2_custom(double y, double x) {  // riemann_fit.jl:338-350
  if (x > 0) return std::atan(y / x);
  if (x < 0) return std::atan(y / x) + M_PI;
  if (y > 0 && x == 0) return M_PI / 2;
  if (y < 0 && x == 0) return -M_PI / 2;
  return NAN;
}

bool inverse(const double* A, int n, double* Inv) {  // symmetric positive definite, L D L^T
  double L[kMaxN][kMaxN] = {}, D[kMaxN], Li[kMaxN][kMaxN] = {};
  for (int j = 0; j < n; ++j) {
    double d = A[j * n + j];
    for (int k = 0; k < j; ++k) d -= L[j][k] * L[j][k] * D[k];
    D[j] = d;
    L[j][j] = 1.0;
    for (int i = j + 1; i < n; ++i) {
      double v = A[i * n + j];
      for (int k = 0; k < j; ++k) v -= L[i][k] * L[j][k] * D[k];
      L[i][j] = v / d;
    }
  }
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

// eigenvector of the smallest eigenvalue of a symmetric 3x3 matrix (cyclic Jacobi)
void min_eigen3(const double A_in[3][3], double v[3], double* lambda) {
  double A[3][3], V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) A[i][j] = A_in[i][j];
  for (int sweep = 0; sweep < 50; ++sweep) {
    const double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
    if (off < 1e-300) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (A[p][q] == 0.0) continue;
        const double th = (A[q][q] - A[p][p]) / (2.0 * A[p][q]);
        const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 3; ++k) {  // A <- J^T A J
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
  for (int i = 1; i < 3; ++i) if (A[i][i] < A[m][m]) m = i;
  *lambda = A[m][m];
  for (int k = 0; k < 3; ++k) v[k] = V[k][m];
}

}  // namespace

int riemann_fit_track(const double* h, const float* ge, int n, double B, double* state5, double* chi2_circle,
                      double* chi2_line, double* pt) {
  if (n < 3 || n > kMaxN) return -1;
  auto X = [&](int i) { return h[3 * i]; };
  auto Y = [&](int i) { return h[3 * i + 1]; };
  auto Zc = [&](int i) { return h[3 * i + 2]; };
  // fast_fit: circle through the first, middle and last hits; tan(theta) from the arc
  double ff[4];
  {
    const int mid = n / 2;
    const double b[2] = {X(mid) - X(0), Y(mid) - Y(0)}, c[2] = {X(n - 1) - X(0), Y(n - 1) - Y(0)};
    const double b2 = b[0] * b[0] + b[1] * b[1], c2 = c[0] * c[0] + c[1] * c[1];
    const bool flip = std::fabs(b[0]) < std::fabs(b[1]);
    const double bx = flip ? b[1] : b[0], by = flip ? b[0] : b[1], cx = flip ? c[1] : c[0], cy = flip ? c[0] : c[1];
    const double div = 2 * (cx * by - bx * cy);
    const double Y0 = (cx * b2 - bx * c2) / div;
    const double X0 = (0.5 * b2 - Y0 * by) / bx;
    ff[0] = X(0) + (flip ? Y0 : X0);
    ff[1] = Y(0) + (flip ? X0 : Y0);
    ff[2] = std::sqrt(X0 * X0 + Y0 * Y0);
    const double d[2] = {X(0) - ff[0], Y(0) - ff[1]}, e[2] = {X(n - 1) - ff[0], Y(n - 1) - ff[1]};
    const double dr = ff[2] * atan2_custom(d[0] * e[1] - d[1] * e[0], d[0] * e[0] + d[1] * e[1]);
    ff[3] = dr / (Zc(n - 1) - Zc(0));
  }
  double rad[kMaxN];
  for (int i = 0; i < n; ++i) rad[i] = std::hypot(X(i), Y(i));
  // ---------------------------------------------------------------- circle fit
  double cov_rad[kMaxN * kMaxN] = {};
  for (int i = 0; i < n; ++i) {  // cov_carttorad_prefit (diagonal)
    const double vxx = ge[6 * i], vxy = ge[6 * i + 1], vyy = ge[6 * i + 2];
    if (rad[i] < 1e-4) {
      cov_rad[i * n + i] = vxx;
    } else {
      const double a[2] = {X(i), Y(i)}, bb[2] = {X(i) - ff[0], Y(i) - ff[1]};
      const double x2 = a[0] * bb[0] + a[1] * bb[1], y2 = a[0] * bb[1] - a[1] * bb[0];
      const double tc = -y2 / x2, tc2 = tc * tc;
      cov_rad[i * n + i] = 1.0 / (1.0 + tc2) * (vxx + vyy * tc2 + 2 * vxy * tc);
    }
  }
  {  // scatter_cov_rad
    const double p_t = std::min(20.0, ff[2] * B);
    const double p_2 = p_t * p_t * (1.0 + 1.0 / (ff[3] * ff[3]));
    double theta = std::atan(ff[3]);
    theta = theta < 0.0 ? theta + M_PI : theta;
    double sv[kMaxN], rl[kMaxN], sig2[kMaxN];
    for (int i = 0; i < n; ++i) {
      const double p[2] = {X(i) - ff[0], Y(i) - ff[1]}, o[2] = {-ff[0], -ff[1]};
      sv[i] = std::fabs(atan2_custom(o[0] * p[1] - o[1] * p[0], o[0] * p[0] + o[1] * p[1]) * ff[2]);
    }
    const double k3 = std::sqrt(1.0 + 1.0 / (ff[3] * ff[3]));
    const double x0inv = 0.06 / 16.0;
    for (int i = 0; i < n; ++i)
      rl[i] = (i == 0 ? sv[0] * k3 : std::fabs(sv[i] * k3 - sv[i - 1] * k3)) * x0inv;
    const double st = std::sin(theta);
    for (int i = 0; i < n; ++i) {
      const double l = 1.0 + 0.038 * std::log(rl[i]);
      sig2[i] = l * l * rl[i] * 0.000225 / (p_2 * st * st);
    }
    for (int k = 0; k < n; ++k)
      for (int l = k; l < n; ++l) {
        double v = 0;
        for (int i = 0; i <= std::min(k, l); ++i) v += (rad[k] - rad[i]) * (rad[l] - rad[i]) * sig2[i];
        cov_rad[k * n + l] += v;
        if (l != k) cov_rad[l * n + k] += v;
      }
  }
  double G[kMaxN * kMaxN];
  inverse(cov_rad, n, G);
  double renorm = 0;
  for (int i = 0; i < n * n; ++i) renorm += G[i];
  for (int i = 0; i < n * n; ++i) G[i] /= renorm;
  double weight[kMaxN];
  for (int j = 0; j < n; ++j) { double s = 0; for (int i = 0; i < n; ++i) s += G[i * n + j]; weight[j] = s; }
  double hm[2] = {0, 0};
  for (int i = 0; i < n; ++i) { hm[0] += X(i); hm[1] += Y(i); }
  hm[0] /= n; hm[1] /= n;
  double p3[3][kMaxN];
  double q2 = 0;
  for (int i = 0; i < n; ++i) {
    p3[0][i] = X(i) - hm[0];
    p3[1][i] = Y(i) - hm[1];
    q2 += p3[0][i] * p3[0][i] + p3[1][i] * p3[1][i];
  }
  const double s = std::sqrt(n / q2);
  for (int i = 0; i < n; ++i) {
    p3[0][i] *= s;
    p3[1][i] *= s;
    p3[2][i] = p3[0][i] * p3[0][i] + p3[1][i] * p3[1][i];
  }
  double r0[3] = {0, 0, 0};
  for (int k = 0; k < 3; ++k) for (int i = 0; i < n; ++i) r0[k] += p3[k][i] * weight[i];
  double Xm[3][kMaxN];
  for (int k = 0; k < 3; ++k) for (int i = 0; i < n; ++i) Xm[k][i] = p3[k][i] - r0[k];
  double A[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double v = 0;
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) v += Xm[a][i] * G[i * n + j] * Xm[b][j];
      A[a][b] = v;
    }
  double v[3], lam;
  min_eigen3(A, v, &lam);
  if (!(v[2] > 0)) { v[0] = -v[0]; v[1] = -v[1]; v[2] = -v[2]; }
  const double c = -(v[0] * r0[0] + v[1] * r0[1] + v[2] * r0[2]);
  const double hh = std::sqrt(1 - v[2] * v[2] - 4 * c * v[2]);
  const double v2x2_inv = 1 / (2 * v[2]);
  const double uvr[3] = {-v[0] * v2x2_inv, -v[1] * v2x2_inv, hh * v2x2_inv};
  const double cpar[3] = {uvr[0] / s + hm[0], uvr[1] / s + hm[1], uvr[2] / s};
  const int q = ((X(1) - X(0)) * (cpar[1] - Y(0)) - (Y(1) - Y(0)) * (cpar[0] - X(0))) > 0 ? -1 : 1;
  *chi2_circle = std::fabs(lam) * renorm / ((2 * v[2] * uvr[2] * s) * (2 * v[2] * uvr[2] * s));
  // ---------------------------------------------------------------- line fit
  double theta = -q * std::atan(ff[3]);
  theta = theta < 0 ? theta + M_PI : theta;
  const double sn = std::sin(theta), cs = std::cos(theta);
  const double rot[2][2] = {{sn, cs}, {-cs, sn}};
  double sarc[kMaxN], zz[kMaxN], cov_zz[kMaxN];
  const double o[2] = {cpar[0], cpar[1]};
  for (int i = 0; i < n; ++i) {
    const double p[2] = {X(i) - o[0], Y(i) - o[1]};
    const double cr = -o[0] * p[1] + o[1] * p[0], dt = -o[0] * p[0] - o[1] * p[1];
    const double at = -q * atan2_custom(cr, dt);
    sarc[i] = at * cpar[2];
    const double temp0 = -q * cpar[2] / (dt * dt + cr * cr);
    const double d_x = temp0 * (o[1] * dt + o[0] * cr), d_y = temp0 * (-o[0] * dt + o[1] * cr);
    const float* g = ge + 6 * i;
    // J = [[d_x, d_y, 0], [0, 0, 1]] on (x, y, z); tmp = J V J^T; cov_sz = rot tmp rot^T
    const double V[3][3] = {{g[0], g[1], g[3]}, {g[1], g[2], g[4]}, {g[3], g[4], g[5]}};
    const double J[2][3] = {{d_x, d_y, 0}, {0, 0, 1}};
    double t[2][2];
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b) {
        double v2 = 0;
        for (int k = 0; k < 3; ++k) for (int l = 0; l < 3; ++l) v2 += J[a][k] * V[k][l] * J[b][l];
        t[a][b] = v2;
      }
    // lower-right entry of rot t rot^T
    cov_zz[i] = rot[1][0] * (rot[1][0] * t[0][0] + rot[1][1] * t[0][1]) + rot[1][1] * (rot[1][0] * t[1][0] + rot[1][1] * t[1][1]);
    zz[i] = Zc(i);
  }
  double cov_ms[kMaxN * kMaxN] = {};
  {  // scatter_cov_line
    const double p_t = std::min(20.0, ff[2] * B);
    const double p_2 = p_t * p_t * (1.0 + 1.0 / (ff[3] * ff[3]));
    double S[kMaxN], rl[kMaxN], sig2[kMaxN];
    for (int i = 0; i < n; ++i) S[i] = std::sqrt(sarc[i] * sarc[i] + zz[i] * zz[i]);
    const double x0inv = 0.06 / 16.0;
    for (int i = 0; i < n; ++i) rl[i] = (i == 0 ? S[0] : std::fabs(S[i] - S[i - 1])) * x0inv;
    for (int i = 0; i < n; ++i) {
      const double l = 1.0 + 0.038 * std::log(rl[i]);
      sig2[i] = 0.000225 / p_2 * (l * l) * rl[i];
    }
    for (int k = 0; k < n; ++k) {
      cov_ms[k * n + k] = cov_zz[k];
      for (int l = k; l < n; ++l) {
        double v2 = 0;
        for (int i = 0; i <= std::min(k, l); ++i) v2 += std::fabs(S[k] - S[i]) * std::fabs(S[l] - S[i]) * sig2[i];
        cov_ms[k * n + l] += v2;
        if (l != k) cov_ms[l * n + k] = cov_ms[k * n + l];
      }
    }
  }
  double xr[kMaxN], yr[kMaxN];
  for (int i = 0; i < n; ++i) {
    xr[i] = rot[0][0] * sarc[i] + rot[0][1] * zz[i];
    yr[i] = rot[1][0] * sarc[i] + rot[1][1] * zz[i];
  }
  double Vi[kMaxN * kMaxN];
  inverse(cov_ms, n, Vi);
  // normal equations of y = p0 + p1 x with weight matrix Vi
  double M[2][2] = {{0, 0}, {0, 0}}, rhs[2] = {0, 0};
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      const double w = Vi[i * n + j];
      M[0][0] += w;
      M[0][1] += w * xr[j];
      M[1][0] += xr[i] * w;
      M[1][1] += xr[i] * w * xr[j];
      rhs[0] += w * yr[j];
      rhs[1] += xr[i] * w * yr[j];
    }
  const double det = M[0][0] * M[1][1] - M[0][1] * M[1][0];
  const double Cp[2][2] = {{M[1][1] / det, -M[0][1] / det}, {-M[1][0] / det, M[0][0] / det}};
  const double sol[2] = {Cp[0][0] * rhs[0] + Cp[0][1] * rhs[1], Cp[1][0] * rhs[0] + Cp[1][1] * rhs[1]};
  const double cf = 1 / (sn - sol[1] * cs);
  const double m = cf * (sol[1] * sn + cs);
  const double zip = cf * sol[0];
  double chi2 = 0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      chi2 += (yr[i] - sol[0] - sol[1] * xr[i]) * Vi[i * n + j] * (yr[j] - sol[0] - sol[1] * xr[j]);
  *chi2_line = chi2;
  // ---------------------------------------------------------------- (phi, d0, q/pT, cot(theta), zip)
  const double rc = std::hypot(cpar[0], cpar[1]);
  state5[0] = std::atan2(q * cpar[0], -q * cpar[1]);
  state5[1] = q * (rc - cpar[2]);
  *pt = cpar[2] * B;
  state5[2] = q / *pt;
  state5[3] = m;
  state5[4] = zip;
  return (std::isfinite(state5[0]) && std::isfinite(state5[2])) ? 0 : 1;
}

}  // namespace orc
