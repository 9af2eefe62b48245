// Hand-written adjoint of the broken-line fit: d(chi2_line + chi2_circle)/d(hits).
//
// Both broken-line systems are the stationarity conditions of a quadratic form
// in the corrections u: C = (1/2) Hessian(Q) and the right-hand side is w*Z, where
//   Q_line(u)   = sum_i w_i (Z_i - u_i)^2 + sum_kinks beta_i^2 / VB_i,
//   Q_circle(u) = same with the curvature correction u_N added to each kink,
// and the fit's chi2 is Q at the solution u*. By the envelope theorem
// d chi2 / d theta = dQ/d theta at fixed u*, so the backward pass needs no
// adjoint solve: it recomputes the forward fit (nothing is stored between the
// passes), takes the partial derivatives of Q with respect to the weights w,
// residuals Z, abscissae s or S and scattering variances VB, and propagates them
// by hand, in reverse order, through the line weights, the multiple-scattering
// model, the (s, z) rotation, the arc lengths and the fast-fit circle down to the
// hit coordinates. The chi2 is invariant under a common translation of the hits,
// so the hit-0 frame of the forward fit is kept and hit 0 receives minus the sum
// of the others' gradients.
//
// Arithmetic is FP64 throughout (the gradient is checked against central finite
// differences and forward-mode derivatives at 1e-6 relative).
#pragma once
#include "bl_fit.cuh"

namespace pxl {
namespace bl {

// d atan2(y, x) = (x dy - y dx) / (x^2 + y^2)
BL_HD void atan2_adj(double y, double x, double g, double& gy, double& gx) {
  const double r2 = x * x + y * y;
  gy += g * x / r2;
  gx -= g * y / r2;
}

// mult_scatt(L, B, R, m) and its partial derivatives with respect to L, R and m
BL_HD double mult_scatt_d(double L, double B, double R, double m, double& dL, double& dR, double& dm) {
  const double XXI_0 = 0.06 / 16.0;
  const double fact = 0.7 * ((13.6 / 1000) * (13.6 / 1000));
  const double c = 0.038;
  const double br = B * R;
  const bool capped = !(br < 20.0);
  const double pt = capped ? 20.0 : br;
  const double sig = 1.0 + m * m;
  const double K = fact / (pt * pt * sig);
  const double Y = fabs(L) * XXI_0;
  const double l = 1.0 + c * log(Y);
  const double ms = K * Y * (l * l);
  const double sgn = L < 0 ? -1.0 : 1.0;
  dL = K * XXI_0 * sgn * (l * l + 2.0 * c * l);
  dR = capped ? 0.0 : ms * (-2.0 / R);
  dm = ms * (-2.0 * m / sig);
  return ms;
}

// chi2 of the fit and its gradient with respect to the hit coordinates (grad[3][N])
template <int N>
BL_HD double chi2_adjoint(const double hits[3][N], const float ge[6][N], double B, double grad[3][N]) {
  using T = double;
  Geo<N, T> G;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    G.h0[a] = hits[a][0];
#pragma unroll
    for (int i = 0; i < N; ++i) G.p[a][i] = hits[a][i] - hits[a][0];
  }
  // ---------------------------------------------------------------- forward (recomputed)
  Prep<N, T> P;
  fast_fit<N, T>(G, P);
  prepare<N, T>(G, B, P);
  T wl[N];
  Band<N, false> fl;
  double ul[N];
  line_system<N, T>(ge, P, wl, fl, ul);
  T VBc[N], Zc[N], rn[N], wc[N];
  Band<N, true> fc;
  double uc[N + 1];
  circle_system<N, T>(ge, G, P, VBc, Zc, rn, wc, fc, uc);
  const T m = P.slope, a = P.Rl[0][0], b = P.Rl[0][1];
  const T sig = 1.0 + m * m;
  const T* s = P.s;
  const T* S = P.S;
  double chi2 = 0.0;

  // adjoint accumulators
  double gS[N] = {}, gs[N] = {}, gZl[N] = {}, gwl[N] = {}, gVB[N] = {}, gwc[N] = {}, gZc[N] = {};
  double grx[N] = {}, gry[N] = {}, gp[3][N] = {};
  double gm = 0.0, gR = 0.0, ga = 0.0, gb = 0.0;

  // ---------------------------------------------------------------- line chi2 partials
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const double r = P.Z[i] - ul[i];
    chi2 += wl[i] * r * r;
    gwl[i] += r * r;
    gZl[i] += 2.0 * wl[i] * r;
    if (i > 0 && i < N - 1) {
      const double d1 = S[i] - S[i - 1], d2 = S[i + 1] - S[i];
      const double beta = ul[i - 1] / d1 - ul[i] * ((d1 + d2) / (d2 * d1)) + ul[i + 1] / d2;
      chi2 += beta * beta / P.VB[i];
      const double gbeta = 2.0 * beta / P.VB[i];
      gVB[i] += -beta * beta / (P.VB[i] * P.VB[i]);
      const double dd1 = (ul[i] - ul[i - 1]) / (d1 * d1), dd2 = (ul[i] - ul[i + 1]) / (d2 * d2);
      gS[i] += gbeta * (dd1 - dd2);
      gS[i - 1] -= gbeta * dd1;
      gS[i + 1] += gbeta * dd2;
    }
  }
  // ---------------------------------------------------------------- circle chi2 partials
  double gsig = 0.0;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const double r = Zc[i] - uc[i];
    chi2 += wc[i] * r * r;
    gwc[i] += r * r;
    gZc[i] += 2.0 * wc[i] * r;
    if (i > 0 && i < N - 1) {
      const double e1 = s[i] - s[i - 1], e2 = s[i + 1] - s[i], e3 = s[i + 1] - s[i - 1];
      const double t = uc[i - 1] / e1 - (uc[i] * e3) / (e1 * e2) + uc[i + 1] / e2 + (e3 * uc[N]) / 2.0;
      chi2 += t * t / VBc[i];
      const double gt = 2.0 * t / VBc[i];
      const double gvbc = -t * t / (VBc[i] * VBc[i]);
      gVB[i] += gvbc * sig;
      gsig += gvbc * P.VB[i];
      const double dd1 = (uc[i] - uc[i - 1]) / (e1 * e1) + 0.5 * uc[N];
      const double dd2 = (uc[i] - uc[i + 1]) / (e2 * e2) + 0.5 * uc[N];
      gs[i] += gt * (dd1 - dd2);
      gs[i - 1] -= gt * dd1;
      gs[i + 1] += gt * dd2;
    }
  }
  gm += gsig * 2.0 * m;
  // circle weights w = |r|^2 / (r^T V r) and residuals Z = |r| - R
  {
    const double tol = 1e-12;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      auto z = [&](float v) { return fabs(double(v)) < tol ? 0.0 : double(v); };
      const double vxx = z(ge[0][i]), vxy = z(ge[1][i]), vyy = z(ge[2][i]);
      const double rx = P.rx[i], ry = P.ry[i];
      const double Q = rx * rx * vxx + 2.0 * rx * ry * vxy + ry * ry * vyy;
      const double n2 = rx * rx + ry * ry;
      const double dQx = 2.0 * (rx * vxx + ry * vxy), dQy = 2.0 * (ry * vyy + rx * vxy);
      grx[i] += gwc[i] * (2.0 * rx * Q - n2 * dQx) / (Q * Q);
      gry[i] += gwc[i] * (2.0 * ry * Q - n2 * dQy) / (Q * Q);
      grx[i] += gZc[i] * rx / rn[i];
      gry[i] += gZc[i] * ry / rn[i];
      gR -= gZc[i];
    }
  }
  // ---------------------------------------------------------------- multiple scattering VB(S)
#pragma unroll
  for (int i = 1; i < N - 1; ++i) {
    double dL, dR, dm;
    mult_scatt_d(S[i + 1] - S[i], B, P.R, m, dL, dR, dm);
    gS[i + 1] += gVB[i] * dL;
    gS[i] -= gVB[i] * dL;
    gR += gVB[i] * dR;
    gm += gVB[i] * dm;
    mult_scatt_d(S[i] - S[i - 1], B, P.R, m, dL, dR, dm);
    gS[i] += gVB[i] * dL;
    gS[i - 1] -= gVB[i] * dL;
    gR += gVB[i] * dR;
    gm += gVB[i] * dm;
  }
  // ---------------------------------------------------------------- line weights
  {
    const double tol = 1e-12;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      auto z = [&](float v) { return fabs(double(v)) < tol ? 0.0 : double(v); };
      const double V[3][3] = {{double(ge[0][i]), z(ge[1][i]), z(ge[3][i])}, {z(ge[1][i]), double(ge[2][i]), z(ge[4][i])},
                              {z(ge[3][i]), z(ge[4][i]), double(ge[5][i])}};
      const double rx = P.rx[i], ry = P.ry[i];
      const double n = sqrt(rx * rx + ry * ry);
      const double rj[3] = {-b * ry / n, b * rx / n, a};
      // w = 1 / (rj^T V rj): g_rj = -w^2 * 2 V rj * g_w
      const double gm22 = -gwl[i] * wl[i] * wl[i];
      double grj[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) grj[k] = 2.0 * gm22 * (V[k][0] * rj[0] + V[k][1] * rj[1] + V[k][2] * rj[2]);
      gb += grj[0] * (-ry / n) + grj[1] * (rx / n);
      ga += grj[2];
      gry[i] += grj[0] * (-b / n);
      grx[i] += grj[1] * (b / n);
      const double gn = grj[0] * (b * ry / (n * n)) + grj[1] * (-b * rx / (n * n));
      grx[i] += gn * rx / n;
      gry[i] += gn * ry / n;
    }
  }
  // ---------------------------------------------------------------- rotation (S, Z) = R(m) (s, z)
#pragma unroll
  for (int i = 0; i < N; ++i) {
    gs[i] += a * gS[i] - b * gZl[i];
    gp[2][i] += b * gS[i] + a * gZl[i];
    ga += s[i] * gS[i] + G.p[2][i] * gZl[i];
    gb += G.p[2][i] * gS[i] - s[i] * gZl[i];
  }
  gm += ga * (-m * a * a * a) + gb * (a * a * a);
  // ---------------------------------------------------------------- arc lengths s_i = -q R atan2(u x p_i, |u|^2 + u.p_i)
  const double q = P.q;
  const double ux = -P.cx, uy = -P.cy;
  double gux = 0.0, guy = 0.0, guu = 0.0;
#pragma unroll
  for (int i = 1; i < N; ++i) {
    const double px = G.p[0][i], py = G.p[1][i];
    const double cr = ux * py - uy * px, dt = ux * ux + uy * uy + ux * px + uy * py;
    const double alpha = bl_atan2<double>(cr, dt);
    const double galpha = -q * P.R * gs[i];
    gR += -q * alpha * gs[i];
    double gcr = 0.0, gdt = 0.0;
    atan2_adj(cr, dt, galpha, gcr, gdt);
    gux += gcr * py + gdt * px;
    guy += -gcr * px + gdt * py;
    gp[1][i] += gcr * ux + gdt * uy;
    gp[0][i] += -gcr * uy + gdt * ux;
    guu += gdt;
  }
  gux += 2.0 * ux * guu;
  guy += 2.0 * uy * guu;
  double gcx = -gux, gcy = -guy;
  // radii r_i = p_i - c
#pragma unroll
  for (int i = 0; i < N; ++i) {
    gp[0][i] += grx[i];
    gp[1][i] += gry[i];
    gcx -= grx[i];
    gcy -= gry[i];
  }
  // ---------------------------------------------------------------- slope m = -q / f3, f3 = R theta / dz
  constexpr int n1 = N - 1;
  {
    const double gf3 = gm * q / (P.f3 * P.f3);
    const double d1 = -P.cx, d2 = -P.cy;
    const double pnx = G.p[0][n1], pny = G.p[1][n1], pnz = G.p[2][n1];
    const double de = d1 * pny - d2 * pnx;
    const double dotde = d1 * d1 + d2 * d2 + d1 * pnx + d2 * pny;
    const double th = bl_atan2<double>(de, dotde);
    gR += gf3 * th / pnz;
    const double gth = gf3 * P.R / pnz;
    gp[2][n1] += -gf3 * P.R * th / (pnz * pnz);
    double gde = 0.0, gdot = 0.0;
    atan2_adj(de, dotde, gth, gde, gdot);
    double gd1 = gde * pny + gdot * (2.0 * d1 + pnx);
    double gd2 = -gde * pnx + gdot * (2.0 * d2 + pny);
    gp[1][n1] += gde * d1 + gdot * d2;
    gp[0][n1] += -gde * d2 + gdot * d1;
    gcx -= gd1;
    gcy -= gd2;
  }
  // ---------------------------------------------------------------- R = |c|
  gcx += gR * P.cx / P.R;
  gcy += gR * P.cy / P.R;
  // ---------------------------------------------------------------- fast-fit centre (circumcentre of hits 0, mid, N-1)
  {
    constexpr int mid = N >> 1;
    const double a1 = G.p[0][mid], a2 = G.p[1][mid];
    const double c1 = -G.p[0][n1], c2 = -G.p[1][n1];
    const double ca = c1 * a2 - c2 * a1;
    const double nc = c1 * c1 + c2 * c2, na = a1 * a1 + a2 * a2;
    const double tmp = 0.5 / ca;
    const double Nx = a2 * nc + c2 * na, Ny = a1 * nc + c1 * na;
    const double gNx = -gcx * tmp, gNy = gcy * tmp;
    const double gtmp = -gcx * Nx + gcy * Ny;
    const double gca = -gtmp * tmp / ca;
    double ga1 = gNy * nc - gca * c2, ga2 = gNx * nc + gca * c1;
    double gc1 = gNy * na + gca * a2, gc2 = gNx * na - gca * a1;
    const double gnc = gNx * a2 + gNy * a1, gna = gNx * c2 + gNy * c1;
    gc1 += 2.0 * c1 * gnc;
    gc2 += 2.0 * c2 * gnc;
    ga1 += 2.0 * a1 * gna;
    ga2 += 2.0 * a2 * gna;
    gp[0][mid] += ga1;
    gp[1][mid] += ga2;
    gp[0][n1] -= gc1;
    gp[1][n1] -= gc2;
  }
  // ---------------------------------------------------------------- p_i = h_i - h_0
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    double sum = 0.0;
#pragma unroll
    for (int i = 1; i < N; ++i) {
      grad[k][i] = gp[k][i];
      sum += gp[k][i];
    }
    grad[k][0] = -sum;
  }
  return chi2;
}

}  // namespace bl
}  // namespace pxl
