// Boys function F_m(T) = int_0^1 t^(2m) exp(-T t^2) dt, orders 0..M at once.
//
// Three regimes (the method of Helgaker, Jorgensen & Olsen, Molecular
// Electronic-Structure Theory, sec. 9.8.2: tabulated Taylor expansion plus
// asymptotic form, with the standard recursions between orders):
//
//   T >= fe_boys_asym_T[M] : F_0 = sqrt(pi/T)/2 and F_(m+1) = (2m+1)/(2T) F_m.
//                            The neglected terms are below 1e-16 relative for
//                            all orders <= M (thresholds computed in 40-digit
//                            arithmetic by gen_classes.py).
//   20 <= T < threshold    : F_0 = sqrt(pi/T)/2 - e^-T/(2T) S(1/T) with S the
//                            asymptotic series of erfc (Abramowitz & Stegun
//                            7.1.23), S(u) = sum_k (-1)^k (2k-1)!! (u/2)^k,
//                            12 terms (truncation below 1e-17 of F_0 at T = 20),
//                            then the upward recursion
//                            F_(m+1) = ((2m+1) F_m - e^-T)/(2T), which loses at
//                            most a few percent of an ulp per step at T >= 20.
//   T < 20                 : F_M from an 8-term Taylor expansion about the
//                            nearest point of a 1/16 grid (truncation below
//                            3e-17 relative), then the stable downward recursion
//                            F_(m-1) = (2T F_m + e^-T)/(2m-1).
//
// rsqrt is CUDA's own; e^-T comes from a table of e^(-i/16) and a short Taylor
// polynomial (fe_exp_neg); the grid values F_n(i/16) and e^(-i/16) are 40-digit
// reference values generated into classes_gen.cuh.
#pragma once
#include "common.cuh"
#include "classes_gen.cuh"

#define FE_SQRT_PI_2 0.88622692545275801365   // sqrt(pi)/2

// S(u) = sum_(k=0..11) (-1)^k (2k-1)!! (u/2)^k, Horner form.
FE_DEV double fe_erfc_asym_series(double u) {
  const double v = 0.5 * u;
  double s = -13749310575.0;                       // -(21)!!
#pragma unroll
  for (int k = 10; k >= 0; --k) {
    double c = 1.0;                                // (2k-1)!! with the sign (-1)^k
    for (int q = 2 * k - 1; q > 1; q -= 2) c *= double(q);
    s = fma(s, v, (k & 1) ? -c : c);
  }
  return s;
}

// e^-T for 0 <= T < 64 from a table of e^(-i h) on the Boys grid (h = 1/16,
// 40-digit values) times the 8-term Taylor polynomial of e^d, d = i h - T,
// |d| <= 1/32 (truncation below 3e-17 relative): the table-driven method of
// P. T. P. Tang (ACM TOMS 15, 1989) with a finer table and no reduction step.
// ``i`` is round(T / h), in range.
FE_DEV double fe_exp_neg(double T, int i) {
  const double d = double(i) * FE_BOYS_GRID_H - T;      // exact
  double e = 1.0 / 5040.0;
  e = fma(e, d, 1.0 / 720.0);
  e = fma(e, d, 1.0 / 120.0);
  e = fma(e, d, 1.0 / 24.0);
  e = fma(e, d, 1.0 / 6.0);
  e = fma(e, d, 0.5);
  e = fma(e, d, 1.0);
  e = fma(e, d, 1.0);
  return __ldg(fe_exp_grid + i) * e;
}

template <int M>
FE_DEV void fe_boys_f64(const double T, double (&F)[M + 1]) {
  constexpr double t_asym = fe_boys_asym_T[M];
  if (T >= t_asym) {
    const double r = rsqrt(T);
    const double h = 0.5 * r * r;               // 1/(2T)
    F[0] = FE_SQRT_PI_2 * r;
#pragma unroll
    for (int m = 0; m < M; ++m) F[m + 1] = F[m] * (double(2 * m + 1) * h);
  } else if (T >= FE_BOYS_GRID_TMAX) {
    const double r = rsqrt(T);
    const double h = 0.5 * r * r;
    // T < t_asym <= 64 here
    const double e = fe_exp_neg(T, min(__double2int_rn(T * FE_BOYS_GRID_INV_H), FE_EXP_NROW - 1));
    F[0] = fma(-h * e, fe_erfc_asym_series(h + h), FE_SQRT_PI_2 * r);
#pragma unroll
    for (int m = 0; m < M; ++m) F[m + 1] = fma(double(2 * m + 1), F[m], -e) * h;
  } else {
    // clamped: a NaN argument (a NaN point) converts to an arbitrary integer,
    // and a malformed table could give T < 0; both must still read in bounds
    const int i = min(max(__double2int_rn(T * FE_BOYS_GRID_INV_H), 0), FE_BOYS_NROW - 1);
    const double d = -(T - double(i) * FE_BOYS_GRID_H);   // exact: |d| <= h/2
    const double* row = fe_boys_grid + i * FE_BOYS_NTAB + M;
    double f = __ldg(row + FE_BOYS_TAYLOR_K - 1);
#pragma unroll
    for (int k = FE_BOYS_TAYLOR_K - 2; k >= 0; --k)
      f = fma(f, d * (1.0 / double(k + 1)), __ldg(row + k));
    F[M] = f;
    const double e = fe_exp_neg(T, i);
    const double t2 = T + T;
#pragma unroll
    for (int m = M; m > 0; --m) F[m - 1] = fma(t2, F[m], e) * (1.0 / double(2 * m - 1));
  }
}

// FP32 Boys vectors for the mixed-precision evaluator, in the scaled form
// F^_m(T) = F_m(T) / s_m, s_m = (sqrt(pi)/2) (2m-1)!!/2^m (the FP32 records
// carry s_m folded into their coefficients, in FP64).  In that form
//  * the asymptotic branch is F^_m = T^-(m+1/2): F^_0 = rt, F^_(m+1) = F^_m / T;
//  * the downward recursion is F^_(m-1) = T F^_m + E_m with E_m = e^-T / (2 s_m),
//    E_(m-1) = E_m (2m-1)/2; the upward one F^_(m+1) = (F^_m - E_(m+1)) / T;
// every constant in them is exact in FP32 (E_M takes 1/(2 s_M) as a float
// hi/lo pair), so no rounded constant biases all pairs alike.
// Asymptotic above fe_boys32_asym_T[M] (2e-8 relative); below it a 6-term
// Taylor expansion about the nearest point of a 1/4 grid over 0 <= T < 32 held
// in shared memory (``grid``, truncation below 6e-9 relative), then the
// downward recursion.  The FP32 thresholds of orders <= 6 lie below 32, so the
// common classes have only these two branches; for higher orders the stretch
// from 32 to the threshold uses the upward recursion from erf.  ``rt`` is
// T^-1/2, which the caller already has.  This scalar form reads the unscaled
// rows fe_boys_grid32 and scales F_M by 1/s_M (a float hi/lo pair).
template <int M>
FE_DEV void fe_boys_f32(const float T, const float rt, const float* __restrict__ grid,
                        float (&F)[M + 1]) {
  constexpr float t_asym = fe_boys32_asym_T[M];
  constexpr float kh = fe_boys32_kappa_hi[M], kl = fe_boys32_kappa_lo[M];
  constexpr float sh = fe_boys32_sinv_hi[M], sl = fe_boys32_sinv_lo[M];
  if (T >= t_asym) {
    const float it = rt * rt;
    F[0] = rt;
#pragma unroll
    for (int m = 0; m < M; ++m) F[m + 1] = F[m] * it;
  } else if (t_asym > FE_BOYS32_GRID_TMAX && T >= FE_BOYS32_GRID_TMAX) {
    const float it = rt * rt;
    const float e = __expf(-T);
    float E[M + 1];
    E[M] = fmaf(e, kh, e * kl);
#pragma unroll
    for (int m = M; m > 1; --m) E[m - 1] = E[m] * (float(2 * m - 1) * 0.5f);
    F[0] = rt * erff(T * rt);
#pragma unroll
    for (int m = 0; m < M; ++m) F[m + 1] = (F[m] - E[m + 1]) * it;
  } else {
    const int i = min(max(__float2int_rn(T * FE_BOYS32_GRID_INV_H), 0), FE_BOYS32_NROW - 1);
    const float d = -(T - float(i) * FE_BOYS32_GRID_H);
    const float* row = grid + i * FE_BOYS32_NTAB + M;
    float f = row[FE_BOYS32_TAYLOR_K - 1];
#pragma unroll
    for (int k = FE_BOYS32_TAYLOR_K - 2; k >= 0; --k) f = fmaf(f, d * (1.0f / float(k + 1)), row[k]);
    F[M] = fmaf(f, sh, f * sl);
    const float e = __expf(-T);
    float E = fmaf(e, kh, e * kl);
#pragma unroll
    for (int m = M; m > 0; --m) {
      F[m - 1] = fmaf(T, F[m], E);
      E = E * (float(2 * m - 1) * 0.5f);
    }
  }
}

// Packed FP32 Boys vectors of two arguments (one per float2 lane), for the
// orders whose FP32 asymptotic threshold lies below the grid's end (M <= 6):
// the tabulated and the asymptotic branch only, in the form the FP32 records'
// coefficients c_k = K G_k s_m p^-(m+1/2) take: F~_m = F_m(T) p^(m+1/2) / s_m,
// which in the asymptotic range is exactly 1/|R|^(2m+1) (T = p |R|^2), so an
// asymptotic lane needs only ``ir`` = 1/|R|.  A tabulated lane evaluates
// F^_M = F_M / s_M from the per-order scaled rows fe_boys_grid32s
// (F_(M+k)/(k! s_M), Taylor polynomial in d directly) in ``grid``, the
// downward recursion of fe_boys_f32, then multiplies order m by
// sqrt(p) p^m (``sp``, ``p``).  When the lanes fall in different branches both
// are computed and each lane keeps its own.
template <int M>
FE_DEV void fe_boys_f32x2(const float2 T, const float2 ir, const float2 sp, const float2 p,
                          const float* __restrict__ grid, float2 (&F)[M + 1]) {
  constexpr float t_asym = fe_boys32_asym_T[M];
  constexpr float kh = fe_boys32_kappa_hi[M], kl = fe_boys32_kappa_lo[M];
  static_assert(fe_boys32_asym_T[M] <= FE_BOYS32_GRID_TMAX, "two-branch form only");
  const bool ax = T.x >= t_asym, ay = T.y >= t_asym;
  float2 A[M + 1], G[M + 1];
  if (ax || ay) {
    const float2 ir2 = ir * ir;
    A[0] = ir;
#pragma unroll
    for (int m = 0; m < M; ++m) A[m + 1] = A[m] * ir2;
  }
  if (!(ax && ay)) {
    // a lane in the asymptotic range reads a clamped, in-range row; its result is dropped
    const float2 ti = T * fe_f2(FE_BOYS32_GRID_INV_H);
    const int ix = min(max(__float2int_rn(ti.x), 0), FE_BOYS32_NROW - 1);
    const int iy = min(max(__float2int_rn(ti.y), 0), FE_BOYS32_NROW - 1);
    const float2 d = make_float2(float(ix), float(iy)) * fe_f2(FE_BOYS32_GRID_H) - T;   // exact
    const float* rx = grid + (M * FE_BOYS32_NROW + ix) * FE_BOYS32_TAYLOR_K;
    const float* ry = grid + (M * FE_BOYS32_NROW + iy) * FE_BOYS32_TAYLOR_K;
    float2 f = make_float2(rx[FE_BOYS32_TAYLOR_K - 1], ry[FE_BOYS32_TAYLOR_K - 1]);
#pragma unroll
    for (int k = FE_BOYS32_TAYLOR_K - 2; k >= 0; --k) f = fe_fma(f, d, make_float2(rx[k], ry[k]));
    G[M] = f;
    const float2 e = make_float2(__expf(-T.x), __expf(-T.y));
    float2 E = fe_fma(e, fe_f2(kh), e * fe_f2(kl));
#pragma unroll
    for (int m = M; m > 0; --m) {
      G[m - 1] = fe_fma(T, G[m], E);
      if (m > 1) E = E * fe_f2(float(2 * m - 1) * 0.5f);
    }
    float2 w = sp;
    G[0] = G[0] * w;
#pragma unroll
    for (int m = 1; m <= M; ++m) {
      w = w * p;
      G[m] = G[m] * w;
    }
  }
  if (ax && ay) {
#pragma unroll
    for (int m = 0; m <= M; ++m) F[m] = A[m];
  } else if (!ax && !ay) {
#pragma unroll
    for (int m = 0; m <= M; ++m) F[m] = G[m];
  } else {
#pragma unroll
    for (int m = 0; m <= M; ++m) F[m] = make_float2(ax ? A[m].x : G[m].x, ay ? A[m].y : G[m].y);
  }
}
