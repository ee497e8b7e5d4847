// Mixed-precision ESP evaluation (same result as eval_f64 to <= 1e-6 a.u.).
//
// FP32 for the per-pair Boys vector, the monomial/Horner polynomial and the
// products; FP64 where FP32 would not hold the error budget:
//
//  * routing: the FP32 rounding error of a pair's contribution scales with
//    K sum_k |G_k R^a F_m(p R^2)|, which is at most sum_n b_n / |R|^(n+1)
//    (F_m(T) <= Gamma(m + 1/2) / (2 T^(m + 1/2)), and |R^a| <= |R|^|a| times
//    the maximum of |u^a| on the unit sphere; n = 2m - |a|, the b_n computed by
//    the table build in FP64 and stored rounded up).  When that bound reaches
//    ``tau`` for any point of a warp's point set, the (pair, warp) is
//    evaluated in FP64 instead.  fe_eval_f32_kernel takes the
//    decision, evaluates every (pair, warp) left in FP32 and records the others
//    as one bit per (pair, warp) in a routing mask in the workspace;
//    fe_eval_fix64_kernel evaluates exactly those in FP64 from the pairs' FP64
//    records.  Neither kernel carries the other's code, so each keeps its
//    registers.
//  * the classes up to 6 run two points per packed FP32x2 lane (sm_100
//    __ffma2_rn / __fadd2_rn / __fmul2_rn), with the coefficients stored twice
//    in the FP32 records so that a 16-byte load gives two packed operands; the
//    g-shell classes run scalar.
//  * R = C - P from float hi/lo splits of both coordinates, so R carries about
//    one float ulp of R itself rather than of |C|.
//  * accumulation: every pair's FP32 contribution K s, rounded once, is added
//    to an FP64 sum per point (the FP64 pipe is otherwise idle in the FP32
//    kernel, so two conversions and two DADDs per point pair cost less than a
//    compensated FP32 two-sum); FP64 contributions into an FP64 sum; the splits,
//    the nuclear term and the final nuclear - electron subtraction are FP64.
//
// Grid and pipeline of the FP32 kernel as eval_f64 (class-major grid rows,
// points in registers, record tiles streamed to shared memory by 1-D TMA bulk
// copies over an mbarrier ring).  Both kernels use the same point blocks
// (FE_MX_NT threads x FE_MX_NP points), so warp g covers the same points in
// both; its mask row is words [g * wtotal, (g+1) * wtotal), class L from
// woff[L].  The FP32 kernel's pair parts sit on multiples of 32 pairs, so every
// mask word has exactly one writer and the mask needs no clearing.
#pragma once
#include "eval_f64.cuh"

#ifndef FE_MX_NP
#define FE_MX_NP 4            // points per thread of both mixed kernels
#endif
#define FE_MX_NT 128          // threads per block of both mixed kernels

struct FeMixedArgs {
  const unsigned char* table;
  const double* pts;
  int npts;
  int nsplit;
  double* partial;               // [nsplit][ld] partial electron sums of this kernel
  int ld;
  float tau;                     // FP64 routing threshold (a.u.)
  unsigned long long* n64;       // optional: count of (pair, warp) FP64 evaluations
  unsigned* mask;                // routing mask (one bit per pair and warp)
  long long mask_words;          // its capacity in 32-bit words
  int lmin, lmax;                // classes evaluated (a sub-range for per-class timing)
};

__constant__ int fe_c_tile32[FE_NCLASS] = {
  FE_STAGE_BYTES / (4 * fe_class_rec32[0]), FE_STAGE_BYTES / (4 * fe_class_rec32[1]),
  FE_STAGE_BYTES / (4 * fe_class_rec32[2]), FE_STAGE_BYTES / (4 * fe_class_rec32[3]),
  FE_STAGE_BYTES / (4 * fe_class_rec32[4]), FE_STAGE_BYTES / (4 * fe_class_rec32[5]),
  FE_STAGE_BYTES / (4 * fe_class_rec32[6]), FE_STAGE_BYTES / (4 * fe_class_rec32[7]),
  FE_STAGE_BYTES / (4 * fe_class_rec32[8])};

// The routing test of one class-L pair for this thread's points: the pair is
// routed for the warp when the bound sum_n b_n / |R|^(n+1) (record floats
// after the coefficients) reaches tau for any of the warp's points.  Written
// !(bound < tau) so that a NaN or overflowing bound (a point on the pair's
// centre) routes.
template <int L, int NP>
FE_DEV bool fe_route(const float* __restrict__ rec, const float (&cxh)[NP], const float (&cyh)[NP],
                     const float (&czh)[NP], const float (&cxl)[NP], const float (&cyl)[NP],
                     const float (&czl)[NP], float (&x)[NP], float (&y)[NP], float (&z)[NP],
                     float (&r2)[NP], float (&ir)[NP], float tau) {
  const float* bn = rec + 12 + 2 * fe_class_nterm[L];
  bool need = false;
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    x[j] = __fadd_rn(__fsub_rn(cxh[j], rec[2]), __fsub_rn(cxl[j], rec[5]));
    y[j] = __fadd_rn(__fsub_rn(cyh[j], rec[3]), __fsub_rn(cyl[j], rec[6]));
    z[j] = __fadd_rn(__fsub_rn(czh[j], rec[4]), __fsub_rn(czl[j], rec[7]));
    r2[j] = fmaf(x[j], x[j], fmaf(y[j], y[j], __fmul_rn(z[j], z[j])));
    ir[j] = rsqrtf(r2[j]);
    float bound = bn[L];
#pragma unroll
    for (int n = L - 1; n >= 0; --n) bound = fmaf(bound, ir[j], bn[n]);
    need |= !(__fmul_rn(bound, ir[j]) < tau);
  }
  return __any_sync(0xffffffffu, need);
}

template <int NP>
FE_DEV void fe_load_points_split(const double* __restrict__ pts, int npts, int p0, int stride,
                                 float (&cxh)[NP], float (&cyh)[NP], float (&czh)[NP],
                                 float (&cxl)[NP], float (&cyl)[NP], float (&czl)[NP]) {
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const int q = min(p0 + j * stride, npts - 1);
    const double c0 = pts[3 * q], c1 = pts[3 * q + 1], c2 = pts[3 * q + 2];
    cxh[j] = float(c0); cxl[j] = float(c0 - double(cxh[j]));
    cyh[j] = float(c1); cyl[j] = float(c1 - double(cyh[j]));
    czh[j] = float(c2); czl[j] = float(c2 - double(czh[j]));
  }
}

// FP32 evaluation of a tile, recording the (pair, warp) routed to FP64 in the
// mask instead.  ``first`` is the class-local index of the tile's first pair,
// ``hi`` the end of this split's range of the class; ``bits`` carries the
// current mask word across tiles (identical in every lane, lane 0 stores it).
// The record's coefficients carry K and p^-(m+1/2) (table.cuh), so the scaled
// Boys vector F^_m of fe_boys_f32 is multiplied by sqrt(p) p^m.
template <int L, int NP>
FE_DEV void fe_tile_f32(const float* __restrict__ rec, int first, int n, int hi,
                        const float (&cxh)[NP], const float (&cyh)[NP], const float (&czh)[NP],
                        const float (&cxl)[NP], const float (&cyl)[NP], const float (&czl)[NP],
                        double (&acc)[NP], const float* __restrict__ grid, float tau,
                        unsigned* __restrict__ mw, unsigned& bits) {
  constexpr int S32 = fe_class_rec32[L];
  const bool lane0 = (threadIdx.x & 31) == 0;
#pragma unroll 1
  for (int i = 0; i < n; ++i, rec += S32) {
    const int gi = first + i;
    float x[NP], y[NP], z[NP], r2[NP], ir[NP];
    const bool routed = fe_route<L, NP>(rec, cxh, cyh, czh, cxl, cyl, czl, x, y, z, r2, ir, tau);
    bits |= unsigned(routed) << (gi & 31);
    if ((gi & 31) == 31 || gi + 1 == hi) {
      if (lane0 && mw) mw[gi >> 5] = bits;
      bits = 0u;
    }
    if (routed) continue;
    const float pe = rec[0], sp = rec[1], rsp = rec[9];
    float F[NP][L + 1], s[NP];
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      fe_boys_f32<L>(pe * r2[j], ir[j] * rsp, grid, F[j]);
      float w = sp;
      F[j][0] *= w;
#pragma unroll
      for (int m = 1; m <= L; ++m) {
        w *= pe;
        F[j][m] *= w;
      }
    }
    fe_poly<L, float, NP>(rec + 12, x, y, z, F, s);
#pragma unroll
    for (int j = 0; j < NP; ++j) acc[j] += double(s[j]);
  }
}

// The routing test of fe_route for two points per float2 lane, from |R|^2:
// also returns ir = 1/|R|.
template <int L, int NQ>
FE_DEV bool fe_route2(const float* __restrict__ rec, const float2 (&r2)[NQ], float2 (&ir)[NQ],
                      float tau) {
  const float* bn = rec + 12 + 2 * fe_class_nterm[L];
  bool need = false;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    ir[q] = make_float2(rsqrtf(r2[q].x), rsqrtf(r2[q].y));
    float2 bound = fe_f2(bn[L]);
#pragma unroll
    for (int n = L - 1; n >= 0; --n) bound = fe_fma(bound, ir[q], fe_f2(bn[n]));
    bound = bound * ir[q];
    need |= !(bound.x < tau) || !(bound.y < tau);
  }
  return __any_sync(0xffffffffu, need);
}

// The same with two points per float2 lane (packed FP32x2 instructions; point
// 2q + e of the thread in lane e of q).  Per pair, R and |R|^2 first; then
//  * far pairs -- every point of the warp at least the record's rfar from the
//    centre (only when ``fast``: the routing threshold is at least the one rfar
//    was computed for): no point routes and every Boys vector is asymptotic,
//    F~_m = 1/|R|^(2m+1), so s = (1/|R|) sum_m (1/|R|^2)^m h_m (fe_poly32x2a);
//  * the others: the exact per-point routing test of fe_route, then the Boys
//    vectors of fe_boys_f32x2 and the polynomial.
// The far test is a sufficient condition for the others' outcome (no route,
// asymptotic branch), so both give the same decisions; it only skips work.
template <int L, int NQ>
FE_DEV void fe_tile_f32x2(const float* __restrict__ rec, int first, int n, int hi,
                          const float2 (&cxh)[NQ], const float2 (&cyh)[NQ],
                          const float2 (&czh)[NQ], const float2 (&cxl)[NQ],
                          const float2 (&cyl)[NQ], const float2 (&czl)[NQ],
                          double (&acc)[2 * NQ], const float* __restrict__ grid, float tau,
                          bool fast, unsigned* __restrict__ mw, unsigned& bits) {
  constexpr int S32 = fe_class_rec32[L];
  const bool lane0 = (threadIdx.x & 31) == 0;
  // pairs in runs that end on a routing-mask word boundary (or the split's
  // end), so the word is stored once per run, not tested per pair
  for (int i = 0; i < n;) {
    const int gi0 = first + i;
    const int run = min(n - i, 32 - (gi0 & 31));
#pragma unroll 1
    for (int r = 0; r < run; ++r, rec += S32) {
      const float4 h0 = *reinterpret_cast<const float4*>(rec);
      const float4 h1 = *reinterpret_cast<const float4*>(rec + 4);
      const float rf2 = rec[8];
      const float2 pxh = fe_f2(h0.z), pyh = fe_f2(h0.w), pzh = fe_f2(h1.x);
      const float2 pxl = fe_f2(h1.y), pyl = fe_f2(h1.z), pzl = fe_f2(h1.w);
      float2 x[NQ], y[NQ], z[NQ], r2[NQ];
      bool far = fast;
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        x[q] = (cxh[q] - pxh) + (cxl[q] - pxl);
        y[q] = (cyh[q] - pyh) + (cyl[q] - pyl);
        z[q] = (czh[q] - pzh) + (czl[q] - pzl);
        r2[q] = fe_fma(x[q], x[q], fe_fma(y[q], y[q], z[q] * z[q]));
        far = far && r2[q].x >= rf2 && r2[q].y >= rf2;
      }
      if (__all_sync(0xffffffffu, far)) {
        float2 ir[NQ], ir2[NQ], s[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
          ir[q] = make_float2(rsqrtf(r2[q].x), rsqrtf(r2[q].y));
          ir2[q] = ir[q] * ir[q];
        }
        fe_poly32x2a<L, NQ>(rec + 12, x, y, z, ir2, s);
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
          const float2 v = s[q] * ir[q];
          acc[2 * q] += double(v.x);
          acc[2 * q + 1] += double(v.y);
        }
      } else {
        float2 ir[NQ];
        if (fe_route2<L, NQ>(rec, r2, ir, tau)) {
          bits |= 1u << ((gi0 + r) & 31);
        } else {
          const float2 pe = fe_f2(h0.x), sp = fe_f2(h0.y);
          float2 F[NQ][L + 1], s[NQ];
#pragma unroll
          for (int q = 0; q < NQ; ++q) fe_boys_f32x2<L>(pe * r2[q], ir[q], sp, pe, grid, F[q]);
          fe_poly32x2<L, NQ>(rec + 12, x, y, z, F, s);
#pragma unroll
          for (int q = 0; q < NQ; ++q) {
            acc[2 * q] += double(s[q].x);
            acc[2 * q + 1] += double(s[q].y);
          }
        }
      }
    }
    i += run;
    const int gl = first + i - 1;                  // last pair of the run
    if ((gl & 31) == 31 || gl + 1 == hi) {
      if (lane0 && mw) mw[gl >> 5] = bits;
      bits = 0u;
    }
  }
}

// FP64 evaluation of one routed pair (its FP64 record ``rec64``) for
// this thread's points, two at a time for instruction-level parallelism.
template <int L, int NP>
FE_DEV void fe_pair_fix64(const double* __restrict__ rec64, const double (&cx)[NP],
                          const double (&cy)[NP], const double (&cz)[NP], double (&a64)[NP]) {
  static_assert(NP % 2 == 0, "points are evaluated in pairs");
  const double pe = rec64[0], px = rec64[1], py = rec64[2], pz = rec64[3], K = rec64[4];
#pragma unroll 1
  for (int h = 0; h < NP; h += 2) {
    double xx[2], yy[2], zz[2], F[2][L + 1], s[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      xx[j] = cx[h + j] - px;
      yy[j] = cy[h + j] - py;
      zz[j] = cz[h + j] - pz;
      fe_boys_f64<L>(pe * fma(xx[j], xx[j], fma(yy[j], yy[j], zz[j] * zz[j])), F[j]);
    }
    fe_poly<L, double, 2>(rec64 + 6, xx, yy, zz, F, s);
#pragma unroll
    for (int j = 0; j < 2; ++j) a64[h + j] = fma(K, s[j], a64[h + j]);
  }
}

// Dispatch on the tile's class among the compiled range [LLO, LHI] only.
#define FE_IN(l) ((l) >= LLO && (l) <= LHI ? (l) : LLO)
#define FE_MX_SWITCH(CALL)                                                        \
  if (L < LLO || L > LHI) fe_flag(FE_ST_BADCLASS);                                \
  if (0 >= LLO && 0 <= LHI && L == 0) CALL(FE_IN(0));                             \
  if (1 >= LLO && 1 <= LHI && L == 1) CALL(FE_IN(1));                             \
  if (2 >= LLO && 2 <= LHI && L == 2) CALL(FE_IN(2));                             \
  if (3 >= LLO && 3 <= LHI && L == 3) CALL(FE_IN(3));                             \
  if (4 >= LLO && 4 <= LHI && L == 4) CALL(FE_IN(4));                             \
  if (5 >= LLO && 5 <= LHI && L == 5) CALL(FE_IN(5));                             \
  if (6 >= LLO && 6 <= LHI && L == 6) CALL(FE_IN(6));                             \
  if (7 >= LLO && 7 <= LHI && L == 7) CALL(FE_IN(7));                             \
  if (8 >= LLO && 8 <= LHI && L == 8) CALL(FE_IN(8));

template <int MINB, int LLO, int LHI>
__global__ void __launch_bounds__(FE_MX_NT, MINB) fe_eval_f32_kernel(const FeMixedArgs a) {
  constexpr int NP = FE_MX_NP, NT = FE_MX_NT;
  // classes up to 6 run packed (two points per float2 lane); the g-shell
  // classes, whose FP32 Boys vector also has the erf branch, run scalar
  constexpr bool PACKED = LHI <= 6 && NP % 2 == 0;
  constexpr int NQ = NP / 2;
  extern __shared__ __align__(128) unsigned char fe_smem[];
  __shared__ uint64_t full_bar[FE_NSTAGE];
  __shared__ FeBlockWork w;
  // packed classes: the per-order scaled rows of orders 0..LHI (the highest
  // order a class of the range asks for); g-shell classes: the plain rows
  constexpr int GRIDN = PACKED ? (LHI + 1) * FE_BOYS32_NROW * FE_BOYS32_TAYLOR_K
                               : FE_BOYS32_NROW * FE_BOYS32_NTAB;
  __shared__ float grid[GRIDN];
  const FeTableHdr* hdr = reinterpret_cast<const FeTableHdr*>(a.table);
  const int tid = threadIdx.x;
  for (int k = tid; k < GRIDN; k += NT) grid[k] = PACKED ? fe_boys_grid32s[k] : fe_boys_grid32[k];
  float cxh[NP], cyh[NP], czh[NP], cxl[NP], cyl[NP], czl[NP];
  double acc[NP];
  const int p0 = int(blockIdx.x) * (NT * NP) + tid;
  fe_load_points_split<NP>(a.pts, a.npts, p0, NT, cxh, cyh, czh, cxl, cyl, czl);
#pragma unroll
  for (int j = 0; j < NP; ++j) acc[j] = 0.0;
  float2 cxh2[NQ], cyh2[NQ], czh2[NQ], cxl2[NQ], cyl2[NQ], czl2[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    cxh2[q] = make_float2(cxh[2 * q], cxh[2 * q + 1]);
    cyh2[q] = make_float2(cyh[2 * q], cyh[2 * q + 1]);
    czh2[q] = make_float2(czh[2 * q], czh[2 * q + 1]);
    cxl2[q] = make_float2(cxl[2 * q], cxl[2 * q + 1]);
    cyl2[q] = make_float2(cyl[2 * q], cyl[2 * q + 1]);
    czl2[q] = make_float2(czl[2 * q], czl[2 * q + 1]);
  }
  FeTilePipe pipe{a.table, fe_c_tile32, fe_c_rec32, hdr->off32, 4, fe_smem, full_bar, &w};
  int Lrow, part, nparts;
  fe_class_rows(hdr, max(LLO, a.lmin), min(LHI, a.lmax), a.nsplit, blockIdx.y, Lrow, part, nparts);
  if (Lrow >= 0) pipe.start(hdr, part, nparts, Lrow, Lrow, 32);
  else pipe.start(hdr, 0, 1, 1, 0, 32);                 // idle row: no tiles
  const int total = w.total;
  const long long warp_g = (long long)blockIdx.x * (NT / 32) + (tid >> 5);
  unsigned* mrow = a.mask + warp_g * w.wtotal;
  if ((warp_g + 1) * w.wtotal > a.mask_words) {
    mrow = nullptr;
    fe_flag(FE_ST_OVERFLOW);
  }
  unsigned bits = 0u;
  // the records' far radius holds for routing thresholds at least tau_fast
  const bool fast = a.tau >= hdr->tau_fast;
  for (int i = 0; i < total; ++i) {
    if (!pipe.wait(i)) {
      pipe.abort(i);
      fe_poison_row<NP>(a.partial + size_t(blockIdx.y) * a.ld, p0, NT, a.npts);
      return;
    }
    int L, first, n;
    fe_item(w, fe_c_tile32, i, L, first, n);
    const float* rec = reinterpret_cast<const float*>(pipe.stage(i));
    unsigned* mw = mrow ? mrow + w.woff[L] : nullptr;
    if constexpr (PACKED) {
#define FE_CALL32(l) fe_tile_f32x2<l, NQ>(rec, first, n, w.hi[L], cxh2, cyh2, czh2, cxl2, cyl2, \
                                          czl2, acc, grid, a.tau, fast, mw, bits)
      FE_MX_SWITCH(FE_CALL32)
#undef FE_CALL32
    } else {
#define FE_CALL32(l) fe_tile_f32<l, NP>(rec, first, n, w.hi[L], cxh, cyh, czh, cxl, cyl, czl, \
                                        acc, grid, a.tau, mw, bits)
      FE_MX_SWITCH(FE_CALL32)
#undef FE_CALL32
    }
    pipe.release(i);
  }
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const int p = p0 + j * NT;
    if (p < a.npts) a.partial[size_t(blockIdx.y) * a.ld + p] = acc[j];
  }
}

// The FP64 part: grid row y takes one class and a part of its mask words
// (fe_class_rows, class-major so that concurrently running blocks execute the
// same class's code).  Each warp walks its own mask row, 32 words at a time
// (one word per lane, the non-empty ones found by a ballot), and evaluates
// every pair whose bit is set for its points.  The pair's FP64 record comes
// into the warp's own shared-memory buffer by cp.async, the next routed pair's
// while the warp evaluates the current one (two buffers), so the coefficient
// reads are shared-memory broadcasts rather than L1 round trips on the
// critical path.  No block barrier: a warp with nothing
// routed finishes early.  Every warp accumulates its pairs in pair order and
// every grid row writes its own partial sums, so the result is deterministic.
template <int MINB, int LLO, int LHI>
__global__ void __launch_bounds__(FE_MX_NT, MINB) fe_eval_fix64_kernel(const FeMixedArgs a) {
  constexpr int NP = FE_MX_NP, NT = FE_MX_NT, NW = FE_MX_NT / 32;
  constexpr int RMAX = fe_class_rec64[LHI];          // largest record of the range
  __shared__ FeBlockWork w;
  __shared__ __align__(16) double fix_rec[NW][2][RMAX];
  const FeTableHdr* hdr = reinterpret_cast<const FeTableHdr*>(a.table);
  const int tid = threadIdx.x, lane = tid & 31, wi = tid >> 5;
  double cx[NP], cy[NP], cz[NP], a64[NP];
  const int p0 = int(blockIdx.x) * (NT * NP) + tid;
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const int q = min(p0 + j * NT, a.npts - 1);
    cx[j] = a.pts[3 * q];
    cy[j] = a.pts[3 * q + 1];
    cz[j] = a.pts[3 * q + 2];
    a64[j] = 0.0;
  }
  if (tid == 0) {
    const int one[FE_NCLASS] = {1, 1, 1, 1, 1, 1, 1, 1, 1};
    fe_block_work(hdr, 0, 1, one, 0, FE_NCLASS - 1, w);    // word offsets only
  }
  __syncthreads();
  const long long warp0 = (long long)blockIdx.x * NW;
  unsigned n64 = 0;
  int L, part, nparts;
  fe_class_rows(hdr, max(LLO, a.lmin), min(LHI, a.lmax), a.nsplit, blockIdx.y, L, part, nparts);
  if ((warp0 + NW) * w.wtotal > a.mask_words) {
    if (tid == 0) fe_flag(FE_ST_OVERFLOW);
    L = -1;
  }
  if (L >= 0) {
    const int nw = (hdr->count[L] + 31) / 32;
    const int w0 = int((long long)nw * part / nparts);
    const int w1 = int((long long)nw * (part + 1) / nparts);
    const int S64 = fe_c_rec64[L];
    const double* base = reinterpret_cast<const double*>(a.table + hdr->off64[L]);
    const unsigned* mrow = a.mask + (warp0 + wi) * w.wtotal + w.woff[L];
    // the warp's routed pairs in order: mask words 32 at a time (one per
    // lane), then the set bits of each non-zero word (warp-uniform state)
    int c0 = w0 - 32;
    unsigned wv = 0u, nz = 0u, mine = 0u;
    long long pair0 = 0;
    auto next = [&]() -> long long {
      for (;;) {
        if (mine) {
          const int bit = __ffs(mine) - 1;
          mine &= mine - 1;
          return pair0 + bit;
        }
        if (nz) {
          const int k = __ffs(nz) - 1;
          nz &= nz - 1;
          mine = __shfl_sync(0xffffffffu, wv, k);
          pair0 = (long long)(c0 + k) * 32;
          continue;
        }
        c0 += 32;
        if (c0 >= w1) return -1;
        wv = c0 + lane < w1 ? mrow[c0 + lane] : 0u;
        nz = __ballot_sync(0xffffffffu, wv != 0u);
      }
    };
    // each routed pair's FP64 record is copied to this warp's shared buffer
    // (16-byte cp.async by the lanes) while the warp evaluates the previous one
    auto fetch = [&](long long pr, int b) {
      const double* src = base + pr * S64;
      double* dst = fix_rec[wi][b];
      for (int c = lane; c < S64 / 2; c += 32)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst + 2 * c)),
                     "l"(src + 2 * c) : "memory");
      asm volatile("cp.async.commit_group;" ::: "memory");
    };
    long long cur = next();
    int b = 0;
    if (cur >= 0) fetch(cur, 0);
    while (cur >= 0) {                                // warp-uniform
      const long long nxt = next();
      if (nxt >= 0) {
        fetch(nxt, b ^ 1);
        asm volatile("cp.async.wait_group 1;" ::: "memory");
      } else {
        asm volatile("cp.async.wait_group 0;" ::: "memory");
      }
      __syncwarp();
      ++n64;
      const double* rec = fix_rec[wi][b];
#define FE_CALLP(l) fe_pair_fix64<l, NP>(rec, cx, cy, cz, a64)
      FE_MX_SWITCH(FE_CALLP)
#undef FE_CALLP
      __syncwarp();                                   // before the buffer is refilled
      cur = nxt;
      b ^= 1;
    }
  }
  if (a.n64 && lane == 0) atomicAdd(a.n64, (unsigned long long)n64);
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const int p = p0 + j * NT;
    if (p < a.npts) a.partial[size_t(blockIdx.y) * a.ld + p] = a64[j];
  }
}
