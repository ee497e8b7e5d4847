// Pair-table build: replaces build_pairs (fastesp/native/build_pairs.cpp:162-425)
// and build_table / ESPEngine (fastesp/table.py:176-259, fastesp/esp.py:168-257).
//
// One thread per primitive pair.  Work items are grouped by the shell pair's
// (la, lb), one launch per group (fe_build_kernel<la, lb>, the groups side by
// side on forked streams); a pair that survives the screen is written to a
// fixed slot of its class's staging array (slots are numbered in the
// reference's pair order), with a keep flag.  A thread spends at most
// FE_SCREEN_BUDGET box/point tests on the screen; the pairs it leaves
// undecided are finished by one warp each (fe_screen_pending_kernel).
// A scan of the flags, then one fe_records_kernel<L> per class, compact every
// class in order into the table and derive its mixed-precision records.
//
// Per primitive pair (a = exponent of shell si, b = of sj):
//   p = a + b, P = (aA + bB)/p, K = exp(-ab/p |A-B|^2)       (esp.py:226-230)
//   E^x_t, E^y_t, E^z_t Hermite coefficients                 (esp.py:108-147)
//   etab[t] = sum_mu,nu w_mu,nu Ex Ey Ez, w = (D_ij + D_ji) c_a c_b  (esp.py:239-247)
//   G_k = (2 pi/p)(2p)^m_k sum_t M0[k,t] etab[t]              (esp.py:248-250),
//         stored at record position fe_gpos_L[k] (the order the kernels read them)
//   bound = (2p)^-1.5 sum_t |etab_t| M_tx M_ty M_tz (2p)^(|t|/2), reff = 1.6 sqrt((L+2)/p)
//   screen: rule 0 keeps unless K bound / max(dmin, 0.05) < tol   (table.py:190-194);
//           dmin is the exact nearest-point distance, found by a pruned search
//           over point-block bounding boxes
//           rule 1 drops if K bound / max(dmin - reff, 0.05) < tol,
//                  and drops pairs with c_a c_b == 0 or all G == 0 (build_pairs.cpp:243,309,326-328)
#pragma once
#include "common.cuh"
#include "classes_gen.cuh"
#include "table.cuh"

struct FeShell {
  int atom, l, fn0, prim0, nprim, pad_;
  double c[3];
};

struct FeTask {          // one shell pair (si <= sj) with a non-empty class slot range
  int si, sj;
  int slot0;             // class slot of primitive pair (0, 0)
  int pad_;
};

struct FeBuildArgs {
  const FeShell* shells;
  const double* sexp;            // per-shell primitive exponents (shell.prim0 + i)
  const double* scoef;           // per-shell contraction coefficients
  const FeTask* tasks;
  const int* work_task;          // work item -> task
  const int* work_ij;            // work item -> (i << 16) | j
  int n_func;
  const double* dens;            // (n_func, n_func) Cartesian density
  const double* pts;             // (npts, 3)
  const float4* ptsf;            // the same points rounded to float (x, y, z, 0)
  const double* pbox;            // their bounding box: lo xyz, hi xyz
  int npts;
  const double* box;             // per 32-point block: lo xyz, hi xyz (6 doubles)
  const double* sbox;            // per 32-block superblock: the same
  int nbox, nsbox;
  double tol;
  int rule;
  const long long* class_slot0;  // first global slot of class L in the staging arrays
  double* stage;                 // staging records, class L at stage_off[L] doubles
  const long long* stage_off;
  int* keep;                     // per global slot: 0 dropped, 1 kept
  double* srule;                 // per global slot: K (pi/p)^1.5 etab[0]
  int* swork;                    // per global slot: its work item
  int* pending;                  // slots whose screen ran past the thread's budget
  int* npending;                 // their count (capacity: the slot count)
};

// Box or point tests a thread spends on a pair's screen before it hands the
// pair to the warp-parallel screen (fe_screen_warp).  Most pairs are decided
// within it; the few that need the exact nearest distance over many points
// would otherwise hold their whole warp (one thread per pair).  32 (about the
// superbox sweep of 30000 points) measured faster than 64, 128 or 256.
#ifndef FE_SCREEN_BUDGET
#define FE_SCREEN_BUDGET 32
#endif

#define FE_SCAN_BLOCK 1024     // slots per block of the keep-flag scan

__constant__ signed char fe_cart[5][15][3] = {
  {{0, 0, 0}},
  {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}},
  {{2, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 2, 0}, {0, 1, 1}, {0, 0, 2}},
  {{3, 0, 0}, {2, 1, 0}, {2, 0, 1}, {1, 2, 0}, {1, 1, 1}, {1, 0, 2}, {0, 3, 0}, {0, 2, 1},
   {0, 1, 2}, {0, 0, 3}},
  {{4, 0, 0}, {3, 1, 0}, {3, 0, 1}, {2, 2, 0}, {2, 1, 1}, {2, 0, 2}, {1, 3, 0}, {1, 2, 1},
   {1, 1, 2}, {1, 0, 3}, {0, 4, 0}, {0, 3, 1}, {0, 2, 2}, {0, 1, 3}, {0, 0, 4}}};

// The exponent along axis k of Cartesian function idx of angular momentum l, in
// the order of fe_cart (lx descending, then ly): a pure function, so inside
// fully unrolled loops it folds to a constant.
FE_DEV constexpr int fe_cart_exp(int l, int idx, int k) {
  int i = 0;
  for (int lx = l; lx >= 0; --lx)
    for (int ly = l - lx; ly >= 0; --ly) {
      if (i == idx) return k == 0 ? lx : (k == 1 ? ly : l - lx - ly);
      ++i;
    }
  return 0;
}

__constant__ double fe_screen_mom[12] = {
  2.5066282746310002, 2.0, 1.5957691216057308, 4.0, 10.212920779565312, 33.63284766793385,
  136.5963625280984, 665.1416330443616, 3768.863619586618, 25506.330595911374,
  202331.81842358326, 1872154.2572862155};

template <int L>
FE_DEV int fe_tri(int tx, int ty, int tz) {
  // compact index of (tx, ty, tz), |t| <= L, x-major then y then z
  int base = 0;
  for (int a = 0; a < tx; ++a) base += (L + 1 - a) * (L + 2 - a) / 2;
  for (int b = 0; b < ty; ++b) base += L + 1 - tx - b;
  return base + tz;
}

template <int L>
FE_DEV const short* fe_m0_ptr() {
  if constexpr (L == 0) return fe_m0_ptr_L0; else if constexpr (L == 1) return fe_m0_ptr_L1;
  else if constexpr (L == 2) return fe_m0_ptr_L2; else if constexpr (L == 3) return fe_m0_ptr_L3;
  else if constexpr (L == 4) return fe_m0_ptr_L4; else if constexpr (L == 5) return fe_m0_ptr_L5;
  else if constexpr (L == 6) return fe_m0_ptr_L6; else if constexpr (L == 7) return fe_m0_ptr_L7;
  else return fe_m0_ptr_L8;
}
template <int L>
FE_DEV const short* fe_m0_col() {
  if constexpr (L == 0) return fe_m0_col_L0; else if constexpr (L == 1) return fe_m0_col_L1;
  else if constexpr (L == 2) return fe_m0_col_L2; else if constexpr (L == 3) return fe_m0_col_L3;
  else if constexpr (L == 4) return fe_m0_col_L4; else if constexpr (L == 5) return fe_m0_col_L5;
  else if constexpr (L == 6) return fe_m0_col_L6; else if constexpr (L == 7) return fe_m0_col_L7;
  else return fe_m0_col_L8;
}
template <int L>
FE_DEV const float* fe_m0_val() {
  if constexpr (L == 0) return fe_m0_val_L0; else if constexpr (L == 1) return fe_m0_val_L1;
  else if constexpr (L == 2) return fe_m0_val_L2; else if constexpr (L == 3) return fe_m0_val_L3;
  else if constexpr (L == 4) return fe_m0_val_L4; else if constexpr (L == 5) return fe_m0_val_L5;
  else if constexpr (L == 6) return fe_m0_val_L6; else if constexpr (L == 7) return fe_m0_val_L7;
  else return fe_m0_val_L8;
}
template <int L>
FE_DEV const short* fe_gpos() {
  if constexpr (L == 0) return fe_gpos_L0; else if constexpr (L == 1) return fe_gpos_L1;
  else if constexpr (L == 2) return fe_gpos_L2; else if constexpr (L == 3) return fe_gpos_L3;
  else if constexpr (L == 4) return fe_gpos_L4; else if constexpr (L == 5) return fe_gpos_L5;
  else if constexpr (L == 6) return fe_gpos_L6; else if constexpr (L == 7) return fe_gpos_L7;
  else return fe_gpos_L8;
}
template <int L>
FE_DEV const signed char* fe_m0_m() {
  if constexpr (L == 0) return fe_m0_m_L0; else if constexpr (L == 1) return fe_m0_m_L1;
  else if constexpr (L == 2) return fe_m0_m_L2; else if constexpr (L == 3) return fe_m0_m_L3;
  else if constexpr (L == 4) return fe_m0_m_L4; else if constexpr (L == 5) return fe_m0_m_L5;
  else if constexpr (L == 6) return fe_m0_m_L6; else if constexpr (L == 7) return fe_m0_m_L7;
  else return fe_m0_m_L8;
}

// Squared distance from P to the box [lo, hi] (0 inside); a lower bound of the
// squared distance to every point in it.
FE_DEV double fe_box_lb2(const double* __restrict__ b, const double (&P)[3]) {
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double g = fmax(fmax(b[k] - P[k], P[k] - b[3 + k]), 0.0);
    s += g * g;
  }
  return s;
}

// Squared distance from P to the farthest corner of the box [lo, hi]: an upper
// bound of the squared distance to every point in it.
FE_DEV double fe_box_ub2(const double* __restrict__ b, const double (&P)[3]) {
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double g = fmax(fabs(P[k] - b[k]), fabs(b[3 + k] - P[k]));
    s += g * g;
  }
  return s;
}

// Bounding boxes of consecutive 32-point blocks (level 0: points -> boxes) and
// of 32-box superblocks (level 1: boxes -> superboxes).  One warp per box: a
// lane per member, min/max by shuffles.
FE_DEV void fe_warp_box(double (&lo)[3], double (&hi)[3]) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      lo[k] = fmin(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
      hi[k] = fmax(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
    }
}

__global__ void fe_point_boxes_kernel(const double* __restrict__ pts, int npts, double* box,
                                      int nbox) {
  const int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (b >= nbox) return;                       // whole warps: nbox is per warp
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  const int q = 32 * b + lane;
  if (q < npts)
#pragma unroll
    for (int k = 0; k < 3; ++k) lo[k] = hi[k] = pts[3 * q + k];
  fe_warp_box(lo, hi);
  if (lane < 3) {
    box[6 * b + lane] = lo[lane];
    box[6 * b + 3 + lane] = hi[lane];
  }
}

__global__ void fe_super_boxes_kernel(const double* __restrict__ box, int nbox, double* sbox,
                                      int nsbox) {
  const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (s >= nsbox) return;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  const int b = 32 * s + lane;
  if (b < nbox)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      lo[k] = box[6 * b + k];
      hi[k] = box[6 * b + 3 + k];
    }
  fe_warp_box(lo, hi);
  if (lane < 3) {
    sbox[6 * s + lane] = lo[lane];
    sbox[6 * s + 3 + lane] = hi[lane];
  }
}

// The screen's points in a spatially coherent order.  The screen's decision
// depends on the point set only, not its order, but its 32-point boxes are
// only as tight as consecutive points are close: callers' point orders (a
// Fibonacci spiral per atom, a grid row) give boxes spanning a whole sphere.
// The points are bucketed by the Morton code of a 16 x 16 x 16 grid of cells
// over their bounding box (a counting sort; the order within a cell does not
// matter to the screen).
#define FE_SORT_CELLS 4096

// Partial bounding boxes of the points: block b writes [lo, hi] of its
// grid-stride share to bb[6 b..6 b + 5]; fe_points_count_kernel combines the
// FE_BBOX_BLOCKS partials.
#define FE_BBOX_BLOCKS 64
__global__ void __launch_bounds__(256) fe_points_bbox_kernel(const double* __restrict__ pts,
                                                             int npts, double* __restrict__ bb) {
  __shared__ double red[6][8];
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < npts; q += gridDim.x * blockDim.x)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      lo[k] = fmin(lo[k], pts[3 * q + k]);
      hi[k] = fmax(hi[k], pts[3 * q + k]);
    }
  fe_warp_box(lo, hi);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      red[k][w] = lo[k];
      red[3 + k][w] = hi[k];
    }
  __syncthreads();
  if (threadIdx.x < 3) {
    double l = 1e300, h = -1e300;
    for (int i = 0; i < 8; ++i) {
      l = fmin(l, red[threadIdx.x][i]);
      h = fmax(h, red[3 + threadIdx.x][i]);
    }
    bb[6 * blockIdx.x + threadIdx.x] = l;
    bb[6 * blockIdx.x + 3 + threadIdx.x] = h;
  }
}

// Morton code of the cell holding point q in a grid of 2^BITS cells per axis
// over the bounding box bb = [lo, hi].
template <int BITS>
FE_DEV int fe_morton_cell(const double* __restrict__ q, const double* __restrict__ bb) {
  constexpr int N = 1 << BITS;
  int code = 0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double ext = bb[3 + k] - bb[k];
    const double cs = ext > 0.0 ? ext * (1.0 / N) * (1.0 + 1e-9) : 1.0;
    // fmax/fmin first: a NaN coordinate goes to cell 0
    const int c = int(fmin(fmax((q[k] - bb[k]) / cs, 0.0), double(N - 1)));
#pragma unroll
    for (int b = 0; b < BITS; ++b) code |= ((c >> b) & 1) << (3 * b + k);
  }
  return code;
}

// cell[q] and the per-cell counts (2^(3 BITS) cells, counts zeroed by the caller);
// bbp[6 FE_BBOX_BLOCKS ..] receives the combined bounding box.
template <int BITS>
__global__ void fe_points_count_kernel(const double* __restrict__ pts, int npts,
                                       double* __restrict__ bbp, int* __restrict__ cell,
                                       int* __restrict__ count) {
  __shared__ double bb[6];
  if (threadIdx.x < 6) {
    double v = threadIdx.x < 3 ? 1e300 : -1e300;
    for (int i = 0; i < FE_BBOX_BLOCKS; ++i)
      v = threadIdx.x < 3 ? fmin(v, bbp[6 * i + threadIdx.x]) : fmax(v, bbp[6 * i + threadIdx.x]);
    bb[threadIdx.x] = v;
    if (blockIdx.x == 0) bbp[6 * FE_BBOX_BLOCKS + threadIdx.x] = v;   // the whole box
  }
  __syncthreads();
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npts) return;
  const int c = fe_morton_cell<BITS>(pts + 3 * q, bb);
  cell[q] = c;
  atomicAdd(count + c, 1);
}

// ``cursor`` starts as the exclusive scan of the cell counts.
__global__ void fe_points_place_kernel(const double* __restrict__ pts, int npts,
                                       const int* __restrict__ cell, int* __restrict__ cursor,
                                       double* __restrict__ out, float4* __restrict__ outf) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npts) return;
  const int at = atomicAdd(cursor + cell[q], 1);
  if (at < 0 || at >= npts) {
    fe_flag(FE_ST_OVERFLOW);
    return;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) out[3 * at + k] = pts[3 * q + k];
  outf[at] = make_float4(float(pts[3 * q]), float(pts[3 * q + 1]), float(pts[3 * q + 2]), 0.0f);
}

// E[i][j][t] of (u + xa)^i (u + xb)^j exp(-p u^2), i <= LA, j <= LB, t <= LA+LB.
template <int LA, int LB>
FE_DEV void fe_hermite_1d(double ip, double xa, double xb,
                          double (&e)[LA + 1][LB + 1][LA + LB + 1]) {
  constexpr int TM = LA + LB;
#pragma unroll
  for (int i = 0; i <= LA; ++i)
#pragma unroll
    for (int j = 0; j <= LB; ++j)
#pragma unroll
      for (int t = 0; t <= TM; ++t) e[i][j][t] = 0.0;
  e[0][0][0] = 1.0;
#pragma unroll
  for (int i = 0; i <= LA; ++i)
#pragma unroll
    for (int j = 0; j <= LB; ++j) {
      if (i == 0 && j == 0) continue;
      const int si = i > 0 ? i - 1 : i, sj = i > 0 ? j : j - 1;
      const double x = i > 0 ? xa : xb;
#pragma unroll
      for (int t = 0; t <= TM; ++t) {
        double v = 0.0;
        if (t >= 1) v += e[si][sj][t - 1] * ip;
        v += x * e[si][sj][t];
        if (t + 1 <= TM) v += double(t + 1) * e[si][sj][t + 1];
        e[i][j][t] = v;
      }
    }
}

// The reference's point screen (keep unless K bound / max(d, 0.05) < tol,
// d = dmin or dmin - reff, dmin the exact IEEE minimum of ((dx^2 + dy^2) +
// dz^2) over the points), decided without the full minimum where the answer
// is certain: with r* = K bound / tol,
//  * r* < 0.05 (1 - 1e-9): dropped, whatever dmin is;
//  * only points within rcut = (r* (1 + 1e-9) [+ reff]) can matter: boxes of
//    32 points (and superboxes of 1024) whose distance lower bound exceeds
//    rcut, or the best distance so far, are skipped;
//  * a point that makes the pair kept with a 1e-9 relative margin ends the
//    search (kept); no point within rcut means dropped;
//  * otherwise the minimum over the points within rcut is the exact dmin and
//    the reference's formula decides.
// The 1e-9 margins are far above the rounding of the tests themselves.
struct FeScreen {
  double KB, tol, rcut2, reff;
  int rule;
  bool none;                          // decided "drop" without a search
  FE_DEV FeScreen(const FeBuildArgs& a, double kb, double rf)
      : KB(kb), tol(a.tol), rcut2(0.0), reff(rf), rule(a.rule), none(false) {
    const double rstar = KB / tol;
    if (rstar < 0.05 * (1.0 - 1e-9)) {
      none = true;
    } else {
      const double rcut = (rstar * (1.0 + 1e-9) + (rule == 1 ? reff : 0.0)) * (1.0 + 1e-12);
      rcut2 = rcut * rcut;
    }
  }
  FE_DEV static double dist2(const double* q, const double (&P)[3]) {
    const double dx = __dsub_rn(q[0], P[0]);
    const double dy = __dsub_rn(q[1], P[1]);
    const double dz = __dsub_rn(q[2], P[2]);
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
  }
  FE_DEV bool sure_keep(double d2) const {
    double d = __dsqrt_rn(d2);
    if (rule == 1) d = d - reff;
    return KB >= tol * (1.0 + 1e-9) * fmax(d, 0.05);
  }
  // Every point of a (non-empty) box whose farthest corner is at squared
  // distance ub2 passes sure_keep: the corner distance, widened by 1e-12 for
  // rounding, meets the test with twice its margin.  Then the pair is kept
  // without looking at the points.
  FE_DEV bool sure_box(double ub2) const {
    double d = sqrt(ub2) * (1.0 + 1e-12);
    if (rule == 1) d = d - reff;
    return KB >= tol * (1.0 + 2e-9) * fmax(d, 0.05);
  }
  // the reference's decision from the exact minimum over the points within rcut
  FE_DEV bool keep_exact(double d2min) const {
    if (!(d2min < 1e300)) return false;
    double dd = __dsqrt_rn(d2min);
    if (rule == 1) dd = dd - reff;
    dd = fmax(dd, 0.05);
    return !(__ddiv_rn(KB, dd) < tol);
  }
};

// FP32 pre-test of the point screens.  With every coordinate of the points and
// of P rounded to float (error at most eps M, eps = 2^-24, M the largest
// coordinate magnitude of the points' box and of P), the FP32 distance of a
// point within rcut of P -- three roundings in the difference, three in the
// sum of squares -- is below (rcut + 4 eps M)(1 + 4 eps).  A point whose FP32
// squared distance exceeds that bound, rounded up to float, lies beyond rcut
// and is skipped; the others get the exact FP64 test, so the screen's
// minimum over the points within rcut, and its decision, are unchanged.
struct FeScreenF32 {
  float px, py, pz, r2f;
  FE_DEV FeScreenF32(const FeBuildArgs& a, const double (&P)[3], double rcut2) {
    double M = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k)
      M = fmax(M, fmax(fabs(P[k]), fmax(fabs(a.pbox[k]), fabs(a.pbox[3 + k]))));
    const double eps = 5.9604644775390625e-08;
    const double rf = (sqrt(rcut2) + 4.0 * eps * M) * (1.0 + 4.0 * eps);
    px = float(P[0]);
    py = float(P[1]);
    pz = float(P[2]);
    r2f = __double2float_ru(rf * rf);
  }
  FE_DEV bool maybe_within(float4 q) const {
    const float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
    return fmaf(dx, dx, fmaf(dy, dy, dz * dz)) <= r2f;
  }
};

// One thread's screen with a budget of FE_SCREEN_BUDGET box/point tests:
// 0 dropped, 1 kept, 2 undecided (the warp-parallel screen finishes it).
// (Not inlining it -- one copy for the 25 (la, lb) instances -- was measured:
// no faster, and the call spilled more of the caller to local memory.)
FE_DEV int fe_screen_thread(const FeBuildArgs& a, double px, double py, double pz, double KB,
                            double reff) {
  const double P[3] = {px, py, pz};
  if (a.npts == 0 || a.tol <= 0.0) return 1;        // no points, or tol 0: every pair is kept
  const FeScreen sc(a, KB, reff);
  if (sc.none) return 0;
  const FeScreenF32 sf(a, P, sc.rcut2);
  double d2min = 1e300;
  int steps = 0;
  for (int sb = 0; sb < a.nsbox; ++sb) {
    if (++steps > FE_SCREEN_BUDGET) return 2;
    const double ls = fe_box_lb2(a.sbox + 6 * sb, P) * (1.0 - 1e-12);
    if (ls > sc.rcut2 || ls > d2min) continue;
    if (sc.sure_box(fe_box_ub2(a.sbox + 6 * sb, P))) return 1;
    const int b1 = min(32 * sb + 32, a.nbox);
    for (int b = 32 * sb; b < b1; ++b) {
      if (++steps > FE_SCREEN_BUDGET) return 2;
      const double lb = fe_box_lb2(a.box + 6 * b, P) * (1.0 - 1e-12);
      if (lb > sc.rcut2 || lb > d2min) continue;
      if (sc.sure_box(fe_box_ub2(a.box + 6 * b, P))) return 1;
      const int q1 = min(32 * b + 32, a.npts);
      steps += q1 - 32 * b;
      for (int q = 32 * b; q < q1; ++q) {
        if (!sf.maybe_within(a.ptsf[q])) continue;
        const double d2 = FeScreen::dist2(a.pts + 3 * q, P);
        if (d2 <= sc.rcut2) d2min = fmin(d2min, d2);
      }
      if (d2min < 1e300 && sc.sure_keep(d2min)) return 1;
    }
  }
  return sc.keep_exact(d2min) ? 1 : 0;
}

template <int LA, int LB>
FE_DEV long long fe_build_pair(const FeBuildArgs& a, int w) {
  constexpr int L = LA + LB;
  constexpr int NA = (LA + 1) * (LA + 2) / 2, NB = (LB + 1) * (LB + 2) / 2;
  constexpr int NTRI = (L + 1) * (L + 2) * (L + 3) / 6;
  constexpr int NT = fe_class_nterm[L];
  constexpr int REC = fe_class_rec64[L];
  const FeTask tk = a.tasks[a.work_task[w]];
  const int ij = a.work_ij[w];
  const int ii = ij >> 16, jj = ij & 0xffff;
  const FeShell& A = a.shells[tk.si];
  const FeShell& B = a.shells[tk.sj];
  const long long slot = a.class_slot0[L] + tk.slot0 + ii * B.nprim + jj;
  a.keep[slot] = 0;
  a.srule[slot] = 0.0;
  a.swork[slot] = w;

  // density block of the shell pair (both orderings for si != sj); read again
  // where it is used (L1 hits) rather than held in a per-thread array, which
  // would live in local memory
  auto wdens = [&](int mu, int nu) {
    double d = a.dens[size_t(A.fn0 + mu) * a.n_func + (B.fn0 + nu)];
    if (tk.si != tk.sj) d += a.dens[size_t(B.fn0 + nu) * a.n_func + (A.fn0 + mu)];
    return d;
  };
  double wmax = 0.0;
#pragma unroll
  for (int mu = 0; mu < NA; ++mu)
#pragma unroll
    for (int nu = 0; nu < NB; ++nu) wmax = fmax(wmax, fabs(wdens(mu, nu)));
  if (!(wmax >= 1e-15)) return -1;

  const double al = a.sexp[A.prim0 + ii], be = a.sexp[B.prim0 + jj];
  const double cc = a.scoef[A.prim0 + ii] * a.scoef[B.prim0 + jj];
  const double p = al + be;
  double ab2 = 0.0, P[3], xa[3], xb[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double d = A.c[k] - B.c[k];
    ab2 += d * d;
  }
  const double K = exp(-(al * be) / p * ab2);
  if (!(K >= 1e-30)) return -1;
  if (a.rule == 1 && cc == 0.0) return -1;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    P[k] = (al * A.c[k] + be * B.c[k]) / p;
    xa[k] = P[k] - A.c[k];
    xb[k] = P[k] - B.c[k];
  }
  const double ip = 1.0 / (2.0 * p);
  double ex[LA + 1][LB + 1][L + 1], ey[LA + 1][LB + 1][L + 1], ez[LA + 1][LB + 1][L + 1];
  fe_hermite_1d<LA, LB>(ip, xa[0], xb[0], ex);
  fe_hermite_1d<LA, LB>(ip, xa[1], xb[1], ey);
  fe_hermite_1d<LA, LB>(ip, xa[2], xb[2], ez);

  double etab[NTRI];
#pragma unroll
  for (int t = 0; t < NTRI; ++t) etab[t] = 0.0;
  if constexpr (NA * NB <= 9) {
    // small shell pairs: every loop fully unrolled, so every index is a
    // compile-time constant and the E and etab arrays stay in registers
#pragma unroll
    for (int mu = 0; mu < NA; ++mu)
#pragma unroll
      for (int nu = 0; nu < NB; ++nu) {
        const int ax = fe_cart_exp(LA, mu, 0), ay = fe_cart_exp(LA, mu, 1), az = fe_cart_exp(LA, mu, 2);
        const int bx = fe_cart_exp(LB, nu, 0), by = fe_cart_exp(LB, nu, 1), bz = fe_cart_exp(LB, nu, 2);
        const double wt = wdens(mu, nu) * cc;
#pragma unroll
        for (int tx = 0; tx <= ax + bx; ++tx) {
          const double vx = wt * ex[ax][bx][tx];
#pragma unroll
          for (int ty = 0; ty <= ay + by; ++ty) {
            const double vxy = vx * ey[ay][by][ty];
            const int base = fe_tri<L>(tx, ty, 0);
#pragma unroll
            for (int tz = 0; tz <= az + bz; ++tz) etab[base + tz] += vxy * ez[az][bz][tz];
          }
        }
      }
  } else {
#pragma unroll 1
  for (int mu = 0; mu < NA; ++mu) {
    const int ax = fe_cart[LA][mu][0], ay = fe_cart[LA][mu][1], az = fe_cart[LA][mu][2];
#pragma unroll 1
    for (int nu = 0; nu < NB; ++nu) {
      const double wt = wdens(mu, nu) * cc;
      if (wt == 0.0) continue;
      const int bx = fe_cart[LB][nu][0], by = fe_cart[LB][nu][1], bz = fe_cart[LB][nu][2];
      for (int tx = 0; tx <= ax + bx; ++tx) {
        const double vx = wt * ex[ax][bx][tx];
        for (int ty = 0; ty <= ay + by; ++ty) {
          const double vxy = vx * ey[ay][by][ty];
          const int base = fe_tri<L>(tx, ty, 0);
          for (int tz = 0; tz <= az + bz; ++tz) etab[base + tz] += vxy * ez[az][bz][tz];
        }
      }
    }
  }
  }
  // sum rule: int rho_pair = K (pi/p)^1.5 etab[0]   (build_pairs.cpp:294-296)
  a.srule[slot] = K * pow(3.14159265358979323846 / p, 1.5) * etab[0];

  const double tp = 2.0 * p;
  const short* rp = fe_m0_ptr<L>();
  const short* rc = fe_m0_col<L>();
  const float* rv = fe_m0_val<L>();
  const signed char* rm = fe_m0_m<L>();
  // small pairs: the contraction sums as straight-line code (etab and the sums
  // stay in registers); larger ones walk the sparse rows
  constexpr bool kStraight = NA * NB <= 9;
  static_assert(!kStraight || L <= FE_M0_UNROLL_LMAX, "small pair above the straight-line classes");
  double gs[kStraight ? NT : 1];
  if constexpr (kStraight) fe_m0_rows<L>(etab, gs);
  if (a.rule == 1) {
    // the C++ builder drops pairs whose G are all zero (build_pairs.cpp:309)
    bool anyg = false;
    if constexpr (kStraight) {
#pragma unroll
      for (int k = 0; k < NT; ++k) anyg |= gs[k] != 0.0;
    } else {
#pragma unroll 1
      for (int k = 0; k < NT && !anyg; ++k) {
        double sk = 0.0;
        for (int q = rp[k]; q < rp[k + 1]; ++q) sk += double(rv[q]) * etab[rc[q]];
        anyg = sk != 0.0;
      }
    }
    if (!anyg) return -1;
  }

  // screening bound (esp.py:251-254)
  const double sq = sqrt(tp);
  double sqp[L + 1];
  sqp[0] = 1.0;
#pragma unroll
  for (int m = 1; m <= L; ++m) sqp[m] = sqp[m - 1] * sq;
  double bsum = 0.0;
#pragma unroll
  for (int tx = 0; tx <= L; ++tx)
#pragma unroll
    for (int ty = 0; ty <= L - tx; ++ty)
#pragma unroll
      for (int tz = 0; tz <= L - tx - ty; ++tz)
        bsum += fabs(etab[fe_tri<L>(tx, ty, tz)]) * (fe_screen_mom[tx] * fe_screen_mom[ty]
                 * fe_screen_mom[tz]) * sqp[tx + ty + tz];
  const double bound = pow(tp, -1.5) * bsum;
  const double reff = 1.6 * sqrt((L + 2.0) / p);
  const double KB = __dmul_rn(K, bound);
  const int decided = fe_screen_thread(a, P[0], P[1], P[2], KB, reff);
  if (decided == 0) return -1;

  // G_k = (2 pi / p) (2p)^m_k sum_t M0[k,t] etab[t], at record position fe_gpos_L[k]
  const double cf = 2.0 * 3.14159265358979323846 / p;
  double pw[L + 1];
  pw[0] = 1.0;
#pragma unroll
  for (int m = 1; m <= L; ++m) pw[m] = pw[m - 1] * tp;
  double* rec = a.stage + a.stage_off[L] + (slot - a.class_slot0[L]) * REC;
  if constexpr (kStraight) {
    fe_g_store<L>(gs, pw, cf, rec + 6);
  } else {
    const short* gpos = fe_gpos<L>();
#pragma unroll 1
    for (int k = 0; k < NT; ++k) {
      double sk = 0.0;
      for (int q = rp[k]; q < rp[k + 1]; ++q) sk += double(rv[q]) * etab[rc[q]];
      rec[6 + gpos[k]] = cf * pw[rm[k]] * sk;
    }
  }
  rec[0] = p;
  rec[1] = P[0];
  rec[2] = P[1];
  rec[3] = P[2];
  rec[4] = K;
  rec[5] = KB;
#pragma unroll
  for (int k = 6 + NT; k < REC; ++k) rec[k] = 0.0;
  if (decided == 2) return slot;        // undecided: fe_screen_pending_kernel finishes it
  a.keep[slot] = decided;
  return -1;
}

// The screen of one pair that its thread left undecided (fe_screen_thread ran
// past its budget), by the 32 lanes of a warp that all pass the same slot:
// superboxes across the lanes; then, one candidate superbox at a time, its
// boxes across the lanes, and the points of the boxes whose bounds leave them
// candidates, one box at a time across the lanes.  The decision is the serial search's:
// it depends only on whether some candidate box lies wholly within the keep
// radius (sure_box) and on the minimum squared distance over the points
// within rcut, which the box bounds only prune -- a box whose lower bound
// exceeds the minimum found so far holds no point that lowers it.  The lanes
// agree on d2min after each superbox (a shuffle reduction), so the decision
// comes back in every lane.
FE_DEV bool fe_screen_warp(const FeBuildArgs& a, const double (&P)[3], const FeScreen& sc,
                           int lane) {
  const FeScreenF32 sf(a, P, sc.rcut2);
  double d2min = 1e300;
  bool sure = sc.none;                        // (cannot happen: its thread searched)
  for (int sb0 = 0; sb0 < a.nsbox && !sure; sb0 += 32) {
    bool cand = false;
    if (sb0 + lane < a.nsbox) {
      const double ls = fe_box_lb2(a.sbox + 6 * (sb0 + lane), P) * (1.0 - 1e-12);
      cand = ls <= sc.rcut2 && ls <= d2min;
    }
    unsigned cm = __ballot_sync(0xffffffffu, cand);
    while (cm && !sure) {
      const int sbi = sb0 + __ffs(cm) - 1;
      cm &= cm - 1;
      if (fe_box_lb2(a.sbox + 6 * sbi, P) * (1.0 - 1e-12) > d2min) continue;
      if (sc.sure_box(fe_box_ub2(a.sbox + 6 * sbi, P))) {
        sure = true;
        break;
      }
      const int b = 32 * sbi + lane;
      bool bsure = false, bc = false;
      if (b < a.nbox) {
        const double lb = fe_box_lb2(a.box + 6 * b, P) * (1.0 - 1e-12);
        if (lb <= sc.rcut2 && lb <= d2min) {
          if (sc.sure_box(fe_box_ub2(a.box + 6 * b, P))) bsure = true;
          else bc = true;
        }
      }
      if (__any_sync(0xffffffffu, bsure)) {
        sure = true;
        break;
      }
      // the candidate boxes' points, one box at a time across the lanes
      // (coalesced), the minimum reduced once for the superbox
      double dl = 1e300;
      unsigned bm = __ballot_sync(0xffffffffu, bc);
      while (bm) {
        const int q = 32 * (32 * sbi + __ffs(bm) - 1) + lane;
        bm &= bm - 1;
        if (q < a.npts && sf.maybe_within(a.ptsf[q])) {
          const double d2 = FeScreen::dist2(a.pts + 3 * q, P);
          if (d2 <= sc.rcut2) dl = fmin(dl, d2);
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) dl = fmin(dl, __shfl_xor_sync(0xffffffffu, dl, o));
      d2min = fmin(d2min, dl);
      sure = d2min < 1e300 && sc.sure_keep(d2min);
    }
  }
  return sure || sc.keep_exact(d2min);
}

// The same for a pending pair, from its staging record.
FE_DEV bool fe_screen_warp(const FeBuildArgs& a, long long slot, int L, int lane) {
  const double* rec = a.stage + a.stage_off[L] + (slot - a.class_slot0[L]) * fe_c_rec64[L];
  const double P[3] = {rec[1], rec[2], rec[3]};
  const FeScreen sc(a, rec[5], 1.6 * sqrt((L + 2.0) / rec[0]));
  return fe_screen_warp(a, P, sc, lane);
}

// Shared-memory doubles per warp of fe_build_pair_warp<LA, LB>: the three E
// tables, the density block and etab.
template <int LA, int LB>
constexpr int fe_warp_pair_smem() {
  constexpr int L = LA + LB;
  return 3 * (LA + 1) * (LB + 1) * (L + 1) + (LA + 1) * (LA + 2) / 2 * ((LB + 1) * (LB + 2) / 2) +
         (L + 1) * (L + 2) * (L + 3) / 6;
}

// fe_build_pair for the heavy shell-pair groups, one warp per primitive pair:
// the work a thread would do alone for such a pair (about a hundred density
// elements, each spread over tens of Hermite entries, and a sparse
// contraction of over a hundred rows) is split over the lanes, and the point
// screen is the warp search from the start.  Every number is formed as in
// fe_build_pair, in the same order, so the records and decisions are the same
// bit for bit:
//  * lanes 0-2 compute the x, y, z E tables, kept in shared memory;
//  * lane l owns the Hermite entries t = l, l + 32, ...: it adds the
//    contributions of every density element (mu outer, nu inner, as the
//    thread does) to its entries, in registers;
//  * lane 0 sums the screening bound over etab in the thread's order;
//  * lane l owns the contraction rows k = l, l + 32, ...
// ``sh`` is this warp's fe_warp_pair_smem<LA, LB>() doubles.
template <int LA, int LB>
FE_DEV void fe_build_pair_warp(const FeBuildArgs& a, int w, int lane, double* sh) {
  constexpr int L = LA + LB;
  constexpr int NA = (LA + 1) * (LA + 2) / 2, NB = (LB + 1) * (LB + 2) / 2;
  constexpr int NTRI = (L + 1) * (L + 2) * (L + 3) / 6;
  constexpr int NT = fe_class_nterm[L];
  constexpr int REC = fe_class_rec64[L];
  constexpr int NE = (LA + 1) * (LB + 1) * (L + 1);
  constexpr int RT = (NTRI + 31) / 32, RK = (NT + 31) / 32;
  double* sE = sh;                     // [3][LA+1][LB+1][L+1]
  double* sW = sh + 3 * NE;            // [NA][NB]
  double* sT = sW + NA * NB;           // etab[NTRI]
  const FeTask tk = a.tasks[a.work_task[w]];
  const int ij = a.work_ij[w];
  const int ii = ij >> 16, jj = ij & 0xffff;
  const FeShell& A = a.shells[tk.si];
  const FeShell& B = a.shells[tk.sj];
  const long long slot = a.class_slot0[L] + tk.slot0 + ii * B.nprim + jj;
  if (lane == 0) {
    a.keep[slot] = 0;
    a.srule[slot] = 0.0;
    a.swork[slot] = w;
  }
  // density block (both orderings for si != sj)
  double wmax = 0.0;
  for (int c = lane; c < NA * NB; c += 32) {
    const int mu = c / NB, nu = c - mu * NB;
    double d = a.dens[size_t(A.fn0 + mu) * a.n_func + (B.fn0 + nu)];
    if (tk.si != tk.sj) d += a.dens[size_t(B.fn0 + nu) * a.n_func + (A.fn0 + mu)];
    sW[c] = d;
    wmax = fmax(wmax, fabs(d));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) wmax = fmax(wmax, __shfl_xor_sync(0xffffffffu, wmax, o));
  if (!(wmax >= 1e-15)) return;

  const double al = a.sexp[A.prim0 + ii], be = a.sexp[B.prim0 + jj];
  const double cc = a.scoef[A.prim0 + ii] * a.scoef[B.prim0 + jj];
  const double p = al + be;
  double ab2 = 0.0, P[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double d = A.c[k] - B.c[k];
    ab2 += d * d;
  }
  const double K = exp(-(al * be) / p * ab2);
  if (!(K >= 1e-30)) return;
  if (a.rule == 1 && cc == 0.0) return;
#pragma unroll
  for (int k = 0; k < 3; ++k) P[k] = (al * A.c[k] + be * B.c[k]) / p;
  const double ip = 1.0 / (2.0 * p);
  if (lane < 3) {
    double e[LA + 1][LB + 1][L + 1];
    fe_hermite_1d<LA, LB>(ip, P[lane] - A.c[lane], P[lane] - B.c[lane], e);
    double* dst = sE + lane * NE;
#pragma unroll
    for (int i = 0; i <= LA; ++i)
#pragma unroll
      for (int j = 0; j <= LB; ++j)
#pragma unroll
        for (int t = 0; t <= L; ++t) dst[(i * (LB + 1) + j) * (L + 1) + t] = e[i][j][t];
  }
  __syncwarp();

  // this lane's Hermite entries: t = lane + 32 r in the compact x-major order
  int tx[RT], ty[RT], tz[RT];
  double acc[RT];
#pragma unroll
  for (int r = 0; r < RT; ++r) {
    acc[r] = 0.0;
    tx[r] = ty[r] = tz[r] = L + 1;               // beyond every a + b: never added to
    int t = lane + 32 * r, n = 0;
    for (int x = 0; x <= L; ++x)
      for (int y = 0; y <= L - x; ++y)
        for (int z = 0; z <= L - x - y; ++z, ++n)
          if (n == t) {
            tx[r] = x;
            ty[r] = y;
            tz[r] = z;
          }
  }
  const double* EX = sE;
  const double* EY = sE + NE;
  const double* EZ = sE + 2 * NE;
#pragma unroll 1
  for (int mu = 0; mu < NA; ++mu) {
    const int ax = fe_cart[LA][mu][0], ay = fe_cart[LA][mu][1], az = fe_cart[LA][mu][2];
#pragma unroll 1
    for (int nu = 0; nu < NB; ++nu) {
      const double wt = sW[mu * NB + nu] * cc;
      const int bx = fe_cart[LB][nu][0], by = fe_cart[LB][nu][1], bz = fe_cart[LB][nu][2];
#pragma unroll
      for (int r = 0; r < RT; ++r)
        if (tx[r] <= ax + bx && ty[r] <= ay + by && tz[r] <= az + bz) {
          const double vx = wt * EX[(ax * (LB + 1) + bx) * (L + 1) + tx[r]];
          const double vxy = vx * EY[(ay * (LB + 1) + by) * (L + 1) + ty[r]];
          acc[r] += vxy * EZ[(az * (LB + 1) + bz) * (L + 1) + tz[r]];
        }
    }
  }
#pragma unroll
  for (int r = 0; r < RT; ++r)
    if (lane + 32 * r < NTRI) sT[lane + 32 * r] = acc[r];
  __syncwarp();
  // sum rule: int rho_pair = K (pi/p)^1.5 etab[0]   (build_pairs.cpp:294-296)
  if (lane == 0) a.srule[slot] = K * pow(3.14159265358979323846 / p, 1.5) * sT[0];

  // this lane's contraction sums: rows k = lane + 32 r
  const double tp = 2.0 * p;
  const short* rp = fe_m0_ptr<L>();
  const short* rc = fe_m0_col<L>();
  const float* rv = fe_m0_val<L>();
  const signed char* rm = fe_m0_m<L>();
  double gsum[RK];
  bool anyg = false;
#pragma unroll
  for (int r = 0; r < RK; ++r) {
    const int k = lane + 32 * r;
    double sk = 0.0;
    if (k < NT)
      for (int q = rp[k]; q < rp[k + 1]; ++q) sk += double(rv[q]) * sT[rc[q]];
    gsum[r] = sk;
    anyg |= sk != 0.0;
  }
  // the C++ builder drops pairs whose G are all zero (build_pairs.cpp:309)
  if (a.rule == 1 && !__any_sync(0xffffffffu, anyg)) return;

  // screening bound (esp.py:251-254), summed by lane 0 in the thread's order
  double KB = 0.0;
  if (lane == 0) {
    const double sq = sqrt(tp);
    double sqp[L + 1];
    sqp[0] = 1.0;
#pragma unroll
    for (int m = 1; m <= L; ++m) sqp[m] = sqp[m - 1] * sq;
    double bsum = 0.0;
#pragma unroll
    for (int x = 0; x <= L; ++x)
#pragma unroll
      for (int y = 0; y <= L - x; ++y)
#pragma unroll
        for (int z = 0; z <= L - x - y; ++z)
          bsum += fabs(sT[fe_tri<L>(x, y, z)]) * (fe_screen_mom[x] * fe_screen_mom[y]
                   * fe_screen_mom[z]) * sqp[x + y + z];
    const double bound = pow(tp, -1.5) * bsum;
    KB = __dmul_rn(K, bound);
  }
  KB = __shfl_sync(0xffffffffu, KB, 0);
  const double reff = 1.6 * sqrt((L + 2.0) / p);
  bool keep;
  if (a.npts == 0 || a.tol <= 0.0) {
    keep = true;                                 // no points, or tol 0: every pair is kept
  } else {
    const FeScreen sc(a, KB, reff);
    keep = !sc.none && fe_screen_warp(a, P, sc, lane);
  }
  if (!keep) return;

  // G_k = (2 pi / p) (2p)^m_k sum_t M0[k,t] etab[t], at record position fe_gpos_L[k]
  const double cf = 2.0 * 3.14159265358979323846 / p;
  double pw[L + 1];
  pw[0] = 1.0;
#pragma unroll
  for (int m = 1; m <= L; ++m) pw[m] = pw[m - 1] * tp;
  double* rec = a.stage + a.stage_off[L] + (slot - a.class_slot0[L]) * REC;
  const short* gpos = fe_gpos<L>();
#pragma unroll
  for (int r = 0; r < RK; ++r) {
    const int k = lane + 32 * r;
    if (k < NT) rec[6 + gpos[k]] = cf * pw[rm[k]] * gsum[r];
  }
  if (lane == 0) {
    rec[0] = p;
    rec[1] = P[0];
    rec[2] = P[1];
    rec[3] = P[2];
    rec[4] = K;
    rec[5] = KB;
  }
  for (int k = 6 + NT + lane; k < REC; k += 32) rec[k] = 0.0;
  if (lane == 0) a.keep[slot] = 1;
}

// Groups whose pairs take one warp each: those with at least this many
// density elements per shell pair (p-f and up; d-d).
#ifndef FE_WARP_PAIR_MIN
#define FE_WARP_PAIR_MIN 30
#endif
__host__ __device__ constexpr bool fe_warp_pair_group(int la, int lb) {
  return (la + 1) * (la + 2) / 2 * ((lb + 1) * (lb + 2) / 2) >= FE_WARP_PAIR_MIN;
}

// Threads per block of fe_build_warp_kernel (one pair per warp).
#define FE_WARP_BLOCK 128

template <int LA, int LB>
__global__ void __launch_bounds__(FE_WARP_BLOCK) fe_build_warp_kernel(const FeBuildArgs a,
                                                                     int work0, int nwork) {
  constexpr int SH = fe_warp_pair_smem<LA, LB>();
  constexpr int NW = FE_WARP_BLOCK / 32;
  __shared__ double sh[NW * SH];
  const int wid = int(threadIdx.x >> 5);
  const int w = int(blockIdx.x) * NW + wid;
  if (w < nwork) fe_build_pair_warp<LA, LB>(a, work0 + w, int(threadIdx.x & 31), sh + wid * SH);
}

#ifndef FE_BUILD_THREADS
#define FE_BUILD_THREADS 128
#endif

// One launch per (la, lb) group of work items (all primitive pairs of the
// shell pairs with these angular momenta): each group's code gets its own
// register allocation -- a single kernel over every group took the largest
// group's registers and spilled -- and the groups' launches run side by side
// on forked streams, so the long-running high-(la, lb) threads overlap the
// many light ones.
//
// A pair its thread leaves undecided goes to the pending list, which
// fe_screen_pending_kernel finishes after every group (finishing them inside
// the group's blocks was measured slower: the searching warps hold their
// blocks, and the long heavy-group blocks grow longer still).
template <int LA, int LB>
__global__ void __launch_bounds__(FE_BUILD_THREADS) fe_build_kernel(const FeBuildArgs a,
                                                                    int work0, int nwork) {
  const int w = int(blockIdx.x) * FE_BUILD_THREADS + int(threadIdx.x);
  if (w >= nwork) return;
  const long long slot = fe_build_pair<LA, LB>(a, work0 + w);
  if (slot >= 0) {
    const int at = atomicAdd(a.npending, 1);
    if (at < int(a.class_slot0[FE_NCLASS])) a.pending[at] = int(slot);
    else fe_flag(FE_ST_OVERFLOW);
  }
}

// The pending pairs, one warp each.
__global__ void __launch_bounds__(128) fe_screen_pending_kernel(const FeBuildArgs a) {
  const int lane = threadIdx.x & 31;
  const int warp = int((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarp = int((gridDim.x * blockDim.x) >> 5);
  const int np = min(*a.npending, int(a.class_slot0[FE_NCLASS]));
  for (int i = warp; i < np; i += nwarp) {
    const long long slot = a.pending[i];
    int L = 0;
    while (L + 1 < FE_NCLASS && slot >= a.class_slot0[L + 1]) ++L;
    const bool keep = fe_screen_warp(a, slot, L, lane);
    if (lane == 0) a.keep[slot] = keep ? 1 : 0;
  }
}

using FeBuildKernel = void (*)(const FeBuildArgs, int, int);

// The kernel of group la * 5 + lb: fe_build_warp_kernel (one warp per pair,
// FE_WARP_BLOCK / 32 pairs per block) for the heavy groups,
// fe_build_kernel (one thread per pair) for the rest.
template <int LA, int LB>
constexpr FeBuildKernel fe_group_kernel() {
  if constexpr (fe_warp_pair_group(LA, LB)) return fe_build_warp_kernel<LA, LB>;
  else return fe_build_kernel<LA, LB>;
}
inline FeBuildKernel fe_build_kernel_for(int code) {
#define FE_K(la, lb) fe_group_kernel<la, lb>(),
  static const FeBuildKernel k[25] = {
    FE_K(0, 0) FE_K(0, 1) FE_K(0, 2) FE_K(0, 3) FE_K(0, 4)
    FE_K(1, 0) FE_K(1, 1) FE_K(1, 2) FE_K(1, 3) FE_K(1, 4)
    FE_K(2, 0) FE_K(2, 1) FE_K(2, 2) FE_K(2, 3) FE_K(2, 4)
    FE_K(3, 0) FE_K(3, 1) FE_K(3, 2) FE_K(3, 3) FE_K(3, 4)
    FE_K(4, 0) FE_K(4, 1) FE_K(4, 2) FE_K(4, 3) FE_K(4, 4)};
#undef FE_K
  return code >= 0 && code < 25 ? k[code] : nullptr;
}
// Threads and pairs per block of group la * 5 + lb's kernel.
inline int fe_build_block_threads(int code) {
  return fe_warp_pair_group(code / 5, code % 5) ? FE_WARP_BLOCK : FE_BUILD_THREADS;
}
inline int fe_build_pairs_per_block(int code) {
  return fe_warp_pair_group(code / 5, code % 5) ? FE_WARP_BLOCK / 32 : FE_BUILD_THREADS;
}

// log2(x) for finite x > 0 and 2^y to about 1e-6 relative (float MUFU on the
// mantissa, exact exponent arithmetic in double): starting points only.
FE_DEV double fe_log2_approx(double x) {
  int e;
  const double m = frexp(x, &e);
  return double(e) + double(__log2f(float(m)));
}
FE_DEV double fe_exp2_approx(double y) {
  const double iy = floor(y);
  return ldexp(double(exp2f(float(y - iy))), int(fmax(fmin(iy, 2000.0), -2000.0)));
}

// Radius beyond which sum_n b_n / r^(n+1) < tau (b_n >= 0): with u = 1/r the
// sum is convex and increasing in u, so Newton's method started above the root
// (at the smallest u where one term alone reaches tau) descends to it
// monotonically.  0 when every b_n is 0 (never routed); +inf when a b_n is not
// finite.  Widened by 1e-6 relative so the radius is never below the exact one.
template <int L>
FE_DEV double fe_route_radius(const double (&b)[L + 1], double tau) {
  double u = 1e300;
  bool any = false;
  const double ltau = fe_log2_approx(tau);
#pragma unroll
  for (int n = 0; n <= L; ++n) {
    if (!(b[n] >= 0.0) || isinf(b[n])) return __longlong_as_double(0x7ff0000000000000LL);
    if (b[n] > 0.0) {
      // (tau / b_n)^(1/(n+1)), to ~1e-6, raised by 1e-4 so that the start is
      // above every single term's root and so above the sum's
      u = fmin(u, fe_exp2_approx((ltau - fe_log2_approx(b[n])) / double(n + 1)) * (1.0 + 1e-4));
      any = true;
    }
  }
  if (!any) return 0.0;
  for (int it = 0; it < 100; ++it) {
    double g = 0.0, dg = 0.0;                 // g = sum b_n u^n and g'(u), Horner
#pragma unroll
    for (int n = L; n >= 0; --n) {
      dg = fma(dg, u, g);
      g = fma(g, u, b[n]);
    }
    const double f = u * g, df = fma(u, dg, g);   // f = u g, f' = g + u g'
    const double step = (f - tau) / df;
    if (!(step > 1e-15 * u)) break;
    u -= step;
  }
  return (1.0 + 1e-6) / u;
}

// The mixed-precision record of one FP64 record ``r`` of class L (layout in
// table.cuh): coefficients c_k = K G_k s_m p^-(m+1/2) and the routing-bound
// coefficients formed in FP64, then rounded to float once.  ``tau_fast`` is
// the routing threshold the far radius is computed for.
template <int L>
FE_DEV void fe_f32_record(const double* __restrict__ r, float* __restrict__ o, float tau_fast) {
  constexpr int R32 = fe_class_rec32[L], NT = fe_class_nterm[L];
  auto split = [](double v, float& hi, float& lo) {
    hi = float(v);
    lo = float(v - double(hi));
  };
  const double p = r[0], K = r[4];
  o[0] = float(p);
  o[1] = float(sqrt(p));
#pragma unroll
  for (int k = 0; k < 3; ++k) split(r[1 + k], o[2 + k], o[5 + k]);
  o[9] = float(1.0 / sqrt(p));
  o[10] = o[11] = 0.0f;
  // s_m = (sqrt(pi)/2) (2m-1)!!/2^m (the FP32 Boys vector is F_m / s_m,
  // boys.cuh) and p^-(m+1/2): with both folded in, F_m of an asymptotic
  // point is 1/|R|^(2m+1) exactly
  double sm[L + 1], pm[L + 1];
  const double ip = 1.0 / p;
  sm[0] = FE_SQRT_PI_2;
  pm[0] = 1.0 / sqrt(p);
#pragma unroll
  for (int m = 1; m <= L; ++m) {
    sm[m] = sm[m - 1] * (0.5 * double(2 * m - 1));
    pm[m] = pm[m - 1] * ip;
  }
  // coefficient pairs, and the routing bound: K sum_k |G_k R^a F_m| <=
  // sum_n b_n / |R|^(n+1) with b_n = K sum_{k: 2m - |a| = n} |G_k| c_k
  // p^-(m + 1/2), rounded up to float
  double b[L + 1];
#pragma unroll
  for (int q = 0; q <= L; ++q) b[q] = 0.0;
  fe_f32_terms<L>(r + 6, K, sm, pm, o + 12, b);
#pragma unroll
  for (int q = 0; q <= L; ++q) {
    o[12 + 2 * NT + q] = __double2float_ru(K * b[q]);
    b[q] = double(o[12 + 2 * NT + q]);
  }
  // far radius: the FP32 Boys vector is asymptotic (T = p r^2 beyond the
  // class's FP32 threshold) and the bound (with the stored, rounded-up b_n)
  // is below tau_fast
  const double rt = fe_route_radius<L>(b, double(tau_fast));
  constexpr double tas = double(fe_boys32_asym_T[L]);
  const double ra2 = tas * ip * (1.0 + 1e-6);
  o[8] = __double2float_ru(fmax(ra2, rt * rt));
#pragma unroll
  for (int k = 13 + 2 * NT + L; k < R32; ++k) o[k] = 0.0f;
}

// Records per block of fe_records_kernel<L>: the tile's FP64 and FP32 records
// are both staged in shared memory (at most 78 KB, class 8).
__host__ __device__ constexpr int fe_records_tile_of(int L) {
  return L <= 3 ? 128 : (L == 4 ? 64 : (L == 5 ? 32 : 16));
}
template <int L>
constexpr int fe_records_tile() { return fe_records_tile_of(L); }

// Shared-memory row strides of the staged records, odd so that the thread of
// each record reads and writes its own row without bank conflicts.
template <int L>
constexpr int fe_records_smem_bytes() {
  return fe_records_tile<L>() * ((fe_class_rec64[L] + 1) * 8 + (fe_class_rec32[L] + 1) * 4);
}

// The table's records of class L, a tile of consecutive records per block:
//
// * build (``keep`` set): the tile is a range of the class's staging slots.
//   The kept slots' FP64 records move, in slot order, to their final rows
//   (``pos``, the exclusive scan of ``keep`` over all slots, gives the first
//   row of the tile), together with each one's work item in the table's
//   source section; then their mixed-precision records are derived.
// * imported table (``keep`` null): the FP64 records are in place and the
//   mixed-precision records of rows 0 .. count-1 are derived.
//
// Global loads and stores are coalesced (consecutive threads, consecutive
// words); each record's FP32 derivation runs in one thread on the staged copy.
template <int L>
__global__ void __launch_bounds__(128) fe_records_kernel(
    const double* __restrict__ stage, const int* __restrict__ keep, const int* __restrict__ pos,
    const int* __restrict__ swork, int nslot, unsigned char* table, float tau_fast) {
  constexpr int T = fe_records_tile<L>();
  constexpr int R64 = fe_class_rec64[L], R32 = fe_class_rec32[L];
  constexpr int S64 = R64 + 1, S32 = R32 + 1;
  extern __shared__ double fe_rec_smem[];
  double* in = fe_rec_smem;                                        // T x S64
  float* out = reinterpret_cast<float*>(fe_rec_smem + T * S64);    // T x S32
  __shared__ int src[T];
  __shared__ int wsum[4];
  FeTableHdr* hdr = reinterpret_cast<FeTableHdr*>(table);
  double* t64 = reinterpret_cast<double*>(table + hdr->off64[L]);
  float* t32 = reinterpret_cast<float*>(table + hdr->off32[L]);
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int n_all = keep ? nslot : min(hdr->count[L], hdr->cap[L]);
  for (int s0 = int(blockIdx.x) * T; s0 < n_all; s0 += int(gridDim.x) * T) {
    const int n = min(T, n_all - s0);
    int nk = n, d0 = s0;
    if (keep) {
      // kept slots of the tile, in order: warp ballots, then the warps' prefix
      const bool k = tid < n && keep[s0 + tid] != 0;
      const unsigned bal = __ballot_sync(0xffffffffu, k);
      if (lane == 0) wsum[wid] = __popc(bal);
      __syncthreads();
      int before = 0;
      nk = 0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        before += q < wid ? wsum[q] : 0;
        nk += wsum[q];
      }
      if (k) src[before + __popc(bal & ((1u << lane) - 1u))] = tid;
      d0 = pos[s0] - pos[0];
      if (d0 + nk > hdr->cap[L]) {
        if (tid == 0) fe_flag(FE_ST_OVERFLOW);
        nk = max(0, hdr->cap[L] - d0);
      }
      __syncthreads();
      // FP64 records to their rows (and to shared memory), work items to the
      // source section
      for (int e = tid; e < nk * R64; e += 128) {
        const int r = e / R64, c = e - r * R64;
        const double v = stage[size_t(s0 + src[r]) * R64 + c];
        in[r * S64 + c] = v;
        t64[size_t(d0) * R64 + e] = v;
      }
      if (tid < nk) {
        long long base = 0;
        for (int l = 0; l < L; ++l) base += hdr->cap[l];
        reinterpret_cast<int*>(table + hdr->off_src)[base + d0 + tid] = swork[s0 + src[tid]];
      }
    } else {
      for (int e = tid; e < n * R64; e += 128) {
        const int r = e / R64, c = e - r * R64;
        in[r * S64 + c] = t64[size_t(s0) * R64 + e];
      }
    }
    __syncthreads();
    if (tid < nk) fe_f32_record<L>(in + tid * S64, out + tid * S32, tau_fast);
    __syncthreads();
    for (int e = tid; e < nk * R32; e += 128) {
      const int r = e / R32, c = e - r * R32;
      t32[size_t(d0) * R32 + e] = out[r * S32 + c];
    }
    __syncthreads();
  }
  if (!keep && L == 0 && blockIdx.x == 0 && tid == 0) {
    hdr->has32 = 1;
    hdr->tau_fast = tau_fast;
  }
}

// Per-class kept counts and the sum rule.  One block of 1024 threads adds the
// per-scan-block sums of the sum-rule terms (``srule``, fixed trees of
// fe_scan_sums_kernel) in a fixed strided order and a fixed-shape tree, so the
// result does not depend on scheduling.  The mixed-precision records
// (fe_records_kernel) were derived for the routing threshold ``tau_fast``.
__global__ void __launch_bounds__(1024) fe_finalize_kernel(
    const long long* class_slot0, int nclass, long long nslot, const int* __restrict__ keep,
    const int* __restrict__ pos, const double* __restrict__ srule, const int* __restrict__ npending,
    unsigned char* table, float tau_fast) {
  __shared__ double red[1024];
  FeTableHdr* hdr = reinterpret_cast<FeTableHdr*>(table);
  const int t = threadIdx.x;
  if (t < nclass) {
    const long long a0 = class_slot0[t], a1 = class_slot0[t + 1];
    hdr->count[t] = a1 > a0 ? pos[a1 - 1] + keep[a1 - 1] - pos[a0] : 0;
  }
  // srule holds one partial sum per scan block (fe_scan_sums_kernel)
  const long long nb = (nslot + FE_SCAN_BLOCK - 1) / FE_SCAN_BLOCK;
  double s = 0.0;
  for (long long q = t; q < nb; q += 1024) s += srule[q];
  red[t] = s;
  __syncthreads();
  for (int h = 512; h > 0; h >>= 1) {
    if (t < h) red[t] += red[t + h];
    __syncthreads();
  }
  if (t == 0) {
    hdr->sum_rule = red[0];
    hdr->has_src = 1;
    hdr->has32 = 1;
    hdr->tau_fast = tau_fast;
    hdr->n_warp_screen = npending ? *npending : 0;
  }
}

// Exclusive scan of the keep flags in three deterministic passes:
// per-block sums, a single-block scan of those sums, then per-block scans.

__global__ void __launch_bounds__(FE_SCAN_BLOCK) fe_scan_sums_kernel(
    const int* __restrict__ keep, long long n, int* __restrict__ bsum,
    const double* __restrict__ srule = nullptr, double* __restrict__ bsr = nullptr) {
  __shared__ int red[FE_SCAN_BLOCK];
  __shared__ double dred[FE_SCAN_BLOCK];
  const long long i = blockIdx.x * (long long)FE_SCAN_BLOCK + threadIdx.x;
  red[threadIdx.x] = i < n ? keep[i] : 0;
  if (srule) dred[threadIdx.x] = i < n ? srule[i] : 0.0;
  __syncthreads();
  for (int h = FE_SCAN_BLOCK / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      red[threadIdx.x] += red[threadIdx.x + h];
      if (srule) dred[threadIdx.x] += dred[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    bsum[blockIdx.x] = red[0];
    if (srule) bsr[blockIdx.x] = dred[0];
  }
}

// In-place exclusive scan of ``bsum`` (nb entries) by one block, in tiles of
// FE_SCAN_BLOCK consecutive entries (coalesced): a shuffle scan over each warp
// and a scan of the warp totals give each entry's offset within the tile, and a
// running carry the tiles before it.
__global__ void __launch_bounds__(FE_SCAN_BLOCK) fe_scan_top_kernel(int* bsum, int nb) {
  __shared__ int wsum[FE_SCAN_BLOCK / 32];
  __shared__ int tile_total;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  int carry = 0;
  for (int base = 0; base < nb; base += FE_SCAN_BLOCK) {
    const int i = base + t;
    const int v = i < nb ? bsum[i] : 0;
    int inc = v;                                   // inclusive scan within the warp
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += u;
    }
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    if (w == 0) {
      const int x0 = lane < FE_SCAN_BLOCK / 32 ? wsum[lane] : 0;
      int x = x0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += u;
      }
      if (lane < FE_SCAN_BLOCK / 32) wsum[lane] = x - x0;   // exclusive warp offsets
      if (lane == 31) tile_total = x;
    }
    __syncthreads();
    if (i < nb) bsum[i] = carry + wsum[w] + inc - v;
    carry += tile_total;
    __syncthreads();                               // wsum and tile_total are reused
  }
}

__global__ void __launch_bounds__(FE_SCAN_BLOCK) fe_scan_apply_kernel(
    const int* __restrict__ keep, long long n, const int* __restrict__ bsum, int* __restrict__ pos) {
  __shared__ int buf[FE_SCAN_BLOCK];
  const long long i = blockIdx.x * (long long)FE_SCAN_BLOCK + threadIdx.x;
  const int v = i < n ? keep[i] : 0;
  buf[threadIdx.x] = v;
  __syncthreads();
  for (int off = 1; off < FE_SCAN_BLOCK; off <<= 1) {
    const int add = threadIdx.x >= off ? buf[threadIdx.x - off] : 0;
    __syncthreads();
    buf[threadIdx.x] += add;
    __syncthreads();
  }
  if (i < n) pos[i] = bsum[blockIdx.x] + buf[threadIdx.x] - v;
}


// ---------------------------------------------------------------------------
// Spatial order of the evaluation points
// ---------------------------------------------------------------------------
// The evaluators decide per warp of points (the mixed path's FP64 routing and
// far-pair test) and branch per warp (the Boys regimes), so a warp whose points
// lie close together does less work than one spread over the molecule.  With
// room in the workspace, the points are evaluated in the order of the Morton
// code of a 16^3 grid of cells over their bounding box, in the caller's order
// within a cell (a stable counting sort: the order, and so every result, is
// the same from run to run), and every result goes back to its caller's row.
#define FE_ORDER_BITS 4
#define FE_ORDER_CELLS (1 << (3 * FE_ORDER_BITS))

// idx: the points grouped by cell, in any order within a cell (``cursor``
// starts as the cells' first positions and ends as their ends).
__global__ void fe_order_place_kernel(const int* __restrict__ cell, int npts,
                                      int* __restrict__ cursor, int* __restrict__ idx) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npts) return;
  const int at = atomicAdd(cursor + cell[q], 1);
  if (at < 0 || at >= npts) {
    fe_flag(FE_ST_OVERFLOW);
    return;
  }
  idx[at] = q;
}

// Point q's final position: its cell's first position plus the number of the
// cell's points with a smaller caller index.  sorted[pos] = pts[q], perm[pos] = q.
// Each point scans its cell's segment, n^2 / 4096 comparisons for n evenly
// spread points: 80 M at the 568,950-point grid (tens of microseconds), small
// against the evaluation, which grows as n times the pair count.
__global__ void fe_order_rank_kernel(const double* __restrict__ pts, int npts,
                                     const int* __restrict__ cell, const int* __restrict__ start,
                                     const int* __restrict__ end, const int* __restrict__ idx,
                                     double* __restrict__ sorted, int* __restrict__ perm) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npts) return;
  const int c = cell[q];
  const int s = start[c], e = min(end[c], npts);
  int r = 0;
  for (int i = s; i < e; ++i) r += idx[i] < q;
  const int pos = s + r;
  if (pos < 0 || pos >= npts) {
    fe_flag(FE_ST_OVERFLOW);
    return;
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) sorted[3 * pos + k] = pts[3 * q + k];
  perm[pos] = q;
}
