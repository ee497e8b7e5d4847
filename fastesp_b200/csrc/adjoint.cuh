// Derivatives of the ESP: the field dV/dC and the adjoint with respect to the
// density matrix.
//
// With R = C - P and S_pair(C) = sum_k G_k R^a_k F_m_k(p R^2),
//   V(C) = sum_A Z_A / |C - R_A| - sum_pairs K S_pair(C)          (fastesp/table.py:73-104)
//   dS/dC_c = sum_k G_k (a_c R^(a - e_c) F_m - 2 p R_c R^a F_(m+1))
// because dF_m/dT = -F_(m+1).  For a loss L(V) with w_i = dL/dV_i,
//   dL/dC_i = w_i dV_i/dC_i,
//   dL/dG_k = -K sum_i w_i R_i^a_k F_m_k(p R_i^2)          (the pair's moments)
// and, through G_k = (2 pi/p)(2p)^m_k sum_t M0[k,t] etab[t] and
// etab[t] = sum_mu,nu W_mu,nu c_a c_b Ex Ey Ez (fastesp/esp.py:239-250),
//   dL/dW_mu,nu = c_a c_b sum_t lambda_t Ex[ax][bx][tx] Ey[ay][by][ty] Ez[az][bz][tz],
//   lambda_t    = sum_k (2 pi/p)(2p)^m_k M0[k,t] dL/dG_k.
// W is D[mu,nu] + D[nu,mu] for shell pairs si < sj and D[mu,nu] for si == sj,
// so dL/dD takes dL/dW summed over the primitive pairs of the shell pair, at
// both (mu,nu) and (nu,mu) when si < sj.  The kept pair set is held fixed: the
// table depends on D and C only through its kept pairs.
//
// Kernels:
//   fe_field_f64_kernel     point-parallel like the FP64 evaluator; four
//                           partial planes (V_el and its three derivatives)
//   fe_field_reduce_kernel  fixed-order sum of the planes, nuclear terms, w_i
//   fe_adj_moments_kernel   one block per (pair, term chunk), its threads
//                           over the points, moments reduced in a fixed order
//   fe_adj_pair_kernel      one thread per pair: the Hermite coefficients are
//                           recomputed (never stored), lambda, dL/dW per component
//   fe_adj_ranges_kernel,   deterministic segmented sum of dL/dW over each
//   fe_adj_gather_kernel    shell pair's primitive pairs into dL/dD
#pragma once
#include "build.cuh"
#include "eval_f64.cuh"

// ---------------------------------------------------------------------------
// field
// ---------------------------------------------------------------------------
struct FeFieldArgs {
  const unsigned char* table;
  const double* pts;
  int npts;
  int nsplit;
  double* partial;     // plane c (0: V_el, 1..3: dV_el/dC_c) starts at partial + c * plane
  size_t plane;        // doubles per plane
  int ld;
};

template <int L, int NP>
FE_DEV void fe_tile_field(const double* __restrict__ rec, int n, const double (&cx)[NP],
                          const double (&cy)[NP], const double (&cz)[NP], double (&acc)[4][NP]) {
  constexpr int S = fe_class_rec64[L];
#pragma unroll 1
  for (int i = 0; i < n; ++i, rec += S) {
    const double pe = rec[0], px = rec[1], py = rec[2], pz = rec[3], K = rec[4];
    double x[NP], y[NP], z[NP], F[NP][L + 2], s[NP], u[NP], dx[NP], dy[NP], dz[NP];
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      x[j] = cx[j] - px;
      y[j] = cy[j] - py;
      z[j] = cz[j] - pz;
      const double T = pe * fma(x[j], x[j], fma(y[j], y[j], z[j] * z[j]));
      fe_boys_f64<L + 1>(T, F[j]);
    }
    fe_grad<L, double, NP>(rec + 6, x, y, z, F, s, u, dx, dy, dz);
    const double tp = 2.0 * pe;
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      const double ku = tp * u[j];
      acc[0][j] = fma(K, s[j], acc[0][j]);
      acc[1][j] = fma(K, fma(-ku, x[j], dx[j]), acc[1][j]);
      acc[2][j] = fma(K, fma(-ku, y[j], dy[j]), acc[2][j]);
      acc[3][j] = fma(K, fma(-ku, z[j], dz[j]), acc[3][j]);
    }
  }
}

template <int NP, int NT, int MINB, int LLO, int LHI>
__global__ void __launch_bounds__(NT, MINB) fe_field_f64_kernel(const FeFieldArgs a) {
  extern __shared__ __align__(128) unsigned char fe_smem[];
  __shared__ uint64_t full_bar[FE_NSTAGE];
  __shared__ FeBlockWork w;
  const FeTableHdr* hdr = reinterpret_cast<const FeTableHdr*>(a.table);
  const int tid = threadIdx.x;
  const int split = blockIdx.y;
  double cx[NP], cy[NP], cz[NP], acc[4][NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const int q = min(int(blockIdx.x) * (NT * NP) + j * NT + tid, a.npts - 1);
    cx[j] = a.pts[3 * q];
    cy[j] = a.pts[3 * q + 1];
    cz[j] = a.pts[3 * q + 2];
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[c][j] = 0.0;
  }
  FeTilePipe pipe{a.table, fe_c_tile64, fe_c_rec64, hdr->off64, 8, fe_smem, full_bar, &w};
  int Lrow, part, nparts;
  fe_class_rows(hdr, LLO, LHI, a.nsplit, split, Lrow, part, nparts);
  if (Lrow >= 0) pipe.start(hdr, part, nparts, Lrow, Lrow);
  else pipe.start(hdr, 0, 1, 1, 0);                     // idle row: no tiles
  const int total = w.total;
  for (int i = 0; i < total; ++i) {
    if (!pipe.wait(i)) {
      pipe.abort(i);
      for (int c = 0; c < 4; ++c)
        fe_poison_row<NP>(a.partial + c * a.plane + size_t(split) * a.ld,
                          int(blockIdx.x) * (NT * NP) + tid, NT, a.npts);
      return;
    }
    int L, first, n;
    fe_item(w, fe_c_tile64, i, L, first, n);
    const double* rec = reinterpret_cast<const double*>(pipe.stage(i));
#define FE_CF(l) if (l >= LLO && l <= LHI && L == l) fe_tile_field<(l >= LLO && l <= LHI ? l : LLO), NP>(rec, n, cx, cy, cz, acc);
    FE_CF(0) FE_CF(1) FE_CF(2) FE_CF(3) FE_CF(4) FE_CF(5) FE_CF(6) FE_CF(7) FE_CF(8)
#undef FE_CF
    if (L < LLO || L > LHI) fe_flag(FE_ST_BADCLASS);
    pipe.release(i);
  }
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const int p = int(blockIdx.x) * (NT * NP) + j * NT + tid;
    if (p < a.npts)
#pragma unroll
      for (int c = 0; c < 4; ++c) a.partial[c * a.plane + size_t(split) * a.ld + p] = acc[c][j];
  }
}

// v[i] = nuclear - sum of plane 0 (if v), g[3i+c] = w_i (dnuc/dC_c - sum of plane
// c+1) (if g; w_i = 1 when w is null).  Rows are added in order.
__global__ void fe_field_reduce_kernel(const unsigned char* table, const double* __restrict__ pts,
                                       int npts, const double* __restrict__ partial, size_t plane,
                                       int nrows, int ld, const double* __restrict__ w,
                                       double* __restrict__ v, double* __restrict__ g) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  const FeTableHdr* hdr = reinterpret_cast<const FeTableHdr*>(table);
  const double* Z = reinterpret_cast<const double*>(table + hdr->off_atoms);
  const double* xyz = Z + hdr->n_atoms;
  const double cx = pts[3 * i], cy = pts[3 * i + 1], cz = pts[3 * i + 2];
  double e[4] = {0.0, 0.0, 0.0, 0.0};
  for (int c = 0; c < 4; ++c)
    for (int s = 0; s < nrows; ++s) e[c] += partial[c * plane + size_t(s) * ld + i];
  double nv = 0.0, nx = 0.0, ny = 0.0, nz = 0.0;
  for (int A = 0; A < hdr->n_atoms; ++A) {
    const double dx = cx - xyz[3 * A], dy = cy - xyz[3 * A + 1], dz = cz - xyz[3 * A + 2];
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double r = sqrt(r2);
    nv += Z[A] / r;
    const double q = Z[A] / (r2 * r);
    nx -= q * dx;
    ny -= q * dy;
    nz -= q * dz;
  }
  if (v) v[i] = nv - e[0];
  if (g) {
    const double wi = w ? w[i] : 1.0;
    g[3 * i] = wi * (nx - e[1]);
    g[3 * i + 1] = wi * (ny - e[2]);
    g[3 * i + 2] = wi * (nz - e[3]);
  }
}

// ---------------------------------------------------------------------------
// adjoint with respect to the density
// ---------------------------------------------------------------------------
#define FE_ADJ_THREADS 128

struct FeAdjArgs {
  const unsigned char* table;
  const double* pts;
  const double* w;             // dL/dV per point
  int npts;
  double* mom;                 // moments, class L at mom + mom_off[L], nt doubles per pair
  long long mom_off[FE_NCLASS];
  // plan
  const FeShell* shells;
  const double* sexp;
  const double* scoef;
  const FeTask* tasks;
  const int* work_task;
  const int* work_ij;
  int n_func;
  // dL/dW per pair (by source index) and the per-shell-pair ranges
  double* dw;
  int dw_stride;
  int* first;                  // per shell pair: first source index, -1 if none
  int* last;                   // per shell pair: one past the last source index
  long long nsrc;              // sum of the class capacities
  double* dD;                  // (n_func, n_func)
};

// mom[pair][k] = sum_i w_i R_i^a_k F_m_k(p R_i^2) for the terms of chunk C.
// One block per pair (and chunk): the pair is warp-uniform, as in the forward
// evaluator, so the lanes -- points i = tid, tid + 128, ... -- share the Boys
// branch of nearby points; each thread accumulates its points' moments in
// registers, then a fixed butterfly per warp and a fixed sum over the warps
// (deterministic) give the pair's moments.
template <int L, int C>
__global__ void __launch_bounds__(FE_ADJ_THREADS) fe_adj_moments_kernel(const FeAdjArgs a) {
  constexpr int K0 = fe_mom_k0[L][C], N = fe_mom_k1[L][C] - fe_mom_k0[L][C];
  constexpr int NTERM = fe_class_nterm[L];
  constexpr int NW = FE_ADJ_THREADS / 32;
  __shared__ double red[NW][N];
  const FeTableHdr* hdr = reinterpret_cast<const FeTableHdr*>(a.table);
  const int i = blockIdx.x;
  if (i >= hdr->count[L]) return;                  // the whole block
  const int tid = threadIdx.x, lane = tid & 31, wi = tid >> 5;
  const double* rec = reinterpret_cast<const double*>(a.table + hdr->off64[L]) +
                      size_t(i) * fe_class_rec64[L];
  const double pe = rec[0], px = rec[1], py = rec[2], pz = rec[3];
  double acc[N];
#pragma unroll
  for (int k = 0; k < N; ++k) acc[k] = 0.0;
#pragma unroll 1
  for (int q = tid; q < a.npts; q += FE_ADJ_THREADS) {
    const double x = a.pts[3 * q] - px, y = a.pts[3 * q + 1] - py, z = a.pts[3 * q + 2] - pz;
    const double T = pe * fma(x, x, fma(y, y, z * z));
    double F[L + 1];
    fe_boys_f64<L>(T, F);
    const double wq = a.w[q];
#pragma unroll
    for (int m = 0; m <= L; ++m) F[m] *= wq;
    fe_mom<L, C, double>(x, y, z, F, acc);
  }
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double v = acc[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[wi][k] = v;
  }
  __syncthreads();
  double* out = a.mom + a.mom_off[L] + size_t(i) * NTERM + K0;
  for (int k = tid; k < N; k += FE_ADJ_THREADS) {
    double v = red[0][k];
#pragma unroll
    for (int u = 1; u < NW; ++u) v += red[u][k];
    out[k] = v;
  }
}

// Source index g (class L, record i): lambda_t from the moments, then
// dL/dW_mu,nu for every component of the pair, written to dw[g][mu * NB + nu].
template <int LA, int LB>
FE_DEV void fe_adj_pair(const FeAdjArgs& a, long long g, int L_, int i, int wk) {
  constexpr int L = LA + LB;
  constexpr int NA = (LA + 1) * (LA + 2) / 2, NB = (LB + 1) * (LB + 2) / 2;
  constexpr int NTRI = (L + 1) * (L + 2) * (L + 3) / 6;
  constexpr int NTERM = fe_class_nterm[L];
  if (L_ != L) { fe_flag(FE_ST_BADCLASS); return; }
  const FeTask tk = a.tasks[a.work_task[wk]];
  const int ij = a.work_ij[wk];
  const int ii = ij >> 16, jj = ij & 0xffff;
  const FeShell& A = a.shells[tk.si];
  const FeShell& B = a.shells[tk.sj];
  // the builder's arithmetic, so p, P and K are bit-identical to the table's
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

  const double cf = 2.0 * 3.14159265358979323846 / p;
  const double tp = 2.0 * p;
  double pw[L + 1];
  pw[0] = 1.0;
#pragma unroll
  for (int m = 1; m <= L; ++m) pw[m] = pw[m - 1] * tp;
  double lam[NTRI];
#pragma unroll
  for (int t = 0; t < NTRI; ++t) lam[t] = 0.0;
  const double* mom = a.mom + a.mom_off[L] + size_t(i) * NTERM;
  const short* rp = fe_m0_ptr<L>();
  const short* rc = fe_m0_col<L>();
  const float* rv = fe_m0_val<L>();
  const signed char* rm = fe_m0_m<L>();
#pragma unroll 1
  for (int k = 0; k < NTERM; ++k) {
    const double gk = -K * mom[k] * cf * pw[rm[k]];      // dL/dG_k times the row's prefactor
    for (int q = rp[k]; q < rp[k + 1]; ++q) lam[rc[q]] += double(rv[q]) * gk;
  }
  double* out = a.dw + size_t(g) * a.dw_stride;
#pragma unroll 1
  for (int mu = 0; mu < NA; ++mu) {
    const int ax = fe_cart[LA][mu][0], ay = fe_cart[LA][mu][1], az = fe_cart[LA][mu][2];
#pragma unroll 1
    for (int nu = 0; nu < NB; ++nu) {
      const int bx = fe_cart[LB][nu][0], by = fe_cart[LB][nu][1], bz = fe_cart[LB][nu][2];
      double s = 0.0;
      for (int tx = 0; tx <= ax + bx; ++tx) {
        const double vx = ex[ax][bx][tx];
        for (int ty = 0; ty <= ay + by; ++ty) {
          const double vxy = vx * ey[ay][by][ty];
          const int base = fe_tri<L>(tx, ty, 0);
          double sz = 0.0;
          for (int tz = 0; tz <= az + bz; ++tz) sz = fma(lam[base + tz], ez[az][bz][tz], sz);
          s = fma(vxy, sz, s);
        }
      }
      out[mu * NB + nu] = cc * s;
    }
  }
}

// Source index -> (class, record); false past the class's kept count.
FE_DEV bool fe_src_class(const FeTableHdr* hdr, long long g, int& L, int& i) {
  long long base = 0;
  for (L = 0; L < FE_NCLASS; ++L) {
    if (g < base + hdr->cap[L]) {
      i = int(g - base);
      return i < hdr->count[L];
    }
    base += hdr->cap[L];
  }
  return false;
}

__global__ void __launch_bounds__(FE_ADJ_THREADS) fe_adj_pair_kernel(const FeAdjArgs a) {
  const long long g = blockIdx.x * (long long)FE_ADJ_THREADS + threadIdx.x;
  if (g >= a.nsrc) return;
  const FeTableHdr* hdr = reinterpret_cast<const FeTableHdr*>(a.table);
  int L, i;
  if (!fe_src_class(hdr, g, L, i)) return;
  const int wk = reinterpret_cast<const int*>(a.table + hdr->off_src)[g];
  const FeTask tk = a.tasks[a.work_task[wk]];
  const int code = a.shells[tk.si].l * 5 + a.shells[tk.sj].l;
  switch (code) {
#define FE_CASE(la, lb) case la * 5 + lb: fe_adj_pair<la, lb>(a, g, L, i, wk); break;
    FE_CASE(0, 0) FE_CASE(0, 1) FE_CASE(0, 2) FE_CASE(0, 3) FE_CASE(0, 4)
    FE_CASE(1, 0) FE_CASE(1, 1) FE_CASE(1, 2) FE_CASE(1, 3) FE_CASE(1, 4)
    FE_CASE(2, 0) FE_CASE(2, 1) FE_CASE(2, 2) FE_CASE(2, 3) FE_CASE(2, 4)
    FE_CASE(3, 0) FE_CASE(3, 1) FE_CASE(3, 2) FE_CASE(3, 3) FE_CASE(3, 4)
    FE_CASE(4, 0) FE_CASE(4, 1) FE_CASE(4, 2) FE_CASE(4, 3) FE_CASE(4, 4)
#undef FE_CASE
    default: fe_flag(FE_ST_BADCLASS); break;
  }
}

// The records of one shell pair are consecutive within their class (the
// builder keeps the reference's order), so each shell pair owns one run of
// source indices: first[] / last[] mark it.
__global__ void fe_adj_ranges_kernel(const FeAdjArgs a) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= a.nsrc) return;
  const FeTableHdr* hdr = reinterpret_cast<const FeTableHdr*>(a.table);
  int L, i;
  if (!fe_src_class(hdr, g, L, i)) return;
  const int* src = reinterpret_cast<const int*>(a.table + hdr->off_src);
  const int t = a.work_task[src[g]];
  if (i == 0 || a.work_task[src[g - 1]] != t) a.first[t] = int(g);
  if (i + 1 == hdr->count[L] || a.work_task[src[g + 1]] != t) a.last[t] = int(g) + 1;
}

// One thread per (shell pair, component): the dL/dD entry is the ordered sum
// over the shell pair's records.  dD must be zero on entry.
__global__ void fe_adj_gather_kernel(const FeAdjArgs a, int ntask) {
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long t = q / a.dw_stride;
  const int c = int(q % a.dw_stride);
  if (t >= ntask) return;
  const int f = a.first[t];
  if (f < 0) return;
  const FeTask tk = a.tasks[t];
  const FeShell& A = a.shells[tk.si];
  const FeShell& B = a.shells[tk.sj];
  const int NB = (B.l + 1) * (B.l + 2) / 2, NA = (A.l + 1) * (A.l + 2) / 2;
  if (c >= NA * NB) return;
  const int mu = c / NB, nu = c % NB;
  double s = 0.0;
  for (int g = f; g < a.last[t]; ++g) s += a.dw[size_t(g) * a.dw_stride + c];
  const size_t n = size_t(a.n_func);
  a.dD[size_t(A.fn0 + mu) * n + (B.fn0 + nu)] = s;
  if (tk.si != tk.sj) a.dD[size_t(B.fn0 + nu) * n + (A.fn0 + mu)] = s;
}
