// FP64 ESP evaluation: V(C) = sum_A Z_A/|C - R_A| - sum_pairs K sum_k G_k R^a F_m(p R^2).
//
// Replaces the reference's esp_pairs_kernel + esp_reduce_kernel
// (fastesp/native/esp_gpu.cu:161-229) and PairTable.electron/esp
// (fastesp/table.py:73-104).
//
// Grid (x = point block, y = pair split).  A block owns FE_EVAL_THREADS * NP
// points (NP per thread, kept in registers) and 1/nsplit of the pairs of every
// class.  Its pairs are walked as tiles of whole records; thread 0 streams the
// tiles into a FE_NSTAGE-deep ring of shared-memory stages with 1-D TMA bulk
// copies completing on per-stage mbarriers, and every thread reads the current
// record as a warp-uniform broadcast, so each coefficient load feeds NP fused
// multiply-adds.  Per point, per pair: R = C - P, T = p|R|^2, the Boys vector
// F_0..F_L, and the class polynomial in nested Horner form.
//
// nsplit == 1: the epilogue adds the nuclear term and writes V directly.
// nsplit > 1 : each split writes its partial electron sum; fe_reduce_kernel
// adds the splits in a fixed order (deterministic) and the nuclear term.
#pragma once
#include "boys.cuh"
#include "table.cuh"

#ifndef FE_STAGE_BYTES
#define FE_STAGE_BYTES 16384
#endif
#ifndef FE_NSTAGE
#define FE_NSTAGE 3
#endif

struct FeEvalArgs {
  const unsigned char* table;      // table base (FeTableHdr at offset 0)
  const double* pts;               // (npts, 3) Bohr
  int npts;
  int nsplit;
  double* partial;                 // [nsplit][ld] when nsplit > 1
  int ld;
  double* out;                     // (npts,) when nsplit == 1
  int mode;                        // 0: V = nuclear - electron, 1: electron only
};

// Pairs of class L per stage / tile.
template <int L>
constexpr int fe_tile64() { return FE_STAGE_BYTES / (8 * fe_class_rec64[L]); }

__constant__ int fe_c_tile64[FE_NCLASS] = {
  FE_STAGE_BYTES / (8 * fe_class_rec64[0]), FE_STAGE_BYTES / (8 * fe_class_rec64[1]),
  FE_STAGE_BYTES / (8 * fe_class_rec64[2]), FE_STAGE_BYTES / (8 * fe_class_rec64[3]),
  FE_STAGE_BYTES / (8 * fe_class_rec64[4]), FE_STAGE_BYTES / (8 * fe_class_rec64[5]),
  FE_STAGE_BYTES / (8 * fe_class_rec64[6]), FE_STAGE_BYTES / (8 * fe_class_rec64[7]),
  FE_STAGE_BYTES / (8 * fe_class_rec64[8])};

// The block's share of class L: pairs [lo, hi).
struct FeBlockWork {
  int lo[FE_NCLASS];
  int ntile[FE_NCLASS];
  int total;
};

FE_DEV void fe_block_work(const FeTableHdr* hdr, int split, int nsplit,
                          const int* tile_sz, FeBlockWork& w) {
  w.total = 0;
#pragma unroll
  for (int L = 0; L < FE_NCLASS; ++L) {
    const long long n = hdr->count[L];
    const int lo = int(n * split / nsplit);
    const int hi = int(n * (split + 1) / nsplit);
    w.lo[L] = lo;
    w.ntile[L] = (hi - lo + tile_sz[L] - 1) / tile_sz[L];
    w.total += w.ntile[L];
  }
}

// Item i of the block -> (class, first pair, pair count).
FE_DEV void fe_item(const FeTableHdr* hdr, const FeBlockWork& w, int split, int nsplit,
                    const int* tile_sz, int i, int& L, int& first, int& n) {
  L = 0;
  while (L < FE_NCLASS - 1 && i >= w.ntile[L]) { i -= w.ntile[L]; ++L; }
  const long long cnt = hdr->count[L];
  const int hi = int(cnt * (split + 1) / nsplit);
  first = w.lo[L] + i * tile_sz[L];
  n = min(tile_sz[L], hi - first);
}

template <int L, int NP>
FE_DEV void fe_tile_f64(const double* __restrict__ rec, int n, const double (&cx)[NP],
                        const double (&cy)[NP], const double (&cz)[NP], double (&acc)[NP]) {
  constexpr int S = fe_class_rec64[L];
#pragma unroll 1
  for (int i = 0; i < n; ++i, rec += S) {
    const double pe = rec[0], px = rec[1], py = rec[2], pz = rec[3], K = rec[4];
    double x[NP], y[NP], z[NP], F[NP][L + 1], s[NP];
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      x[j] = cx[j] - px;
      y[j] = cy[j] - py;
      z[j] = cz[j] - pz;
      const double T = pe * fma(x[j], x[j], fma(y[j], y[j], z[j] * z[j]));
      fe_boys_f64<L>(T, F[j]);
    }
    fe_poly<L, double, NP>(rec + 5, x, y, z, F, s);
#pragma unroll
    for (int j = 0; j < NP; ++j) acc[j] = fma(K, s[j], acc[j]);
  }
}

FE_DEV double fe_nuclear(const double* __restrict__ Z, const double* __restrict__ xyz,
                         int natoms, double cx, double cy, double cz) {
  double v = 0.0;
  for (int a = 0; a < natoms; ++a) {
    const double dx = cx - xyz[3 * a], dy = cy - xyz[3 * a + 1], dz = cz - xyz[3 * a + 2];
    v += Z[a] / sqrt(dx * dx + dy * dy + dz * dz);
  }
  return v;
}

template <int NP, int NT>
__global__ void __launch_bounds__(NT) fe_eval_f64_kernel(const FeEvalArgs a) {
  extern __shared__ __align__(128) unsigned char fe_smem[];
  __shared__ uint64_t full_bar[FE_NSTAGE];
  const FeTableHdr* hdr = reinterpret_cast<const FeTableHdr*>(a.table);
  const int tid = threadIdx.x;
  const int split = blockIdx.y;

  // this thread's points (strided for coalesced loads); out-of-range lanes
  // evaluate a copy of the last point and store nothing
  double cx[NP], cy[NP], cz[NP], acc[NP];
  int pidx[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    pidx[j] = blockIdx.x * (NT * NP) + j * NT + tid;
    const int q = min(pidx[j], a.npts - 1);
    cx[j] = a.pts[3 * q];
    cy[j] = a.pts[3 * q + 1];
    cz[j] = a.pts[3 * q + 2];
    acc[j] = 0.0;
  }

  int tile_sz[FE_NCLASS];
#pragma unroll
  for (int L = 0; L < FE_NCLASS; ++L) tile_sz[L] = fe_c_tile64[L];
  FeBlockWork w;
  fe_block_work(hdr, split, a.nsplit, tile_sz, w);

  if (tid == 0) {
    for (int s = 0; s < FE_NSTAGE; ++s) mbar_init(&full_bar[s], 1);
    mbar_fence_init();
  }
  __syncthreads();

  auto issue = [&](int i) {
    int L, first, n;
    fe_item(hdr, w, split, a.nsplit, tile_sz, i, L, first, n);
    const int s = i % FE_NSTAGE;
    const unsigned bytes = unsigned(n) * unsigned(fe_c_rec64[L]) * 8u;
    const unsigned char* src = a.table + hdr->off64[L] + size_t(first) * fe_c_rec64[L] * 8;
    mbar_expect_tx(&full_bar[s], bytes);
    bulk_g2s(fe_smem + s * FE_STAGE_BYTES, src, bytes, &full_bar[s]);
  };
  if (tid == 0)
    for (int i = 0; i < FE_NSTAGE && i < w.total; ++i) issue(i);

  bool ok = true;
  int i = 0;
  for (; i < w.total; ++i) {
    const int s = i % FE_NSTAGE;
    const bool got = mbar_wait_bounded(&full_bar[s], (i / FE_NSTAGE) & 1);
    if (__syncthreads_or(!got)) { ok = false; break; }
    int L, first, n;
    fe_item(hdr, w, split, a.nsplit, tile_sz, i, L, first, n);
    const double* rec = reinterpret_cast<const double*>(fe_smem + s * FE_STAGE_BYTES);
    switch (L) {
      case 0: fe_tile_f64<0, NP>(rec, n, cx, cy, cz, acc); break;
      case 1: fe_tile_f64<1, NP>(rec, n, cx, cy, cz, acc); break;
      case 2: fe_tile_f64<2, NP>(rec, n, cx, cy, cz, acc); break;
      case 3: fe_tile_f64<3, NP>(rec, n, cx, cy, cz, acc); break;
      case 4: fe_tile_f64<4, NP>(rec, n, cx, cy, cz, acc); break;
      case 5: fe_tile_f64<5, NP>(rec, n, cx, cy, cz, acc); break;
      case 6: fe_tile_f64<6, NP>(rec, n, cx, cy, cz, acc); break;
      case 7: fe_tile_f64<7, NP>(rec, n, cx, cy, cz, acc); break;
      case 8: fe_tile_f64<8, NP>(rec, n, cx, cy, cz, acc); break;
      default: fe_flag(FE_ST_BADCLASS); break;
    }
    __syncthreads();                       // stage s fully consumed
    if (tid == 0 && i + FE_NSTAGE < w.total) issue(i + FE_NSTAGE);
  }
  if (!ok) {
    // drain copies still in flight before the block's shared memory goes away
    if (tid == 0)
      for (int k = i + 1; k < i + FE_NSTAGE && k < w.total; ++k)
        mbar_wait_bounded(&full_bar[k % FE_NSTAGE], (k / FE_NSTAGE) & 1);
    __syncthreads();
    return;
  }

  const double* Z = reinterpret_cast<const double*>(a.table + hdr->off_atoms);
  const double* xyz = Z + hdr->n_atoms;
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    if (pidx[j] >= a.npts) continue;
    if (a.nsplit == 1)
      a.out[pidx[j]] = a.mode == 1 ? acc[j]
                                   : fe_nuclear(Z, xyz, hdr->n_atoms, cx[j], cy[j], cz[j]) - acc[j];
    else
      a.partial[size_t(split) * a.ld + pidx[j]] = acc[j];
  }
}

// out[i] = nuclear(i) - sum_s partial[s][i] (mode 0) or the sum alone (mode 1);
// splits are added in order.
__global__ void fe_reduce_kernel(const unsigned char* table, const double* __restrict__ pts,
                                 int npts, const double* __restrict__ partial, int nsplit,
                                 int ld, double* __restrict__ out, int mode) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  const FeTableHdr* hdr = reinterpret_cast<const FeTableHdr*>(table);
  double e = 0.0;
  for (int s = 0; s < nsplit; ++s) e += partial[size_t(s) * ld + i];
  if (mode == 1) {
    out[i] = e;
    return;
  }
  const double* Z = reinterpret_cast<const double*>(table + hdr->off_atoms);
  out[i] = fe_nuclear(Z, Z + hdr->n_atoms, hdr->n_atoms, pts[3 * i], pts[3 * i + 1],
                      pts[3 * i + 2]) - e;
}

// out[i] = sum_A Z_A/|C_i - R_A| (fastesp/table.py:95-100).
__global__ void fe_nuclear_kernel(const unsigned char* table, const double* __restrict__ pts,
                                  int npts, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  const FeTableHdr* hdr = reinterpret_cast<const FeTableHdr*>(table);
  const double* Z = reinterpret_cast<const double*>(table + hdr->off_atoms);
  out[i] = fe_nuclear(Z, Z + hdr->n_atoms, hdr->n_atoms, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
}
