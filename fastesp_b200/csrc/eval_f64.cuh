// FP64 ESP evaluation: V(C) = sum_A Z_A/|C - R_A| - sum_pairs K sum_k G_k R^a F_m(p R^2).
//
// Replaces the reference's esp_pairs_kernel + esp_reduce_kernel
// (fastesp/native/esp_gpu.cu:161-229) and PairTable.electron/esp
// (fastesp/table.py:73-104).
//
// Grid (x = point block, y = pair rows).  A block owns FE_EVAL_THREADS * NP
// points (NP per thread, kept in registers) and, through fe_class_rows, one
// part of one class's pairs (rows class-major, so concurrently running blocks
// execute the same class's code).  Its pairs are walked as tiles of whole records; thread 0 streams the
// tiles into a FE_NSTAGE-deep ring of shared-memory stages with 1-D TMA bulk
// copies completing on per-stage mbarriers, and every thread reads the current
// record as a warp-uniform broadcast, so each coefficient load feeds NP fused
// multiply-adds.  Per point, per pair: R = C - P, T = p|R|^2, the Boys vector
// F_0..F_L, and the class polynomial in nested Horner form.
//
// Every (point block, split) writes its partial electron sums to its own row of
// the workspace; fe_reduce_kernel adds all rows in a fixed order
// (deterministic) and the nuclear term.
#pragma once
#include "boys.cuh"
#include "table.cuh"

#ifndef FE_STAGE_BYTES
#define FE_STAGE_BYTES 16384
#endif
#ifndef FE_NSTAGE
#define FE_NSTAGE 2          // 2 stages leave more of the SM's shared/L1 to the L1 cache
#endif

struct FeEvalArgs {
  const unsigned char* table;      // table base (FeTableHdr at offset 0)
  const double* pts;               // (npts, 3) Bohr
  int npts;
  int nsplit;
  double* partial;                 // [nsplit][ld] partial electron sums of this kernel
  int ld;
  int lmin, lmax;                  // classes evaluated (a sub-range for per-class timing)
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

// The block's share of every class, kept in shared memory: pairs [lo, hi) of
// class L, cut into ntile tiles; ``total`` tiles in all.
struct FeBlockWork {
  int lo[FE_NCLASS];
  int hi[FE_NCLASS];
  int ntile[FE_NCLASS];
  int total;
  int woff[FE_NCLASS];   // first routing-mask word of class L (mixed path)
  int wtotal;            // routing-mask words per warp
};

// Thread 0 only.  Classes outside [llo, lhi] get no tiles.  ``align`` > 1
// puts every split boundary on a multiple of align pairs (the FP32 kernel uses
// 32 so that each 32-pair word of its routing mask has a single writer).
FE_DEV void fe_block_work(const FeTableHdr* hdr, int split, int nsplit, const int* tile_sz,
                          int llo, int lhi, FeBlockWork& w, int align = 1) {
  int total = 0, words = 0;
  for (int L = 0; L < FE_NCLASS; ++L) {
    const long long n = (L >= llo && L <= lhi) ? hdr->count[L] : 0;
    const long long lo = n * split / nsplit / align * align;
    const long long hi = split + 1 == nsplit ? n : n * (split + 1) / nsplit / align * align;
    w.lo[L] = int(lo);
    w.hi[L] = int(hi);
    w.ntile[L] = int((hi - lo + tile_sz[L] - 1) / tile_sz[L]);
    total += w.ntile[L];
    w.woff[L] = words;
    words += (hdr->count[L] + 31) / 32;
  }
  w.total = total;
  w.wtotal = words;
}

// Class-major assignment of a kernel's ``Y`` grid rows to the classes
// [llo, hi] that hold pairs: class L gets 1 + floor((Y - nz) W_L / sum W) rows
// (nz: classes with pairs; W_L = its 32-pair words times a per-pair cost),
// rows in class order, leftover rows idle (L = -1).  Row y -> (class L, part s
// of nL).  Blocks with consecutive y run the same class's code, so the SMs
// share one class's instructions at a time.  Needs Y >= nz.
FE_DEV void fe_class_rows(const FeTableHdr* hdr, int llo, int lhi, int Y, int y, int& L,
                          int& s, int& nL) {
  double W[FE_NCLASS], sum = 0.0;
  int nz = 0;
  for (int l = 0; l < FE_NCLASS; ++l) {
    const int words = (l >= llo && l <= lhi) ? (hdr->count[l] + 31) / 32 : 0;
    W[l] = double(words) * (2.0 * fe_c_nterm[l] + 20.0);
    sum += W[l];
    nz += words > 0;
  }
  int row = 0;
  for (int l = 0; l < FE_NCLASS; ++l) {
    if (W[l] == 0.0) continue;
    const int n = 1 + int(double(Y - nz) * W[l] / sum);
    if (y < row + n) {
      L = l;
      s = y - row;
      nL = n;
      return;
    }
    row += n;
  }
  L = -1;
  s = 0;
  nL = 1;
}

// Tile i of the block -> (class, first pair, pair count).
FE_DEV void fe_item(const FeBlockWork& w, const int* tile_sz, int i, int& L, int& first, int& n) {
  L = 0;
  while (L < FE_NCLASS - 1 && i >= w.ntile[L]) { i -= w.ntile[L]; ++L; }
  first = w.lo[L] + i * tile_sz[L];
  n = min(tile_sz[L], w.hi[L] - first);
}

// The block's tiles of records stream through a FE_NSTAGE ring of shared-memory
// stages: thread 0 issues 1-D TMA bulk copies that complete on per-stage
// mbarriers; every thread waits for the current stage, evaluates it, and the
// block releases it (a barrier) before thread 0 refills it.  ``elem`` bytes per
// record word, class record words ``rec[L]``, class byte offsets ``off[L]``.
// A persistent block runs several work items through one ring: ``base`` counts
// the tiles of its earlier items, so stage and phase continue from them and the
// mbarriers are initialised once (every issued tile is waited on before an
// item ends, so the ring is idle between items).
struct FeTilePipe {
  const unsigned char* table;
  const int* tile_sz;
  const int* rec;
  const int64_t* off;
  int elem;
  unsigned char* smem;
  uint64_t* bar;
  FeBlockWork* w;
  // optional second record array of the same pairs, staged right after the
  // first one's n records (rec2 == nullptr: none)
  const int* rec2 = nullptr;
  const int64_t* off2 = nullptr;
  int elem2 = 0;
  int base = 0;
  int stage_bytes = FE_STAGE_BYTES;   // bytes per ring stage (the tile sizes follow it)

  FE_DEV void init_barriers() const {
    if (threadIdx.x == 0) {
      for (int s = 0; s < FE_NSTAGE; ++s) mbar_init(&bar[s], 1);
      mbar_fence_init();
    }
  }
  // Work split of this item (thread 0), then the first FE_NSTAGE copies.
  FE_DEV void begin(const FeTableHdr* hdr, int split, int nsplit, int llo, int lhi, int align = 1) {
    if (threadIdx.x == 0) fe_block_work(hdr, split, nsplit, tile_sz, llo, lhi, *w, align);
    __syncthreads();
    if (threadIdx.x == 0)
      for (int i = 0; i < FE_NSTAGE && i < w->total; ++i) issue(i);
  }
  FE_DEV void start(const FeTableHdr* hdr, int split, int nsplit, int llo, int lhi, int align = 1) {
    init_barriers();
    begin(hdr, split, nsplit, llo, lhi, align);
  }
  FE_DEV void issue(int i) const {
    int L, first, n;
    fe_item(*w, tile_sz, i, L, first, n);
    const int s = (base + i) % FE_NSTAGE;
    const unsigned bytes = unsigned(n) * unsigned(rec[L]) * unsigned(elem);
    const unsigned bytes2 = rec2 ? unsigned(n) * unsigned(rec2[L]) * unsigned(elem2) : 0u;
    mbar_expect_tx(&bar[s], bytes + bytes2);
    bulk_g2s(smem + s * stage_bytes, table + off[L] + size_t(first) * rec[L] * elem, bytes,
             &bar[s]);
    if (rec2)
      bulk_g2s(smem + s * stage_bytes + bytes, table + off2[L] + size_t(first) * rec2[L] * elem2,
               bytes2, &bar[s]);
  }
  // Wait for tile i; false (for every thread) if the wait gave up.
  FE_DEV bool wait(int i) const {
    const int g = base + i;
    const bool got = mbar_wait_bounded(&bar[g % FE_NSTAGE], (g / FE_NSTAGE) & 1);
    return !__syncthreads_or(!got);
  }
  FE_DEV const unsigned char* stage(int i) const {
    return smem + ((base + i) % FE_NSTAGE) * stage_bytes;
  }
  FE_DEV void release(int i) const {
    __syncthreads();
    if (threadIdx.x == 0 && i + FE_NSTAGE < w->total) issue(i + FE_NSTAGE);
  }
  // After a failed wait at tile i: drain the copies still in flight.
  FE_DEV void abort(int i) const {
    if (threadIdx.x == 0)
      for (int k = i + 1; k < i + FE_NSTAGE && k < w->total; ++k) {
        const int g = base + k;
        mbar_wait_bounded(&bar[g % FE_NSTAGE], (g / FE_NSTAGE) & 1);
      }
    __syncthreads();
  }
};

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
    fe_poly<L, double, NP>(rec + 6, x, y, z, F, s);
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

template <int NP, int NT, int MINB, int LLO, int LHI>
__global__ void __launch_bounds__(NT, MINB) fe_eval_f64_kernel(const FeEvalArgs a) {
  extern __shared__ __align__(128) unsigned char fe_smem[];
  __shared__ uint64_t full_bar[FE_NSTAGE];
  __shared__ FeBlockWork w;
  const FeTableHdr* hdr = reinterpret_cast<const FeTableHdr*>(a.table);
  const int tid = threadIdx.x;
  const int split = blockIdx.y;

  // this thread's points (strided for coalesced loads); out-of-range lanes
  // evaluate a copy of the last point and store nothing
  double cx[NP], cy[NP], cz[NP], acc[NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const int q = min(int(blockIdx.x) * (NT * NP) + j * NT + tid, a.npts - 1);
    cx[j] = a.pts[3 * q];
    cy[j] = a.pts[3 * q + 1];
    cz[j] = a.pts[3 * q + 2];
    acc[j] = 0.0;
  }
  FeTilePipe pipe{a.table, fe_c_tile64, fe_c_rec64, hdr->off64, 8, fe_smem, full_bar, &w};
  int Lrow, part, nparts;
  fe_class_rows(hdr, max(LLO, a.lmin), min(LHI, a.lmax), a.nsplit, split, Lrow, part, nparts);
  if (Lrow >= 0) pipe.start(hdr, part, nparts, Lrow, Lrow);
  else pipe.start(hdr, 0, 1, 1, 0);                     // idle row: no tiles
  const int total = w.total;
  for (int i = 0; i < total; ++i) {
    if (!pipe.wait(i)) {
      pipe.abort(i);
      fe_poison_row<NP>(a.partial + size_t(split) * a.ld, int(blockIdx.x) * (NT * NP) + tid, NT,
                        a.npts);
      return;
    }
    int L, first, n;
    fe_item(w, fe_c_tile64, i, L, first, n);
    const double* rec = reinterpret_cast<const double*>(pipe.stage(i));
#define FE_C64(l) if (l >= LLO && l <= LHI && L == l) fe_tile_f64<(l >= LLO && l <= LHI ? l : LLO), NP>(rec, n, cx, cy, cz, acc);
    FE_C64(0) FE_C64(1) FE_C64(2) FE_C64(3) FE_C64(4) FE_C64(5) FE_C64(6) FE_C64(7) FE_C64(8)
#undef FE_C64
    if (L < LLO || L > LHI) fe_flag(FE_ST_BADCLASS);
    pipe.release(i);
  }

#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const int p = int(blockIdx.x) * (NT * NP) + j * NT + tid;
    if (p < a.npts) a.partial[size_t(split) * a.ld + p] = acc[j];
  }
}

// out[perm[i]] = nuclear(i) - sum_s partial[s][i] (mode 0) or the sum alone
// (mode 1); splits are added in order.  ``perm`` (the caller's row of
// evaluated point i) may be null: the identity.
__global__ void fe_reduce_kernel(const unsigned char* table, const double* __restrict__ pts,
                                 int npts, const double* __restrict__ partial, int nsplit,
                                 int ld, double* __restrict__ out, int mode,
                                 const int* __restrict__ perm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  const FeTableHdr* hdr = reinterpret_cast<const FeTableHdr*>(table);
  const int o = perm ? perm[i] : i;
  double e = 0.0;
  for (int s = 0; s < nsplit; ++s) e += partial[size_t(s) * ld + i];
  if (mode == 1) {
    out[o] = e;
    return;
  }
  const double* Z = reinterpret_cast<const double*>(table + hdr->off_atoms);
  out[o] = fe_nuclear(Z, Z + hdr->n_atoms, hdr->n_atoms, pts[3 * i], pts[3 * i + 1],
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
