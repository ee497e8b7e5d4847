// Batched FP64 evaluation: many molecules (each its own pair table and points)
// in one persistent launch over a flattened work queue.
//
// A work item is (molecule, point block, class L, part): the block evaluates
// the molecule's points [pb * PPB, (pb + 1) * PPB) against part ``part`` of
// ``nsplit[L]`` of the class-L pairs of its table and writes one row of partial
// sums.  The queue is class-major -- all class-0 items, then class 1, ... --
// and within a class largest first, so the blocks that run at the same time
// execute the same class's unrolled code (instruction-cache locality) and the
// expensive items start early.  Resident blocks take items from a global
// counter.  Every item writes its own row and fe_batch_reduce_kernel adds a
// molecule's rows in a fixed order, so the result is bitwise independent of
// which block ran which item.  The arithmetic per (pair, point) is that of
// fe_eval_f64_kernel: results equal fe_esp_fp64 up to the order of the part
// sums.  The g-shell classes (7, 8) have their own queue and kernel instance.
#pragma once
#include "eval_f64.cuh"

struct FeBatchMolDev {
  const unsigned char* table;
  const double* pts;
  double* out;
  int npts;
  int ld;                  // row length (points, padded to 32)
  int nrows;               // rows of all classes
  int pad_;
  int row0[FE_NCLASS];     // first row of class L
  int nsplit[FE_NCLASS];   // parts of class L (0: class empty)
  long long base;          // its first partial row starts at partial + base (doubles)
  long long pt0;           // first point of this molecule in the flattened point index
};

struct FeBatchHdr {
  int n_mol;
  int np;                  // points per thread of the items' point blocks
  int n_item[2];           // items of the two queues (classes 0..FE_LSPLIT, the rest)
  long long total_pts;
  long long off_mol;       // byte offsets within the descriptor
  long long off_item[2];
};

struct FeBatchItem {
  int mol, pblock, cls, part;
};

// STAGE: bytes per ring stage, i.e. the pair-tile size (STAGE / record bytes
// pairs of a class per tile); the autotuner picks it with the point block.
template <int NP, int MINB, int LLO, int LHI, int Q, int STAGE>
__global__ void __launch_bounds__(128, MINB) fe_batch_f64_kernel(const unsigned char* __restrict__ desc,
                                                                 unsigned* counter,
                                                                 double* partial) {
  constexpr int NT = 128;
  extern __shared__ __align__(128) unsigned char fe_smem[];
  __shared__ uint64_t full_bar[FE_NSTAGE];
  __shared__ FeBlockWork w;
  __shared__ int item_s;
  __shared__ int tile_s[FE_NCLASS];
  if (threadIdx.x < FE_NCLASS) tile_s[threadIdx.x] = STAGE / (8 * fe_c_rec64[threadIdx.x]);
  const FeBatchHdr* bh = reinterpret_cast<const FeBatchHdr*>(desc);
  const FeBatchMolDev* mols = reinterpret_cast<const FeBatchMolDev*>(desc + bh->off_mol);
  const FeBatchItem* items = reinterpret_cast<const FeBatchItem*>(desc + bh->off_item[Q]);
  const int n_item = bh->n_item[Q];
  const int tid = threadIdx.x;
  FeTilePipe pipe{nullptr, tile_s, fe_c_rec64, nullptr, 8, fe_smem, full_bar, &w};
  pipe.stage_bytes = STAGE;
  pipe.init_barriers();
  for (;;) {
    if (tid == 0) item_s = int(atomicAdd(counter, 1u));
    __syncthreads();
    const int it = item_s;
    if (it >= n_item) break;
    const FeBatchItem item = items[it];
    const FeBatchMolDev& m = mols[item.mol];
    const int L = item.cls;
    const FeTableHdr* hdr = reinterpret_cast<const FeTableHdr*>(m.table);
    double cx[NP], cy[NP], cz[NP], acc[NP];
    const int p0 = item.pblock * (NT * NP) + tid;
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      const int q = min(p0 + j * NT, m.npts - 1);
      cx[j] = m.pts[3 * q];
      cy[j] = m.pts[3 * q + 1];
      cz[j] = m.pts[3 * q + 2];
      acc[j] = 0.0;
    }
    pipe.table = m.table;
    pipe.off = hdr->off64;
    if (L >= LLO && L <= LHI) pipe.begin(hdr, item.part, m.nsplit[L], L, L);
    else pipe.begin(hdr, 0, 1, 1, 0);                  // not this instance's class: no tiles
    const int total = w.total;
    bool ok = true;
    for (int i = 0; i < total; ++i) {
      if (!pipe.wait(i)) {
        pipe.abort(i);
        ok = false;
        break;
      }
      int Lt, first, n;
      fe_item(w, tile_s, i, Lt, first, n);
      const double* rec = reinterpret_cast<const double*>(pipe.stage(i));
#define FE_CB(l) if (l >= LLO && l <= LHI && Lt == l) fe_tile_f64<(l >= LLO && l <= LHI ? l : LLO), NP>(rec, n, cx, cy, cz, acc);
      FE_CB(0) FE_CB(1) FE_CB(2) FE_CB(3) FE_CB(4) FE_CB(5) FE_CB(6) FE_CB(7) FE_CB(8)
#undef FE_CB
      pipe.release(i);
    }
    if (!ok) {                     // the status word says why; the points read NaN
      fe_poison_row<NP>(partial + m.base + size_t(m.row0[L] + item.part) * m.ld, p0, NT, m.npts);
      return;
    }
    if (L < LLO || L > LHI) fe_flag(FE_ST_BADCLASS);
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      const int p = p0 + j * NT;
      if (p < m.npts) partial[m.base + size_t(m.row0[L] + item.part) * m.ld + p] = acc[j];
    }
    pipe.base += total;
    __syncthreads();               // w and item_s are rewritten by the next item
  }
}

// One thread per point of the batch: out = nuclear - sum of its molecule's rows.
__global__ void fe_batch_reduce_kernel(const unsigned char* __restrict__ desc,
                                       const double* __restrict__ partial) {
  const FeBatchHdr* bh = reinterpret_cast<const FeBatchHdr*>(desc);
  const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (q >= bh->total_pts) return;
  const FeBatchMolDev* mols = reinterpret_cast<const FeBatchMolDev*>(desc + bh->off_mol);
  int lo = 0, hi = bh->n_mol - 1;          // last molecule with pt0 <= q
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (mols[mid].pt0 <= q) lo = mid; else hi = mid - 1;
  }
  const FeBatchMolDev& m = mols[lo];
  const int i = int(q - m.pt0);
  if (i >= m.npts) return;
  double e = 0.0;
  for (int r = 0; r < m.nrows; ++r) e += partial[m.base + size_t(r) * m.ld + i];
  const FeTableHdr* hdr = reinterpret_cast<const FeTableHdr*>(m.table);
  const double* Z = reinterpret_cast<const double*>(m.table + hdr->off_atoms);
  m.out[i] = fe_nuclear(Z, Z + hdr->n_atoms, hdr->n_atoms, m.pts[3 * i], m.pts[3 * i + 1],
                        m.pts[3 * i + 2]) - e;
}
