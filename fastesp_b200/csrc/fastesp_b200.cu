// libfastesp_b200: the C ABI of include/fastesp_b200.h.
//
// Single translation unit: the device code lives in the included headers,
// this file holds the host-side planning and the extern "C" entry points.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "classes_gen.cuh"
#include "boys.cuh"
#include "table.cuh"
#include "eval_f64.cuh"
#include "eval_mixed.cuh"
#include "build.cuh"
#include "adjoint.cuh"
#include "batch.cuh"
#include "points.cuh"
#include "../../include/fastesp_b200.h"

static_assert(FE_NCLASS <= FE_NCLASS_MAX, "class count");

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define FE_CUDA(call)                                                              \
  do {                                                                             \
    cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess)                                                         \
      return fail(FE_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_),     \
                  __FILE__, __LINE__);                                             \
  } while (0)

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Default FP64 routing threshold of the mixed evaluator (a.u.): the largest
// setting that kept the error against the FP64 path below 1e-6 a.u., with a
// margin, on the 54-atom l<=3 system (three 30000-point surface samples and the
// 568,950-point cubic grid, worst 7.7e-7; 0.05 reached 1.02e-6 on the grid).
// The FP32 records' far radius is computed for it, so smaller thresholds
// evaluate every pair through the exact per-point routing test.
constexpr double kTauDefault = 0.04;

int sm_count() {
  int dev = 0, n = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 148;
}

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// ID of the calling thread's current context (0 when none is current), from
// the driver's entry points as the runtime hands them out (no link to libcuda).
unsigned long long current_ctx_id() {
  static CtxGetCurrentFn get_cur = nullptr;
  static CtxGetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_cur = reinterpret_cast<CtxGetCurrentFn>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<CtxGetIdFn>(f);
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (!get_cur || !get_id || get_cur(&ctx) != CUDA_SUCCESS || !ctx) return 0;
  if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Side streams of the table build, per device: the build's (la, lb) group
// launches fork from the caller's stream onto these and join back through
// events, so the groups run side by side and every later launch on the
// caller's stream waits for all of them.  Created on first use; a device reset
// (a new context ID) makes them be created again.  The mutex is held from the
// fork to the join, so concurrent builds on one device take turns on them.
#ifndef FE_SIDE_STREAMS
#define FE_SIDE_STREAMS 8
#endif
#define FE_SIDE_MAX_DEVICES 128
struct SideStreams {
  cudaStream_t s[FE_SIDE_STREAMS] = {};
  cudaEvent_t fork = nullptr, join[FE_SIDE_STREAMS] = {};
  unsigned long long ctx_id = 0;
};
std::mutex g_side_mu;
SideStreams g_side[FE_SIDE_MAX_DEVICES];

int side_streams(SideStreams** out) {
  int dev = 0;
  FE_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= FE_SIDE_MAX_DEVICES)
    return fail(FE_ERR_UNSUPPORTED, "table build: device ordinal %d too large", dev);
  SideStreams& ss = g_side[dev];
  const unsigned long long id = current_ctx_id();
  if (!ss.fork || id == 0 || id != ss.ctx_id) {
    // handles of a replaced context are not destroyed: they died with it
    ss = SideStreams{};
    for (int i = 0; i < FE_SIDE_STREAMS; ++i) {
      FE_CUDA(cudaStreamCreateWithFlags(&ss.s[i], cudaStreamNonBlocking));
      FE_CUDA(cudaEventCreateWithFlags(&ss.join[i], cudaEventDisableTiming));
    }
    FE_CUDA(cudaEventCreateWithFlags(&ss.fork, cudaEventDisableTiming));
    ss.ctx_id = current_ctx_id();
  }
  *out = &ss;
  return FE_OK;
}

// Two sets side by side: set A (na items) on the caller's stream and the first
// side streams, set B (nb items) on the others; once set A is done,
// after_a(st) runs on the caller's stream while set B may still run; later
// launches on ``st`` wait for both sets.
template <typename FA, typename FM, typename FB>
int fork_join2(int na, int nb, cudaStream_t st, FA&& launch_a, FM&& after_a, FB&& launch_b) {
  std::lock_guard<std::mutex> lock(g_side_mu);
  SideStreams* ss = nullptr;
  int rc = side_streams(&ss);
  if (rc != FE_OK) return rc;
  const int kb = nb > 0 ? std::min(nb, FE_SIDE_STREAMS / 2) : 0;
  const int ka = std::min(std::max(na - 1, 0), FE_SIDE_STREAMS - kb);
  if (ka + kb > 0) FE_CUDA(cudaEventRecord(ss->fork, st));
  for (int i = 0; i < ka + kb; ++i) FE_CUDA(cudaStreamWaitEvent(ss->s[i], ss->fork, 0));
  for (int i = 0; i < na && rc == FE_OK; ++i) {
    const int q = i % (ka + 1);
    rc = launch_a(i, q == 0 ? st : ss->s[q - 1]);
  }
  for (int i = 0; i < nb && rc == FE_OK; ++i) rc = launch_b(i, ss->s[ka + i % kb]);
  for (int i = 0; i < ka; ++i) {
    FE_CUDA(cudaEventRecord(ss->join[i], ss->s[i]));
    FE_CUDA(cudaStreamWaitEvent(st, ss->join[i], 0));
  }
  if (rc == FE_OK) rc = after_a(st);
  for (int i = ka; i < ka + kb; ++i) {
    FE_CUDA(cudaEventRecord(ss->join[i], ss->s[i]));
    FE_CUDA(cudaStreamWaitEvent(st, ss->join[i], 0));
  }
  return rc;
}

// Run launch(i, stream) for i = 0..n-1 side by side: item i goes to the
// caller's stream (i % (k + 1) == 0) or side stream i % (k + 1) - 1, k the
// side streams used; the side streams start after the work already on ``st``
// and every later launch on ``st`` waits for them.  The side streams are
// joined even when a launch fails.
template <typename F>
int fork_join(int n, cudaStream_t st, F&& launch) {
  if (n <= 0) return FE_OK;
  std::lock_guard<std::mutex> lock(g_side_mu);
  SideStreams* ss = nullptr;
  int rc = side_streams(&ss);
  if (rc != FE_OK) return rc;
  const int nside = std::min(n - 1, FE_SIDE_STREAMS);
  if (nside > 0) FE_CUDA(cudaEventRecord(ss->fork, st));
  for (int i = 0; i < nside; ++i) FE_CUDA(cudaStreamWaitEvent(ss->s[i], ss->fork, 0));
  for (int i = 0; i < n && rc == FE_OK; ++i) {
    const int q = i % (nside + 1);
    rc = launch(i, q == 0 ? st : ss->s[q - 1]);
  }
  for (int i = 0; i < nside; ++i) {
    FE_CUDA(cudaEventRecord(ss->join[i], ss->s[i]));
    FE_CUDA(cudaStreamWaitEvent(st, ss->join[i], 0));
  }
  return rc;
}

// fe_records_kernel<L> on ``st``: the build's compaction of class L (``keep``
// set; stage, keep, pos and swork are the class's slices, nslot its slot
// count) or, for an imported table, the derivation of its FP32 records.
template <int L>
int launch_records_l(const double* stage, const int* keep, const int* pos, const int* swork,
                     int nslot, unsigned char* table, unsigned grid, cudaStream_t st) {
  constexpr int smem = fe_records_smem_bytes<L>();
  FE_CUDA(cudaFuncSetAttribute(fe_records_kernel<L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               smem));
  fe_records_kernel<L><<<grid, 128, smem, st>>>(stage, keep, pos, swork, nslot, table,
                                                float(kTauDefault));
  FE_CUDA(cudaGetLastError());
  return FE_OK;
}

int launch_records(int L, const double* stage, const int* keep, const int* pos,
                   const int* swork, int nslot, unsigned char* table, unsigned grid,
                   cudaStream_t st) {
  switch (L) {
#define FE_R(l) case l: return launch_records_l<l>(stage, keep, pos, swork, nslot, table, grid, st);
    FE_R(0) FE_R(1) FE_R(2) FE_R(3) FE_R(4) FE_R(5) FE_R(6) FE_R(7) FE_R(8)
#undef FE_R
    default: return fail(FE_ERR_ARG, "records: class %d out of range", L);
  }
}

// ---------------------------------------------------------------------------
// Evaluation launch geometry
// ---------------------------------------------------------------------------
// Points per thread and minimum resident blocks of 128 threads per SM of the
// FP64 and mixed evaluators (defaults chosen by measurement on B200).
#ifndef FE_NP64
#define FE_NP64 2
#endif
#ifndef FE_MINB64
#define FE_MINB64 4
#endif
#ifndef FE_MINB32
#define FE_MINB32 3
#endif
#ifndef FE_MINB32LO
#define FE_MINB32LO 4
#endif
#ifndef FE_MINBFIX
#define FE_MINBFIX 4
#endif
constexpr int kEvalThreads = 128;
constexpr int kNP64 = FE_NP64, kMinB64 = FE_MINB64;
constexpr int kNP32 = FE_MX_NP, kMinB32 = FE_MINB32, kMinB32Lo = FE_MINB32LO, kMinBFix = FE_MINBFIX;

// Class ranges of the two kernel instances of every evaluator: classes up to
// FE_LSPLIT (s..f shell pairs) and the g-shell classes above it, compiled
// separately so the common classes do not carry the registers of the largest.
#define FE_LSPLIT 6
// The packed FP32 kernel is split once more, at FE_MXSPLIT: classes 0..4 fit in
// 128 registers and, with a 2-stage ring and their 5 Boys-grid orders in shared
// memory, run 4 blocks per SM; classes 5..6 need 159 registers (3 per SM).
#define FE_MXSPLIT 4

struct EvalGeom {
  int nblk_x, ld;
  int split[5];        // FP64: main, high; mixed: FP32 0..4, 5..6, high, FP64 part main, high
  int nkern;
  size_t ws_rows() const {
    size_t r = 0;
    for (int k = 0; k < nkern; ++k) r += size_t(split[k]);
    return r;
  }
};

// Point blocks x pair splits: about 8 waves of resident blocks for the main
// instances, so the last partial wave costs little (splits capped at 256);
// the g-class instances get a few splits (they are empty for s..f bases).
// Every kernel writes its own rows of partial sums; one reduction adds all
// rows in a fixed order.
EvalGeom eval_geom(int npts, int mode) {
  const int ppb = kEvalThreads * (mode == 1 ? kNP32 : kNP64);
  EvalGeom g{};
  g.nblk_x = (npts + ppb - 1) / ppb;
  auto splits = [&](int minb) {
    const int target = 8 * minb * sm_count();
    return std::max(1, std::min(256, (target + g.nblk_x - 1) / std::max(1, g.nblk_x)));
  };
  const int hi_splits = std::max(1, std::min(8, sm_count() / std::max(1, g.nblk_x)));
  g.ld = (npts + 31) & ~31;
  // every kernel needs at least one grid row per class of its range (fe_class_rows)
  const int nlo = FE_LSPLIT + 1, nhi = FE_NCLASS - 1 - FE_LSPLIT;
  if (mode == 1) {
    // classes 5..6 carry about an eighth of the FP32 work: two waves of their own
    g.nkern = 5;
    g.split[0] = std::max(FE_MXSPLIT + 1, splits(kMinB32Lo));
    g.split[1] = std::max(FE_LSPLIT - FE_MXSPLIT, splits(kMinB32) / 4);
    g.split[2] = std::max(nhi, hi_splits);
    g.split[3] = std::max(nlo, splits(kMinBFix));
    g.split[4] = std::max(nhi, hi_splits);
  } else {
    g.nkern = 2;
    g.split[0] = std::max(nlo, splits(kMinB64));
    g.split[1] = std::max(nhi, hi_splits);
  }
  return g;
}

struct Layout {
  size_t off64[FE_NCLASS], off32[FE_NCLASS], off_atoms, off_src, bytes;
};

Layout table_layout(const int* cap, int n_atoms) {
  Layout l{};
  size_t t = FE_TABLE_HDR_BYTES;
  for (int L = 0; L < FE_NCLASS; ++L) {
    l.off64[L] = t;
    t = align256(t + size_t(cap[L]) * fe_class_rec64[L] * 8);
  }
  for (int L = 0; L < FE_NCLASS; ++L) {
    l.off32[L] = t;
    t = align256(t + size_t(cap[L]) * fe_class_rec32[L] * 4);
  }
  l.off_atoms = t;
  t = align256(t + size_t(n_atoms) * 4 * sizeof(double));
  l.off_src = t;
  size_t nrec = 0;
  for (int L = 0; L < FE_NCLASS; ++L) nrec += size_t(cap[L]);
  l.bytes = align256(t + nrec * sizeof(int));
  return l;
}

// Header + atom block of a table with the given capacities (counts zero).
int write_header(unsigned char* d_table, const int* cap, int n_atoms, const double* Z,
                 const double* xyz, double tol, int rule, cudaStream_t st) {
  const Layout lay = table_layout(cap, n_atoms);
  FeTableHdr hdr{};
  hdr.magic = FE_TABLE_MAGIC;
  hdr.nclass = FE_NCLASS;
  hdr.n_atoms = n_atoms;
  hdr.rule = rule;
  hdr.tol = tol;
  for (int L = 0; L < FE_NCLASS; ++L) {
    hdr.cap[L] = cap[L];
    hdr.off64[L] = static_cast<long long>(lay.off64[L]);
    hdr.off32[L] = static_cast<long long>(lay.off32[L]);
  }
  hdr.off_atoms = static_cast<long long>(lay.off_atoms);
  hdr.off_src = static_cast<long long>(lay.off_src);
  hdr.has_src = 0;
  hdr.bytes = static_cast<long long>(lay.bytes);
  std::vector<unsigned char> h(sizeof hdr + size_t(n_atoms) * 4 * sizeof(double));
  memcpy(h.data(), &hdr, sizeof hdr);
  FE_CUDA(cudaMemcpyAsync(d_table, h.data(), sizeof hdr, cudaMemcpyHostToDevice, st));
  if (n_atoms > 0) {
    std::vector<double> atoms(Z, Z + n_atoms);
    atoms.insert(atoms.end(), xyz, xyz + 3 * size_t(n_atoms));
    FE_CUDA(cudaMemcpyAsync(d_table + lay.off_atoms, atoms.data(), atoms.size() * sizeof(double),
                            cudaMemcpyHostToDevice, st));
  }
  FE_CUDA(cudaStreamSynchronize(st));   // host staging buffers are locals
  return FE_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// Plan
// ---------------------------------------------------------------------------
struct fe_plan {
  int n_func = 0, n_atoms = 0;
  std::vector<FeShell> shells;
  std::vector<double> sexp, scoef;
  std::vector<FeTask> tasks;
  std::vector<int> work_task, work_ij;
  std::vector<int> grp_code, grp_work0, grp_nwork;   // (la, lb) groups of work items
  std::vector<long long> class_slot0;   // FE_NCLASS + 1
  std::vector<long long> stage_off;     // FE_NCLASS, in doubles
  std::vector<double> Z, xyz;
  long long nslot = 0;
  int nblocks = 0;
  int cap[FE_NCLASS] = {};
  // device blob layout (byte offsets)
  size_t o_shells, o_sexp, o_scoef, o_tasks, o_wt, o_wij, o_cs, o_so;
  size_t plan_bytes = 0;
  size_t table_bytes = 0;
  size_t o_tab64[FE_NCLASS], o_tab32[FE_NCLASS], o_atoms = 0;
  size_t ws_stage = 0, ws_keep = 0, ws_pos = 0, ws_srule = 0, ws_swork = 0, ws_bsum = 0;
  size_t ws_pending = 0, ws_npend = 0, ws_bsr = 0;
  long long nscan_blocks = 0;
  size_t ws_bytes = 0;
};

extern "C" {

int fe_version(void) { return 100; }

const char* fe_last_error(void) { return g_err.c_str(); }

int fe_status(unsigned* bits, int clear) {
  FE_CUDA(cudaDeviceSynchronize());
  unsigned v = 0;
  FE_CUDA(cudaMemcpyFromSymbol(&v, fe_status_word, sizeof v));
  if (clear) {
    const unsigned z = 0;
    FE_CUDA(cudaMemcpyToSymbol(fe_status_word, &z, sizeof z));
  }
  if (bits) *bits = v;
  return FE_OK;
}

int fe_plan_create(const fe_basis* b, fe_plan** out) {
  if (!b || !out) return fail(FE_ERR_ARG, "fe_plan_create: null argument");
  *out = nullptr;
  if (b->n_func < 0 || b->n_prim < 0 || b->n_atoms < 0)
    return fail(FE_ERR_ARG, "fe_plan_create: negative size");
  auto* p = new fe_plan();
  p->n_func = b->n_func;
  p->n_atoms = b->n_atoms;
  p->Z.assign(b->Z, b->Z + b->n_atoms);
  p->xyz.assign(b->xyz, b->xyz + 3 * size_t(b->n_atoms));
  // shells = contiguous runs of equal fn_shell (build_pairs.cpp:170-182)
  for (int i = 0; i < b->n_func;) {
    int j = i;
    while (j < b->n_func && b->fn_shell[j] == b->fn_shell[i]) ++j;
    FeShell s{};
    s.atom = b->fn_atom[i];
    s.l = b->fn_lx[i] + b->fn_ly[i] + b->fn_lz[i];
    s.fn0 = i;
    s.nprim = b->fn_nprim[i];
    const int nc = (s.l + 1) * (s.l + 2) / 2;
    if (s.l > 4) {
      const int rc = fail(FE_ERR_UNSUPPORTED, "shell %zu has l=%d > 4", p->shells.size(), s.l);
      delete p;
      return rc;
    }
    if (j - i != nc) {
      delete p;
      return fail(FE_ERR_ARG, "shell at function %d has %d functions, expected %d", i, j - i, nc);
    }
    if (s.nprim <= 0 || s.nprim > 65535 || b->fn_off[i] < 0 || b->fn_off[i] + s.nprim > b->n_prim) {
      delete p; return fail(FE_ERR_ARG, "shell at function %d: bad primitive range", i);
    }
    if (s.atom < 0 || s.atom >= b->n_atoms) { delete p; return fail(FE_ERR_ARG, "function %d: atom out of range", i); }
    s.prim0 = int(p->sexp.size());
    for (int k = 0; k < s.nprim; ++k) {
      p->sexp.push_back(b->pexp[b->fn_off[i] + k]);
      p->scoef.push_back(b->pcoef[b->fn_off[i] + k]);
    }
    for (int k = 0; k < 3; ++k) s.c[k] = b->fc[3 * size_t(i) + k];
    p->shells.push_back(s);
    i = j;
  }
  const int ns = int(p->shells.size());
  // shell pairs in reference order, class slot numbering per class
  long long cls_count[FE_NCLASS] = {};
  std::vector<std::vector<int>> grp_tasks(25);
  for (int si = 0; si < ns; ++si)
    for (int sj = si; sj < ns; ++sj) {
      const FeShell& A = p->shells[si];
      const FeShell& B = p->shells[sj];
      const int L = A.l + B.l;
      FeTask t{};
      t.si = si;
      t.sj = sj;
      t.slot0 = int(cls_count[L]);
      cls_count[L] += (long long)A.nprim * B.nprim;
      if (cls_count[L] > (1LL << 30)) { delete p; return fail(FE_ERR_SIZE, "class %d too large", L); }
      grp_tasks[A.l * 5 + B.l].push_back(int(p->tasks.size()));
      p->tasks.push_back(t);
    }
  p->class_slot0.assign(FE_NCLASS + 1, 0);
  p->stage_off.assign(FE_NCLASS, 0);
  long long so = 0;
  for (int L = 0; L < FE_NCLASS; ++L) {
    p->class_slot0[L + 1] = p->class_slot0[L] + cls_count[L];
    p->cap[L] = int(cls_count[L]);
    p->stage_off[L] = so;
    so += cls_count[L] * fe_class_rec64[L];
  }
  p->nslot = p->class_slot0[FE_NCLASS];
  // groups heaviest first (the per-pair work grows steeply with la + lb), so the
  // long-running blocks start in the first wave and light ones fill the tail
  std::array<int, 25> order{};
  for (int c = 0; c < 25; ++c) order[c] = c;
  auto cost = [](int code) {
    const int la = code / 5, lb = code % 5, L = la + lb;
    return (la + 1) * (la + 2) * (lb + 1) * (lb + 2) * (L + 1) * (L + 1) * (L + 1);
  };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
  int block = 0;
  for (int code : order) {
    if (grp_tasks[code].empty()) continue;
    const int w0 = int(p->work_task.size());
    for (int ti : grp_tasks[code]) {
      const FeTask& t = p->tasks[ti];
      const int na = p->shells[t.si].nprim, nb = p->shells[t.sj].nprim;
      for (int i = 0; i < na; ++i)
        for (int j = 0; j < nb; ++j) {
          p->work_task.push_back(ti);
          p->work_ij.push_back((i << 16) | j);
        }
    }
    const int nw = int(p->work_task.size()) - w0;
    if (nw == 0) continue;
    p->grp_code.push_back(code);
    p->grp_work0.push_back(w0);
    p->grp_nwork.push_back(nw);
    block += (nw + FE_BUILD_THREADS - 1) / FE_BUILD_THREADS;
  }
  p->nblocks = block;
  // device plan blob
  size_t o = 0;
  auto put = [&](size_t bytes) { const size_t at = o; o = align256(o + bytes); return at; };
  p->o_shells = put(sizeof(FeShell) * p->shells.size());
  p->o_sexp = put(sizeof(double) * p->sexp.size());
  p->o_scoef = put(sizeof(double) * p->scoef.size());
  p->o_tasks = put(sizeof(FeTask) * p->tasks.size());
  p->o_wt = put(sizeof(int) * p->work_task.size());
  p->o_wij = put(sizeof(int) * p->work_ij.size());
  p->o_cs = put(sizeof(long long) * p->class_slot0.size());
  p->o_so = put(sizeof(long long) * p->stage_off.size());
  p->plan_bytes = std::max<size_t>(o, 256);
  // table layout
  {
    const Layout lay = table_layout(p->cap, p->n_atoms);
    for (int L = 0; L < FE_NCLASS; ++L) {
      p->o_tab64[L] = lay.off64[L];
      p->o_tab32[L] = lay.off32[L];
    }
    p->o_atoms = lay.off_atoms;
    p->table_bytes = lay.bytes;
  }
  // build workspace
  size_t w = 0;
  auto wput = [&](size_t bytes) { const size_t at = w; w = align256(w + bytes); return at; };
  p->ws_stage = wput(size_t(so) * sizeof(double));
  p->ws_keep = wput(size_t(p->nslot + 1) * sizeof(int));
  p->ws_pos = wput(size_t(p->nslot + 1) * sizeof(int));
  p->ws_srule = wput(size_t(p->nslot + 1) * sizeof(double));
  p->ws_swork = wput(size_t(p->nslot + 1) * sizeof(int));
  p->ws_pending = wput(size_t(p->nslot + 1) * sizeof(int));
  p->ws_npend = wput(sizeof(int));
  p->nscan_blocks = (p->nslot + FE_SCAN_BLOCK - 1) / FE_SCAN_BLOCK;
  p->ws_bsum = wput(size_t(p->nscan_blocks + 1) * sizeof(int));
  p->ws_bsr = wput(size_t(p->nscan_blocks + 1) * sizeof(double));
  p->ws_bytes = std::max<size_t>(w, 256);
  *out = p;
  return FE_OK;
}

void fe_plan_destroy(fe_plan* plan) { delete plan; }

int fe_plan_sizes(const fe_plan* p, fe_sizes* s) {
  if (!p || !s) return fail(FE_ERR_ARG, "fe_plan_sizes: null argument");
  s->plan_bytes = p->plan_bytes;
  s->table_bytes = p->table_bytes;
  s->build_ws_bytes = p->ws_bytes;
  s->n_shell = int(p->shells.size());
  s->n_shell_pair = int(p->tasks.size());
  s->n_work = int(p->work_task.size());
  for (int L = 0; L < FE_NCLASS; ++L) s->cap[L] = p->cap[L];
  return FE_OK;
}

int fe_plan_upload(const fe_plan* p, void* d_plan, cudaStream_t st) {
  if (!p || !d_plan) return fail(FE_ERR_ARG, "fe_plan_upload: null argument");
  if (reinterpret_cast<uintptr_t>(d_plan) & 255) return fail(FE_ERR_ARG, "fe_plan_upload: buffer not 256-byte aligned");
  std::vector<unsigned char> h(p->plan_bytes, 0);
  auto cp = [&](size_t off, const void* src, size_t bytes) { if (bytes) memcpy(h.data() + off, src, bytes); };
  cp(p->o_shells, p->shells.data(), sizeof(FeShell) * p->shells.size());
  cp(p->o_sexp, p->sexp.data(), sizeof(double) * p->sexp.size());
  cp(p->o_scoef, p->scoef.data(), sizeof(double) * p->scoef.size());
  cp(p->o_tasks, p->tasks.data(), sizeof(FeTask) * p->tasks.size());
  cp(p->o_wt, p->work_task.data(), sizeof(int) * p->work_task.size());
  cp(p->o_wij, p->work_ij.data(), sizeof(int) * p->work_ij.size());
  cp(p->o_cs, p->class_slot0.data(), sizeof(long long) * p->class_slot0.size());
  cp(p->o_so, p->stage_off.data(), sizeof(long long) * p->stage_off.size());
  FE_CUDA(cudaMemcpyAsync(d_plan, h.data(), h.size(), cudaMemcpyHostToDevice, st));
  FE_CUDA(cudaStreamSynchronize(st));   // h is a local buffer
  return FE_OK;
}

namespace {
// Per-point part of the build workspace, after the plan's part: point-block
// boxes, superboxes, the spatially sorted screen points, their cells, the
// cell counters (FE_SORT_CELLS + 1) and the points' bounding box.
struct ScreenWs {
  size_t box, sbox, sorted, sortedf, cell, count, bb, bytes;
};
ScreenWs screen_ws(size_t base, int n_pts) {
  const size_t nbox = (size_t(n_pts) + 31) / 32, nsbox = (nbox + 31) / 32;
  ScreenWs w{};
  size_t o = base;
  auto put = [&](size_t bytes) { const size_t at = o; o += align256(bytes); return at; };
  w.box = put(nbox * 6 * sizeof(double));
  w.sbox = put(nsbox * 6 * sizeof(double));
  w.sorted = put(size_t(n_pts) * 3 * sizeof(double));
  w.sortedf = put(size_t(n_pts) * sizeof(float4));
  w.cell = put(size_t(n_pts) * sizeof(int));
  w.count = put((FE_SORT_CELLS + 1) * sizeof(int));
  w.bb = put(6 * (FE_BBOX_BLOCKS + 1) * sizeof(double));     // partials, then the whole box
  w.bytes = o;
  return w;
}
}  // namespace

size_t fe_build_ws_bytes(const fe_plan* p, int n_pts) {
  if (!p || n_pts < 0) return 0;
  return screen_ws(p->ws_bytes, n_pts).bytes;
}

int fe_table_build(const fe_plan* p, const void* d_plan, const double* d_dens,
                   const double* d_pts, int n_pts, double tol, int rule, void* d_table,
                   void* d_ws, size_t ws_bytes, cudaStream_t st) {
  if (!p || !d_plan || !d_table || !d_ws || (p->n_func && !d_dens))
    return fail(FE_ERR_ARG, "fe_table_build: null argument");
  if (n_pts < 0 || (n_pts > 0 && !d_pts)) return fail(FE_ERR_ARG, "fe_table_build: bad points");
  if (rule != FE_RULE_NUMPY && rule != FE_RULE_NATIVE) return fail(FE_ERR_ARG, "fe_table_build: unknown rule %d", rule);
  if (!(tol >= 0.0)) return fail(FE_ERR_ARG, "fe_table_build: tol must be >= 0");
  const size_t need = fe_build_ws_bytes(p, n_pts);
  if (ws_bytes < need) return fail(FE_ERR_SIZE, "fe_table_build: workspace %zu < %zu bytes (fe_build_ws_bytes)", ws_bytes, need);
  if ((reinterpret_cast<uintptr_t>(d_table) | reinterpret_cast<uintptr_t>(d_ws) |
       reinterpret_cast<uintptr_t>(d_plan)) & 255)
    return fail(FE_ERR_ARG, "fe_table_build: buffers must be 256-byte aligned");
  const unsigned char* pb = static_cast<const unsigned char*>(d_plan);
  unsigned char* wb = static_cast<unsigned char*>(d_ws);
  unsigned char* tb = static_cast<unsigned char*>(d_table);
  {
    const int rc = write_header(tb, p->cap, p->n_atoms, p->Z.data(), p->xyz.data(), tol, rule, st);
    if (rc != FE_OK) return rc;
  }
  FeBuildArgs a{};
  a.shells = reinterpret_cast<const FeShell*>(pb + p->o_shells);
  a.sexp = reinterpret_cast<const double*>(pb + p->o_sexp);
  a.scoef = reinterpret_cast<const double*>(pb + p->o_scoef);
  a.tasks = reinterpret_cast<const FeTask*>(pb + p->o_tasks);
  a.work_task = reinterpret_cast<const int*>(pb + p->o_wt);
  a.work_ij = reinterpret_cast<const int*>(pb + p->o_wij);
  a.n_func = p->n_func;
  a.dens = d_dens;
  a.pts = d_pts;
  a.npts = n_pts;
  a.tol = tol;
  a.rule = rule;
  a.class_slot0 = reinterpret_cast<const long long*>(pb + p->o_cs);
  a.stage = reinterpret_cast<double*>(wb + p->ws_stage);
  a.stage_off = reinterpret_cast<const long long*>(pb + p->o_so);
  a.keep = reinterpret_cast<int*>(wb + p->ws_keep);
  a.srule = reinterpret_cast<double*>(wb + p->ws_srule);
  a.swork = reinterpret_cast<int*>(wb + p->ws_swork);
  a.pending = reinterpret_cast<int*>(wb + p->ws_pending);
  a.npending = reinterpret_cast<int*>(wb + p->ws_npend);
  a.nbox = (n_pts + 31) / 32;
  a.nsbox = (a.nbox + 31) / 32;
  const ScreenWs pw = screen_ws(p->ws_bytes, n_pts);
  double* box = reinterpret_cast<double*>(wb + pw.box);
  double* sbox = reinterpret_cast<double*>(wb + pw.sbox);
  a.box = box;
  a.sbox = sbox;
  if (a.nbox > 0) {
    // the screen's points bucketed by Morton cell, so that its boxes are compact
    double* sorted = reinterpret_cast<double*>(wb + pw.sorted);
    int* cell = reinterpret_cast<int*>(wb + pw.cell);
    int* count = reinterpret_cast<int*>(wb + pw.count);
    double* bb = reinterpret_cast<double*>(wb + pw.bb);
    FE_CUDA(cudaMemsetAsync(count, 0, (FE_SORT_CELLS + 1) * sizeof(int), st));
    fe_points_bbox_kernel<<<FE_BBOX_BLOCKS, 256, 0, st>>>(d_pts, n_pts, bb);
    fe_points_count_kernel<4><<<(n_pts + 255) / 256, 256, 0, st>>>(d_pts, n_pts, bb, cell, count);
    fe_scan_top_kernel<<<1, FE_SCAN_BLOCK, 0, st>>>(count, FE_SORT_CELLS);
    float4* sortedf = reinterpret_cast<float4*>(wb + pw.sortedf);
    fe_points_place_kernel<<<(n_pts + 255) / 256, 256, 0, st>>>(d_pts, n_pts, cell, count, sorted,
                                                                sortedf);
    FE_CUDA(cudaGetLastError());
    a.pts = sorted;
    a.ptsf = sortedf;
    a.pbox = bb + 6 * FE_BBOX_BLOCKS;
    // one warp per box and per superbox
    fe_point_boxes_kernel<<<(a.nbox + 3) / 4, 128, 0, st>>>(sorted, n_pts, box, a.nbox);
    fe_super_boxes_kernel<<<(a.nsbox + 3) / 4, 128, 0, st>>>(box, a.nbox, sbox, a.nsbox);
    FE_CUDA(cudaGetLastError());
  }
  FE_CUDA(cudaMemsetAsync(a.npending, 0, sizeof(int), st));
  if (p->nblocks > 0) {
    // the (la, lb) groups side by side, heaviest first: the thread-per-pair
    // groups, then the pairs their threads left undecided (one warp each),
    // while the warp-per-pair groups (which leave none) run beside them
    std::vector<int> tg, wg;
    for (int g = 0; g < int(p->grp_code.size()); ++g)
      (fe_warp_pair_group(p->grp_code[g] / 5, p->grp_code[g] % 5) ? wg : tg).push_back(g);
    auto group = [&](int g, cudaStream_t sg) {
      const FeBuildKernel k = fe_build_kernel_for(p->grp_code[g]);
      if (!k) return fail(FE_ERR_ARG, "table build: bad group code %d", p->grp_code[g]);
      const int nw = p->grp_nwork[g], per = fe_build_pairs_per_block(p->grp_code[g]);
      k<<<unsigned((nw + per - 1) / per), fe_build_block_threads(p->grp_code[g]), 0, sg>>>(
          a, p->grp_work0[g], nw);
      FE_CUDA(cudaGetLastError());
      return FE_OK;
    };
    const int rc = fork_join2(
        int(tg.size()), int(wg.size()), st, [&](int i, cudaStream_t sg) { return group(tg[i], sg); },
        [&](cudaStream_t s0) {
          fe_screen_pending_kernel<<<sm_count() * 8, 128, 0, s0>>>(a);
          FE_CUDA(cudaGetLastError());
          return FE_OK;
        },
        [&](int i, cudaStream_t sg) { return group(wg[i], sg); });
    if (rc != FE_OK) return rc;
  }
  int* pos = reinterpret_cast<int*>(wb + p->ws_pos);
  double* bsr = reinterpret_cast<double*>(wb + p->ws_bsr);
  if (p->nslot > 0) {
    int* bsum = reinterpret_cast<int*>(wb + p->ws_bsum);
    const unsigned nb = unsigned(p->nscan_blocks);
    // the per-block keep counts, and the per-block sums of the sum-rule terms
    fe_scan_sums_kernel<<<nb, FE_SCAN_BLOCK, 0, st>>>(a.keep, p->nslot, bsum, a.srule, bsr);
    fe_scan_top_kernel<<<1, FE_SCAN_BLOCK, 0, st>>>(bsum, int(nb));
    fe_scan_apply_kernel<<<nb, FE_SCAN_BLOCK, 0, st>>>(a.keep, p->nslot, bsum, pos);
    FE_CUDA(cudaGetLastError());
    // per class, side by side: the kept records to their rows, then their FP32
    // records
    std::vector<int> cls;
    for (int L = 0; L < FE_NCLASS; ++L)
      if (p->class_slot0[L + 1] > p->class_slot0[L]) cls.push_back(L);
    const int rc = fork_join(int(cls.size()), st, [&](int i, cudaStream_t sg) {
      const int L = cls[i];
      const long long c0 = p->class_slot0[L], n = p->class_slot0[L + 1] - c0;
      const int tile = fe_records_tile_of(L);
      return launch_records(L, a.stage + p->stage_off[L], a.keep + c0, pos + c0, a.swork + c0,
                            int(n), tb, unsigned((n + tile - 1) / tile), sg);
    });
    if (rc != FE_OK) return rc;
  }
  fe_finalize_kernel<<<1, 1024, 0, st>>>(a.class_slot0, FE_NCLASS, p->nslot, a.keep, pos, bsr,
                                         a.npending, tb, float(kTauDefault));
  FE_CUDA(cudaGetLastError());
  return FE_OK;
}

size_t fe_table_bytes(const int* cap, int n_atoms) {
  if (!cap || n_atoms < 0) return 0;
  for (int L = 0; L < FE_NCLASS; ++L)
    if (cap[L] < 0) return 0;
  return table_layout(cap, n_atoms).bytes;
}

int fe_table_offsets(const int* cap, int n_atoms, size_t* off64, size_t* off32, size_t* off_atoms) {
  if (!cap || n_atoms < 0) return fail(FE_ERR_ARG, "fe_table_offsets: bad argument");
  const Layout lay = table_layout(cap, n_atoms);
  for (int L = 0; L < FE_NCLASS; ++L) {
    if (off64) off64[L] = lay.off64[L];
    if (off32) off32[L] = lay.off32[L];
  }
  if (off_atoms) *off_atoms = lay.off_atoms;
  return FE_OK;
}

int fe_table_init(void* d_table, const int* count, int n_atoms, const double* Z,
                  const double* xyz, cudaStream_t st) {
  if (!d_table || !count || n_atoms < 0 || (n_atoms > 0 && (!Z || !xyz)))
    return fail(FE_ERR_ARG, "fe_table_init: bad argument");
  if (reinterpret_cast<uintptr_t>(d_table) & 255) return fail(FE_ERR_ARG, "fe_table_init: buffer not 256-byte aligned");
  unsigned char* tb = static_cast<unsigned char*>(d_table);
  const int rc = write_header(tb, count, n_atoms, Z, xyz, 0.0, -1, st);
  if (rc != FE_OK) return rc;
  // counts equal capacities for an imported table
  FE_CUDA(cudaMemcpyAsync(tb + offsetof(FeTableHdr, count), count, sizeof(int) * FE_NCLASS,
                          cudaMemcpyHostToDevice, st));
  FE_CUDA(cudaStreamSynchronize(st));
  return FE_OK;
}

int fe_table_make_f32(void* d_table, cudaStream_t st) {
  if (!d_table) return fail(FE_ERR_ARG, "fe_table_make_f32: null table");
  // every class (the counts are in the device header): a grid-stride loop of
  // two blocks per SM over the class's tiles
  for (int L = 0; L < FE_NCLASS; ++L) {
    const int rc = launch_records(L, nullptr, nullptr, nullptr, nullptr, 0,
                                  static_cast<unsigned char*>(d_table), unsigned(2 * sm_count()), st);
    if (rc != FE_OK) return rc;
  }
  return FE_OK;
}

int fe_table_info_get(const void* d_table, fe_table_info* info, cudaStream_t st) {
  if (!d_table || !info) return fail(FE_ERR_ARG, "fe_table_info_get: null argument");
  FeTableHdr h{};
  FE_CUDA(cudaMemcpyAsync(&h, d_table, sizeof h, cudaMemcpyDeviceToHost, st));
  FE_CUDA(cudaStreamSynchronize(st));
  if (h.magic != FE_TABLE_MAGIC) return fail(FE_ERR_ARG, "fe_table_info_get: not a pair table");
  info->n_pairs = 0;
  for (int L = 0; L < FE_NCLASS; ++L) {
    info->count[L] = h.count[L];
    info->n_pairs += h.count[L];
  }
  info->n_atoms = h.n_atoms;
  info->sum_rule = h.sum_rule;
  info->tol = h.tol;
  info->rule = h.rule;
  info->has_f32 = h.has32;
  info->n_warp_screen = h.n_warp_screen;
  return FE_OK;
}

}  // extern "C"

namespace {

// Workspace section of the spatial point order (after the partial rows):
// the points in evaluation order, each one's caller row, the cells, the
// points grouped by cell, the per-cell starts and ends, the bounding boxes.
struct OrderWs {
  size_t pts, perm, cell, idx, start, end, bb, bytes;
};
OrderWs order_ws(int n) {
  OrderWs w{};
  size_t o = 0;
  auto put = [&](size_t b) { const size_t at = o; o = align256(o + b); return at; };
  w.pts = put(size_t(n) * 3 * sizeof(double));
  w.perm = put(size_t(n) * sizeof(int));
  w.cell = put(size_t(n) * sizeof(int));
  w.idx = put(size_t(n) * sizeof(int));
  w.start = put((FE_ORDER_CELLS + 1) * sizeof(int));
  w.end = put((FE_ORDER_CELLS + 1) * sizeof(int));
  w.bb = put(6 * (FE_BBOX_BLOCKS + 1) * sizeof(double));    // partials, then the whole box
  w.bytes = o;
  return w;
}

// The points of d_pts in evaluation order into the section at ``ob``.
int order_points(const double* d_pts, int n, unsigned char* ob, const OrderWs& w, cudaStream_t st) {
  int* cell = reinterpret_cast<int*>(ob + w.cell);
  int* start = reinterpret_cast<int*>(ob + w.start);
  int* end = reinterpret_cast<int*>(ob + w.end);
  double* bb = reinterpret_cast<double*>(ob + w.bb);
  FE_CUDA(cudaMemsetAsync(start, 0, (FE_ORDER_CELLS + 1) * sizeof(int), st));
  fe_points_bbox_kernel<<<FE_BBOX_BLOCKS, 256, 0, st>>>(d_pts, n, bb);
  fe_points_count_kernel<FE_ORDER_BITS><<<(n + 255) / 256, 256, 0, st>>>(d_pts, n, bb, cell, start);
  fe_scan_top_kernel<<<1, FE_SCAN_BLOCK, 0, st>>>(start, FE_ORDER_CELLS);
  FE_CUDA(cudaGetLastError());
  FE_CUDA(cudaMemcpyAsync(end, start, FE_ORDER_CELLS * sizeof(int), cudaMemcpyDeviceToDevice, st));
  fe_order_place_kernel<<<(n + 255) / 256, 256, 0, st>>>(cell, n, end,
                                                         reinterpret_cast<int*>(ob + w.idx));
  fe_order_rank_kernel<<<(n + 255) / 256, 256, 0, st>>>(
      d_pts, n, cell, start, end, reinterpret_cast<const int*>(ob + w.idx),
      reinterpret_cast<double*>(ob + w.pts), reinterpret_cast<int*>(ob + w.perm));
  FE_CUDA(cudaGetLastError());
  return FE_OK;
}

}  // namespace

extern "C" {

size_t fe_eval_ws_bytes(int n_pts) {
  if (n_pts <= 0) return 256;
  const EvalGeom g = eval_geom(n_pts, 0);
  return align256(g.ws_rows() * g.ld * sizeof(double));
}

size_t fe_eval_ws_bytes_mixed(int n_pts, const int* cap) {
  if (n_pts <= 0) return 256;
  const EvalGeom g = eval_geom(n_pts, 1);
  long long words = 0;
  for (int L = 0; L < FE_NCLASS; ++L) words += cap ? (std::max(cap[L], 0) + 31) / 32 : 0;
  const long long warps = (long long)g.nblk_x * (FE_MX_NT / 32);
  return align256(g.ws_rows() * g.ld * sizeof(double)) + order_ws(n_pts).bytes +
         align256(size_t(warps * words) * 4);
}

size_t fe_point_order_bytes(int n_pts) { return n_pts > 0 ? order_ws(n_pts).bytes : 0; }

}  // extern "C"

namespace {

int eval_launch(const char* who, const void* d_table, const double* d_pts, int n_pts,
                double* d_out, void* d_ws, size_t ws_bytes, int out_mode, int prec,
                double tau, unsigned long long* d_n64, cudaStream_t st, int lmin = 0,
                int lmax = FE_NCLASS - 1) {
  if (n_pts < 0) return fail(FE_ERR_ARG, "%s: n_pts < 0", who);
  if (n_pts == 0) return FE_OK;
  if (!d_table || !d_pts || !d_out) return fail(FE_ERR_ARG, "%s: null argument", who);
  const EvalGeom g = eval_geom(n_pts, prec);
  const size_t rows_bytes = align256(g.ws_rows() * g.ld * sizeof(double));
  if (!d_ws || ws_bytes < rows_bytes)
    return fail(FE_ERR_SIZE, "%s: workspace too small (need at least %zu bytes)", who, rows_bytes);
  // the points in spatial order when the workspace has room for it (after the
  // rows); the mixed path's routing mask takes what follows
  size_t used = rows_bytes;
  const int* perm = nullptr;
  const OrderWs ow = order_ws(n_pts);
  if (ws_bytes >= rows_bytes + ow.bytes + (prec ? 4 : 0)) {
    unsigned char* ob = static_cast<unsigned char*>(d_ws) + rows_bytes;
    const int rc = order_points(d_pts, n_pts, ob, ow, st);
    if (rc != FE_OK) return rc;
    d_pts = reinterpret_cast<const double*>(ob + ow.pts);
    perm = reinterpret_cast<const int*>(ob + ow.perm);
    used += ow.bytes;
  }
  const int smem = FE_NSTAGE * FE_STAGE_BYTES;
  double* rows = static_cast<double*>(d_ws);
  auto next_rows = [&](int k) {
    double* r = rows;
    rows += size_t(g.split[k]) * g.ld;
    return r;
  };
  const unsigned char* tb = static_cast<const unsigned char*>(d_table);
  if (prec == 0) {
    FeEvalArgs a{};
    a.table = tb;
    a.pts = d_pts;
    a.npts = n_pts;
    a.ld = g.ld;
    a.lmin = lmin;
    a.lmax = lmax;
    auto k0 = fe_eval_f64_kernel<kNP64, kEvalThreads, kMinB64, 0, FE_LSPLIT>;
    auto k1 = fe_eval_f64_kernel<kNP64, kEvalThreads, 1, FE_LSPLIT + 1, FE_NCLASS - 1>;
    a.nsplit = g.split[0];
    a.partial = next_rows(0);
    FE_CUDA(cudaFuncSetAttribute(k0, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k0<<<dim3(g.nblk_x, g.split[0]), kEvalThreads, smem, st>>>(a);
    FE_CUDA(cudaGetLastError());
    a.nsplit = g.split[1];
    a.partial = next_rows(1);
    FE_CUDA(cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k1<<<dim3(g.nblk_x, g.split[1]), kEvalThreads, smem, st>>>(a);
  } else {
    if (ws_bytes - used < 4)
      return fail(FE_ERR_SIZE, "%s: workspace has no room for the routing mask (size it with "
                  "fe_eval_ws_bytes_mixed)", who);
    FeMixedArgs a{};
    a.table = tb;
    a.pts = d_pts;
    a.npts = n_pts;
    a.ld = g.ld;
    a.tau = float(tau);
    a.n64 = d_n64;
    a.mask = reinterpret_cast<unsigned*>(static_cast<unsigned char*>(d_ws) + used);
    a.mask_words = static_cast<long long>((ws_bytes - used) / 4);
    a.lmin = lmin;
    a.lmax = lmax;
    auto f0 = fe_eval_f32_kernel<kMinB32Lo, 0, FE_MXSPLIT>;
    auto f0b = fe_eval_f32_kernel<kMinB32, FE_MXSPLIT + 1, FE_LSPLIT>;
    auto f1 = fe_eval_f32_kernel<1, FE_LSPLIT + 1, FE_NCLASS - 1>;
    auto x0 = fe_eval_fix64_kernel<kMinBFix, 0, FE_LSPLIT>;
    auto x1 = fe_eval_fix64_kernel<1, FE_LSPLIT + 1, FE_NCLASS - 1>;
    const void* ks[5] = {(const void*)f0, (const void*)f0b, (const void*)f1, (const void*)x0,
                         (const void*)x1};
    for (int k = 0; k < 5; ++k) {
      a.nsplit = g.split[k];
      a.partial = next_rows(k);
      const int dyn = k < 3 ? smem : 0;      // the FP64 part uses static buffers only
      if (dyn) FE_CUDA(cudaFuncSetAttribute(ks[k], cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
      void* args[] = {&a};
      FE_CUDA(cudaLaunchKernel(ks[k], dim3(g.nblk_x, g.split[k]), dim3(FE_MX_NT), args, dyn, st));
    }
  }
  FE_CUDA(cudaGetLastError());
  fe_reduce_kernel<<<(n_pts + 255) / 256, 256, 0, st>>>(tb, d_pts, n_pts, static_cast<double*>(d_ws),
                                                        int(g.ws_rows()), g.ld, d_out, out_mode,
                                                        perm);
  FE_CUDA(cudaGetLastError());
  return FE_OK;
}

}  // namespace

extern "C" {

int fe_esp_fp64(const void* d_table, const double* d_pts, int n_pts, double* d_out,
                void* d_ws, size_t ws_bytes, cudaStream_t st) {
  return eval_launch("fe_esp_fp64", d_table, d_pts, n_pts, d_out, d_ws, ws_bytes, 0, 0, 0.0,
                     nullptr, st);
}

int fe_electron_fp64(const void* d_table, const double* d_pts, int n_pts, double* d_out,
                     void* d_ws, size_t ws_bytes, cudaStream_t st) {
  return eval_launch("fe_electron_fp64", d_table, d_pts, n_pts, d_out, d_ws, ws_bytes, 1, 0, 0.0,
                     nullptr, st);
}

int fe_esp_mixed(const void* d_table, const double* d_pts, int n_pts, double* d_out,
                 void* d_ws, size_t ws_bytes, double tau, unsigned long long* d_n64,
                 cudaStream_t st) {
  if (!(tau > 0.0)) tau = kTauDefault;
  return eval_launch("fe_esp_mixed", d_table, d_pts, n_pts, d_out, d_ws, ws_bytes, 0, 1, tau,
                     d_n64, st);
}

int fe_electron_mixed(const void* d_table, const double* d_pts, int n_pts, double* d_out,
                      void* d_ws, size_t ws_bytes, double tau, unsigned long long* d_n64,
                      cudaStream_t st) {
  if (!(tau > 0.0)) tau = kTauDefault;
  return eval_launch("fe_electron_mixed", d_table, d_pts, n_pts, d_out, d_ws, ws_bytes, 1, 1, tau,
                     d_n64, st);
}

int fe_electron_classes(const void* d_table, const double* d_pts, int n_pts, double* d_out,
                        void* d_ws, size_t ws_bytes, int precision, double tau, int lmin,
                        int lmax, unsigned long long* d_n64, cudaStream_t st) {
  if (precision != 0 && precision != 1)
    return fail(FE_ERR_ARG, "fe_electron_classes: precision must be 0 (FP64) or 1 (mixed)");
  if (lmin < 0 || lmax >= FE_NCLASS || lmin > lmax)
    return fail(FE_ERR_ARG, "fe_electron_classes: class range %d..%d outside 0..%d", lmin, lmax,
                FE_NCLASS - 1);
  if (!(tau > 0.0)) tau = kTauDefault;
  return eval_launch("fe_electron_classes", d_table, d_pts, n_pts, d_out, d_ws, ws_bytes, 1,
                     precision, tau, d_n64, st, lmin, lmax);
}

int fe_nuclear_fp64(const void* d_table, const double* d_pts, int n_pts, double* d_out,
                    void* d_ws, size_t ws_bytes, cudaStream_t st) {
  (void)d_ws;
  (void)ws_bytes;
  if (n_pts < 0) return fail(FE_ERR_ARG, "fe_nuclear_fp64: n_pts < 0");
  if (n_pts == 0) return FE_OK;
  if (!d_table || !d_pts || !d_out) return fail(FE_ERR_ARG, "fe_nuclear_fp64: null argument");
  fe_nuclear_kernel<<<(n_pts + 255) / 256, 256, 0, st>>>(static_cast<const unsigned char*>(d_table),
                                                         d_pts, n_pts, d_out);
  FE_CUDA(cudaGetLastError());
  return FE_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Boys function kernel (tests and the boys() API)
// ---------------------------------------------------------------------------
template <int M>
__global__ void fe_boys_kernel(const double* __restrict__ T, int n, double* __restrict__ F) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double f[M + 1];
  fe_boys_f64<M>(T[i], f);
#pragma unroll
  for (int m = 0; m <= M; ++m) F[size_t(i) * (M + 1) + m] = f[m];
}

extern "C" int fe_boys_fp64(const double* d_T, int n, int mmax, double* d_F, cudaStream_t st) {
  if (n < 0 || !d_T || !d_F) return fail(FE_ERR_ARG, "fe_boys_fp64: bad argument");
  if (mmax < 0 || mmax > FE_MMAX) return fail(FE_ERR_UNSUPPORTED, "fe_boys_fp64: mmax %d outside 0..%d", mmax, FE_MMAX);
  if (n == 0) return FE_OK;
  const int blk = 128, grd = (n + blk - 1) / blk;
  switch (mmax) {
#define FE_B(m) case m: fe_boys_kernel<m><<<grd, blk, 0, st>>>(d_T, n, d_F); break;
    FE_B(0) FE_B(1) FE_B(2) FE_B(3) FE_B(4) FE_B(5) FE_B(6) FE_B(7) FE_B(8) FE_B(9)
#undef FE_B
  }
  FE_CUDA(cudaGetLastError());
  return FE_OK;
}

// ---------------------------------------------------------------------------
// FMA throughput probe: the FP64 / FP32 pipe peak used as the roofline
// denominator (8 independent FMA chains per thread, no memory traffic).  The
// packed form issues FP32x2 fused multiply-adds (two lanes per instruction),
// as the mixed evaluator does, so it needs half the issue slots of the scalar
// form for the same FMA-pipe work.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) fe_peak_kernel(long long iters, T* out) {
  T a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = T(threadIdx.x + k) * T(1e-6);
  const T b = T(0.9999999), c = T(1e-7);
#pragma unroll 4
  for (long long it = 0; it < iters; ++it)
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = fe_fma(a[k], b, c);
  T s = T(0);
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k];
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

__global__ void __launch_bounds__(256) fe_peak2_kernel(long long iters, float* out) {
  float2 a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = make_float2(float(threadIdx.x + k) * 1e-6f, float(k) * 1e-6f);
  const float2 b = fe_f2(0.9999999f), c = fe_f2(1e-7f);
#pragma unroll 4
  for (long long it = 0; it < iters; ++it)
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = fe_fma(a[k], b, c);
  float s = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k].x + a[k].y;
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

extern "C" int fe_peak_run(int kind, long long iters, int blocks, void* d_out, cudaStream_t st) {
  if (iters <= 0 || blocks <= 0 || !d_out || kind < 0 || kind > 2)
    return fail(FE_ERR_ARG, "fe_peak_run: bad argument");
  if (kind == 1)
    fe_peak_kernel<double><<<blocks, 256, 0, st>>>(iters, static_cast<double*>(d_out));
  else if (kind == 0)
    fe_peak_kernel<float><<<blocks, 256, 0, st>>>(iters, static_cast<float*>(d_out));
  else
    fe_peak2_kernel<<<blocks, 256, 0, st>>>(iters, static_cast<float*>(d_out));
  FE_CUDA(cudaGetLastError());
  return FE_OK;
}

// ---------------------------------------------------------------------------
// Self-test of the bounded-wait path: one thread waits on an mbarrier that no
// thread arrives on and no copy targets, so the wait must give up after
// ``cycles`` SM clocks, flag FE_ST_TIMEOUT and let the kernel return.
// ---------------------------------------------------------------------------
__global__ void fe_wait_selftest_kernel(long long cycles, int* done) {
  __shared__ uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  mbar_fence_init();
  const bool got = mbar_wait_limited(&bar, 0, cycles);
  *done = got ? 1 : 2;
}

extern "C" int fe_wait_selftest(long long cycles, int* d_done, cudaStream_t st) {
  if (cycles <= 0 || cycles > 4000000000LL || !d_done)
    return fail(FE_ERR_ARG, "fe_wait_selftest: cycles must be in 1..4e9 and d_done non-null");
  fe_wait_selftest_kernel<<<1, 32, 0, st>>>(cycles, d_done);
  FE_CUDA(cudaGetLastError());
  FE_CUDA(cudaStreamSynchronize(st));
  unsigned v = 0;
  FE_CUDA(cudaMemcpyFromSymbol(&v, fe_status_word, sizeof v));
  if (v & FE_ST_TIMEOUT)
    return fail(FE_ERR_DEVICE, "fe_wait_selftest: device status 0x%x (a bounded wait gave up)", v);
  return FE_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free FP64 evaluation.
//
// Some callers cannot allocate device memory: a host application or plugin
// framework that owns the whole device-memory budget and only lends the
// library its input and output buffers, or a binding of the reference's own
// two-buffer interface (pair table and points in, potentials out), which has
// no notion of a workspace.  fe_esp_fp64_noalloc serves them: its partial-sum
// workspace is this file-scope device array instead of a caller buffer.  The
// array is FE_NOALLOC_SCRATCH_BYTES on every GPU that loads the library and
// stays allocated until the process exits.
// ---------------------------------------------------------------------------
#define FE_NOALLOC_SCRATCH_BYTES (16u << 20)
#define FE_NOALLOC_MAX_DEVICES 128

static __device__ __align__(256) unsigned char fe_noalloc_scratch[FE_NOALLOC_SCRATCH_BYTES];

namespace {
// Device address of the scratch array, per device, with the ID of the context
// it was resolved in.  The host-side symbol is only a stand-in, never a device
// address, so the address comes from cudaGetSymbolAddress once per device; a
// device reset replaces the device's context (and may move the array), which
// the context ID shows, and the address is then resolved again.
struct NoallocSlot {
  void* ptr = nullptr;
  unsigned long long ctx_id = 0;
};
std::mutex g_noalloc_mu;
NoallocSlot g_noalloc[FE_NOALLOC_MAX_DEVICES];

// The scratch array's device address on the current device.
int noalloc_scratch(void** out) {
  int dev = 0;
  FE_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= FE_NOALLOC_MAX_DEVICES)
    return fail(FE_ERR_UNSUPPORTED, "fe_esp_fp64_noalloc: device ordinal %d too large", dev);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoallocSlot& s = g_noalloc[dev];
  const unsigned long long id = current_ctx_id();
  if (!s.ptr || id == 0 || id != s.ctx_id) {
    void* p = nullptr;
    FE_CUDA(cudaGetSymbolAddress(&p, fe_noalloc_scratch));
    s.ptr = p;
    s.ctx_id = current_ctx_id();        // the lookup made the device's context current
  }
  *out = s.ptr;
  return FE_OK;
}
}  // namespace

extern "C" size_t fe_noalloc_scratch_bytes(void) { return FE_NOALLOC_SCRATCH_BYTES; }

extern "C" int fe_esp_fp64_noalloc(const void* d_table, const double* d_pts, int n_pts,
                                   double* d_out, cudaStream_t st) {
  if (n_pts < 0) return fail(FE_ERR_ARG, "fe_esp_fp64_noalloc: n_pts < 0");
  if (n_pts == 0) return FE_OK;
  if (!d_table || !d_pts || !d_out) return fail(FE_ERR_ARG, "fe_esp_fp64_noalloc: null argument");
  const size_t need = fe_eval_ws_bytes(n_pts);
  if (need > FE_NOALLOC_SCRATCH_BYTES)
    return fail(FE_ERR_SIZE,
                "fe_esp_fp64_noalloc: %d points need %zu bytes of scratch, more than the "
                "%u-byte static array; use fe_esp_fp64 with a caller workspace",
                n_pts, need, FE_NOALLOC_SCRATCH_BYTES);
  void* scratch = nullptr;
  const int rc = noalloc_scratch(&scratch);
  if (rc != FE_OK) return rc;
  return eval_launch("fe_esp_fp64_noalloc", d_table, d_pts, n_pts, d_out, scratch, need, 0, 0,
                     0.0, nullptr, st);
}

// ---------------------------------------------------------------------------
// Field and adjoint
// ---------------------------------------------------------------------------
#ifndef FE_NPFIELD
#define FE_NPFIELD 1
#endif
#ifndef FE_MINBFIELD
#define FE_MINBFIELD 2
#endif
namespace {

constexpr int kNPField = FE_NPFIELD, kMinBField = FE_MINBFIELD;

struct FieldGeom {
  int nblk_x, ld, split[2];
  size_t plane() const { return size_t(split[0] + split[1]) * ld; }
  size_t bytes() const { return align256(4 * plane() * sizeof(double)); }
};

FieldGeom field_geom(int npts) {
  FieldGeom g{};
  const int ppb = kEvalThreads * kNPField;
  g.nblk_x = (npts + ppb - 1) / ppb;
  const int target = 8 * kMinBField * sm_count();
  // at least one grid row per class of each instance's range (fe_class_rows)
  g.split[0] = std::max(FE_LSPLIT + 1,
                        std::min(256, (target + g.nblk_x - 1) / std::max(1, g.nblk_x)));
  g.split[1] = std::max(FE_NCLASS - 1 - FE_LSPLIT, std::min(8, sm_count() / std::max(1, g.nblk_x)));
  g.ld = (npts + 31) & ~31;
  return g;
}

int field_launch(const char* who, const unsigned char* tb, const double* d_pts, int n_pts,
                 const double* d_w, double* d_v, double* d_g, void* d_ws, size_t ws_bytes,
                 cudaStream_t st) {
  const FieldGeom g = field_geom(n_pts);
  if (!d_ws || ws_bytes < g.bytes())
    return fail(FE_ERR_SIZE, "%s: workspace too small (need at least %zu bytes)", who, g.bytes());
  const int smem = FE_NSTAGE * FE_STAGE_BYTES;
  FeFieldArgs a{};
  a.table = tb;
  a.pts = d_pts;
  a.npts = n_pts;
  a.ld = g.ld;
  a.plane = g.plane();
  auto k0 = fe_field_f64_kernel<kNPField, kEvalThreads, kMinBField, 0, FE_LSPLIT>;
  auto k1 = fe_field_f64_kernel<kNPField, kEvalThreads, 1, FE_LSPLIT + 1, FE_NCLASS - 1>;
  a.nsplit = g.split[0];
  a.partial = static_cast<double*>(d_ws);
  FE_CUDA(cudaFuncSetAttribute(k0, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  k0<<<dim3(g.nblk_x, g.split[0]), kEvalThreads, smem, st>>>(a);
  FE_CUDA(cudaGetLastError());
  a.nsplit = g.split[1];
  a.partial = static_cast<double*>(d_ws) + size_t(g.split[0]) * g.ld;
  FE_CUDA(cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  k1<<<dim3(g.nblk_x, g.split[1]), kEvalThreads, smem, st>>>(a);
  FE_CUDA(cudaGetLastError());
  fe_field_reduce_kernel<<<(n_pts + 255) / 256, 256, 0, st>>>(
      tb, d_pts, n_pts, static_cast<const double*>(d_ws), g.plane(), g.split[0] + g.split[1],
      g.ld, d_w, d_v, d_g);
  FE_CUDA(cudaGetLastError());
  return FE_OK;
}

struct AdjLayout {
  size_t field, mom, dw, first, last, bytes;
  long long mom_off[FE_NCLASS];
  long long nsrc;
  int dw_stride;
};

AdjLayout adj_layout(const fe_plan* p, int n_pts) {
  AdjLayout l{};
  size_t o = 0;
  auto put = [&](size_t bytes) { const size_t at = o; o = align256(o + bytes); return at; };
  l.field = put(n_pts > 0 ? field_geom(n_pts).bytes() : 0);
  long long nm = 0;
  l.nsrc = 0;
  for (int L = 0; L < FE_NCLASS; ++L) {
    l.mom_off[L] = nm;
    nm += (long long)p->cap[L] * fe_class_nterm[L];
    l.nsrc += p->cap[L];
  }
  l.mom = put(size_t(nm) * sizeof(double));
  int lmax = 0;
  for (const FeShell& s : p->shells) lmax = std::max(lmax, s.l);
  const int nc = (lmax + 1) * (lmax + 2) / 2;
  l.dw_stride = nc * nc;
  l.dw = put(size_t(l.nsrc) * l.dw_stride * sizeof(double));
  l.first = put(p->tasks.size() * sizeof(int));
  l.last = put(p->tasks.size() * sizeof(int));
  l.bytes = std::max<size_t>(o, 256);
  return l;
}

template <int L, int C>
int launch_moments(const FeAdjArgs& a, int cap, cudaStream_t st) {
  if constexpr (C < fe_mom_nchunk[L]) {
    if (cap > 0) fe_adj_moments_kernel<L, C><<<cap, FE_ADJ_THREADS, 0, st>>>(a);
    FE_CUDA(cudaGetLastError());
    return launch_moments<L, C + 1>(a, cap, st);
  } else {
    return FE_OK;
  }
}

}  // namespace

extern "C" {

size_t fe_field_ws_bytes(int n_pts) {
  if (n_pts <= 0) return 256;
  return field_geom(n_pts).bytes();
}

int fe_esp_field_fp64(const void* d_table, const double* d_pts, int n_pts, const double* d_w,
                      double* d_v, double* d_dvdc, void* d_ws, size_t ws_bytes, cudaStream_t st) {
  if (n_pts < 0) return fail(FE_ERR_ARG, "fe_esp_field_fp64: n_pts < 0");
  if (n_pts == 0) return FE_OK;
  if (!d_table || !d_pts || (!d_v && !d_dvdc)) return fail(FE_ERR_ARG, "fe_esp_field_fp64: null argument");
  return field_launch("fe_esp_field_fp64", static_cast<const unsigned char*>(d_table), d_pts,
                      n_pts, d_w, d_v, d_dvdc, d_ws, ws_bytes, st);
}

size_t fe_adjoint_ws_bytes(const fe_plan* p, int n_pts) {
  if (!p || n_pts < 0) return 0;
  return adj_layout(p, n_pts).bytes;
}

int fe_esp_adjoint(const fe_plan* p, const void* d_plan, const void* d_table,
                   const double* d_pts, int n_pts, const double* d_dLdV, double* d_dLdC,
                   double* d_dLdP, void* d_ws, size_t ws_bytes, cudaStream_t st) {
  if (!p || !d_table || n_pts < 0 || (n_pts > 0 && (!d_pts || !d_dLdV)))
    return fail(FE_ERR_ARG, "fe_esp_adjoint: bad argument");
  if (d_dLdP && !d_plan) return fail(FE_ERR_ARG, "fe_esp_adjoint: dL/dP needs the device plan");
  const AdjLayout lay = adj_layout(p, n_pts);
  if (!d_ws || ws_bytes < lay.bytes)
    return fail(FE_ERR_SIZE, "fe_esp_adjoint: workspace %zu < %zu bytes", ws_bytes, lay.bytes);
  if (reinterpret_cast<uintptr_t>(d_ws) & 255)
    return fail(FE_ERR_ARG, "fe_esp_adjoint: workspace not 256-byte aligned");
  const unsigned char* tb = static_cast<const unsigned char*>(d_table);
  unsigned char* wb = static_cast<unsigned char*>(d_ws);
  if (d_dLdP) {
    // the table must come from a build with this plan (same capacities, sources filled)
    FeTableHdr h{};
    FE_CUDA(cudaMemcpyAsync(&h, tb, sizeof h, cudaMemcpyDeviceToHost, st));
    FE_CUDA(cudaStreamSynchronize(st));
    if (h.magic != FE_TABLE_MAGIC) return fail(FE_ERR_ARG, "fe_esp_adjoint: not a pair table");
    if (!h.has_src)
      return fail(FE_ERR_ARG, "fe_esp_adjoint: dL/dP needs a table built on the device "
                  "(imported tables carry no pair sources)");
    for (int L = 0; L < FE_NCLASS; ++L)
      if (h.cap[L] != p->cap[L])
        return fail(FE_ERR_ARG, "fe_esp_adjoint: table was not built with this plan");
    FE_CUDA(cudaMemsetAsync(d_dLdP, 0, size_t(p->n_func) * p->n_func * sizeof(double), st));
  }
  if (n_pts == 0) return FE_OK;
  if (d_dLdC) {
    const int rc = field_launch("fe_esp_adjoint", tb, d_pts, n_pts, d_dLdV, nullptr, d_dLdC,
                                wb + lay.field, lay.mom - lay.field, st);
    if (rc != FE_OK) return rc;
  }
  if (!d_dLdP || lay.nsrc == 0) return FE_OK;
  const unsigned char* pb = static_cast<const unsigned char*>(d_plan);
  FeAdjArgs a{};
  a.table = tb;
  a.pts = d_pts;
  a.w = d_dLdV;
  a.npts = n_pts;
  a.mom = reinterpret_cast<double*>(wb + lay.mom);
  for (int L = 0; L < FE_NCLASS; ++L) a.mom_off[L] = lay.mom_off[L];
  a.shells = reinterpret_cast<const FeShell*>(pb + p->o_shells);
  a.sexp = reinterpret_cast<const double*>(pb + p->o_sexp);
  a.scoef = reinterpret_cast<const double*>(pb + p->o_scoef);
  a.tasks = reinterpret_cast<const FeTask*>(pb + p->o_tasks);
  a.work_task = reinterpret_cast<const int*>(pb + p->o_wt);
  a.work_ij = reinterpret_cast<const int*>(pb + p->o_wij);
  a.n_func = p->n_func;
  a.dw = reinterpret_cast<double*>(wb + lay.dw);
  a.dw_stride = lay.dw_stride;
  a.first = reinterpret_cast<int*>(wb + lay.first);
  a.last = reinterpret_cast<int*>(wb + lay.last);
  a.nsrc = lay.nsrc;
  a.dD = d_dLdP;
  int rc = FE_OK;
#define FE_MOM(l) if (rc == FE_OK) rc = launch_moments<l, 0>(a, p->cap[l], st);
  FE_MOM(0) FE_MOM(1) FE_MOM(2) FE_MOM(3) FE_MOM(4) FE_MOM(5) FE_MOM(6) FE_MOM(7) FE_MOM(8)
#undef FE_MOM
  if (rc != FE_OK) return rc;
  const unsigned nb = unsigned((lay.nsrc + FE_ADJ_THREADS - 1) / FE_ADJ_THREADS);
  fe_adj_pair_kernel<<<nb, FE_ADJ_THREADS, 0, st>>>(a);
  FE_CUDA(cudaGetLastError());
  const int ntask = int(p->tasks.size());
  FE_CUDA(cudaMemsetAsync(a.first, 0xff, size_t(ntask) * sizeof(int), st));
  fe_adj_ranges_kernel<<<nb, FE_ADJ_THREADS, 0, st>>>(a);
  FE_CUDA(cudaGetLastError());
  const long long nq = (long long)ntask * lay.dw_stride;
  if (nq > 0) {
    fe_adj_gather_kernel<<<unsigned((nq + 255) / 256), 256, 0, st>>>(a, ntask);
    FE_CUDA(cudaGetLastError());
  }
  return FE_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched evaluation
// ---------------------------------------------------------------------------
struct fe_batch {
  int np = 2;
  int stage = FE_STAGE_BYTES;            // pair-tile (ring stage) bytes
  int grid[2] = {1, 1};
  std::vector<FeBatchMolDev> mols;
  std::vector<FeBatchItem> items[2];     // classes 0..FE_LSPLIT, the g-shell classes
  long long total_pts = 0;
  size_t partial_doubles = 0;
  size_t desc_bytes = 0, ws_bytes = 0;
  size_t off_mol = 0, off_item[2] = {0, 0};
  int n_items() const { return int(items[0].size() + items[1].size()); }
};

namespace {

constexpr size_t kBatchCounterBytes = 256;   // two counters, one per kernel instance

template <int NP, int STAGE>
struct BatchKernels {
  static constexpr int kMinB = NP == 1 ? 4 : kMinB64;
  static const void* main() {
    return reinterpret_cast<const void*>(fe_batch_f64_kernel<NP, kMinB, 0, FE_LSPLIT, 0, STAGE>);
  }
  static const void* high() {
    return reinterpret_cast<const void*>(
        fe_batch_f64_kernel<NP, 1, FE_LSPLIT + 1, FE_NCLASS - 1, 1, STAGE>);
  }
};

int batch_kernels(int np, int stage, const void*& k0, const void*& k1) {
#define FE_BK(n, sb)                                  \
  if (np == n && stage == sb) {                        \
    k0 = BatchKernels<n, sb>::main();                  \
    k1 = BatchKernels<n, sb>::high();                  \
    return FE_OK;                                      \
  }
  FE_BK(1, 8192) FE_BK(1, 16384) FE_BK(1, 32768) FE_BK(2, 8192) FE_BK(2, 16384) FE_BK(2, 32768)
#undef FE_BK
  if (np != 1 && np != 2) return fail(FE_ERR_ARG, "fe_batch_create: points_per_thread must be 1 or 2");
  return fail(FE_ERR_ARG, "fe_batch_create: stage_bytes must be 8192, 16384 or 32768");
}

// Algorithmic FLOPs of one (pair, point) evaluation of class L.
double pair_point_flops(int L) {
  const int nmono = (L + 1) * (L + 2) * (L + 3) / 6;
  return 2.0 * fe_class_nterm[L] + (nmono - 1) + 14 + 3 * L;
}

}  // namespace

extern "C" {

int fe_batch_create(const fe_batch_mol* in, int n_mol, const fe_batch_shape* shape,
                    fe_batch** out, cudaStream_t st) {
  if (!out || n_mol < 0 || (n_mol > 0 && !in)) return fail(FE_ERR_ARG, "fe_batch_create: bad argument");
  *out = nullptr;
  const int np = shape ? shape->points_per_thread : 2;
  const int waves = shape ? shape->waves : 4;
  const int stage = shape && shape->stage_bytes ? shape->stage_bytes : FE_STAGE_BYTES;
  if (waves < 1 || waves > 64) return fail(FE_ERR_ARG, "fe_batch_create: waves must be in 1..64");
  const void* k0 = nullptr;
  const void* k1 = nullptr;
  {
    const int rc = batch_kernels(np, stage, k0, k1);
    if (rc != FE_OK) return rc;
  }
  const int smem = FE_NSTAGE * stage;
  FE_CUDA(cudaFuncSetAttribute(k0, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  FE_CUDA(cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  int occ0 = 0, occ1 = 0;
  FE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ0, k0, 128, smem));
  FE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ1, k1, 128, smem));
  occ0 = std::max(occ0, 1);
  occ1 = std::max(occ1, 1);

  auto* b = new fe_batch();
  b->np = np;
  b->stage = stage;
  const int ppb = 128 * np;
  std::vector<std::array<int, FE_NCLASS>> cnt(n_mol);
  double total = 0.0;
  for (int m = 0; m < n_mol; ++m) {
    cnt[m].fill(0);
    if (in[m].n_pts < 0 || (in[m].n_pts > 0 && (!in[m].d_table || !in[m].d_pts || !in[m].d_out))) {
      delete b;
      return fail(FE_ERR_ARG, "fe_batch_create: molecule %d: bad buffers", m);
    }
    if (!in[m].d_table) continue;
    FeTableHdr h{};
    FE_CUDA(cudaMemcpyAsync(&h, in[m].d_table, sizeof h, cudaMemcpyDeviceToHost, st));
    FE_CUDA(cudaStreamSynchronize(st));
    if (h.magic != FE_TABLE_MAGIC) {
      delete b;
      return fail(FE_ERR_ARG, "fe_batch_create: molecule %d: not a pair table", m);
    }
    for (int L = 0; L < FE_NCLASS; ++L) {
      cnt[m][L] = h.count[L];
      total += double(h.count[L]) * pair_point_flops(L) * in[m].n_pts;
    }
  }
  // parts per (molecule, class): items of about equal cost, ``waves`` items per
  // resident block
  const double target_items = double(waves) * occ0 * sm_count();
  const double item_cost = std::max(1.0, total / target_items);
  struct Keyed { FeBatchItem it; double cost; };
  std::vector<Keyed> q[2];
  long long base = 0, pt0 = 0;
  for (int m = 0; m < n_mol; ++m) {
    FeBatchMolDev d{};
    d.table = static_cast<const unsigned char*>(in[m].d_table);
    d.pts = in[m].d_pts;
    d.out = in[m].d_out;
    d.npts = in[m].n_pts;
    d.ld = (std::max(d.npts, 1) + 31) & ~31;
    int rows = 0;
    for (int L = 0; L < FE_NCLASS; ++L) {
      d.row0[L] = rows;
      d.nsplit[L] = 0;
      if (cnt[m][L] == 0 || d.npts == 0) continue;
      const double w = double(cnt[m][L]) * pair_point_flops(L);      // per point
      int ns = int(std::ceil(ppb * w / item_cost));
      ns = std::max(1, std::min({ns, 256, std::max(1, cnt[m][L] / 32)}));
      d.nsplit[L] = ns;
      rows += ns;
    }
    d.nrows = rows;
    d.base = base;
    d.pt0 = pt0;
    if (d.npts > 0) {
      base += (long long)d.nrows * d.ld;
      pt0 += d.npts;
      const int nb = (d.npts + ppb - 1) / ppb;
      for (int L = 0; L < FE_NCLASS; ++L)
        for (int pb = 0; pb < nb && d.nsplit[L] > 0; ++pb) {
          const int pts = std::min(ppb, d.npts - pb * ppb);
          const double c = double(pts) * cnt[m][L] * pair_point_flops(L) / d.nsplit[L];
          for (int s2 = 0; s2 < d.nsplit[L]; ++s2)
            q[L > FE_LSPLIT].push_back(Keyed{FeBatchItem{m, pb, L, s2}, c});
        }
    }
    b->mols.push_back(d);
  }
  // class-major, largest first within a class (stable: deterministic order)
  for (int k = 0; k < 2; ++k) {
    std::stable_sort(q[k].begin(), q[k].end(), [](const Keyed& x, const Keyed& y) {
      return x.it.cls != y.it.cls ? x.it.cls < y.it.cls : x.cost > y.cost;
    });
    for (const Keyed& e : q[k]) b->items[k].push_back(e.it);
  }
  b->total_pts = pt0;
  b->partial_doubles = size_t(base);
  b->grid[0] = std::max(1, std::min(int(b->items[0].size()), occ0 * sm_count()));
  b->grid[1] = std::max(1, std::min(int(b->items[1].size()), occ1 * sm_count()));
  b->off_mol = align256(sizeof(FeBatchHdr));
  b->off_item[0] = align256(b->off_mol + b->mols.size() * sizeof(FeBatchMolDev));
  b->off_item[1] = align256(b->off_item[0] + b->items[0].size() * sizeof(FeBatchItem));
  b->desc_bytes = align256(b->off_item[1] + b->items[1].size() * sizeof(FeBatchItem));
  b->ws_bytes = kBatchCounterBytes + align256(b->partial_doubles * sizeof(double));
  *out = b;
  return FE_OK;
}

void fe_batch_destroy(fe_batch* b) { delete b; }

int fe_batch_sizes(const fe_batch* b, size_t* desc_bytes, size_t* ws_bytes, int* n_items) {
  if (!b) return fail(FE_ERR_ARG, "fe_batch_sizes: null batch");
  if (desc_bytes) *desc_bytes = b->desc_bytes;
  if (ws_bytes) *ws_bytes = b->ws_bytes;
  if (n_items) *n_items = b->n_items();
  return FE_OK;
}

int fe_batch_upload(const fe_batch* b, void* d_desc, size_t desc_bytes, cudaStream_t st) {
  if (!b || !d_desc) return fail(FE_ERR_ARG, "fe_batch_upload: null argument");
  if (desc_bytes < b->desc_bytes) return fail(FE_ERR_SIZE, "fe_batch_upload: %zu < %zu bytes", desc_bytes, b->desc_bytes);
  if (reinterpret_cast<uintptr_t>(d_desc) & 255) return fail(FE_ERR_ARG, "fe_batch_upload: descriptor not 256-byte aligned");
  std::vector<unsigned char> h(b->desc_bytes, 0);
  FeBatchHdr hdr{};
  hdr.n_mol = int(b->mols.size());
  hdr.np = b->np;
  hdr.total_pts = b->total_pts;
  hdr.off_mol = static_cast<long long>(b->off_mol);
  for (int k = 0; k < 2; ++k) {
    hdr.n_item[k] = int(b->items[k].size());
    hdr.off_item[k] = static_cast<long long>(b->off_item[k]);
  }
  memcpy(h.data(), &hdr, sizeof hdr);
  if (!b->mols.empty()) memcpy(h.data() + b->off_mol, b->mols.data(), b->mols.size() * sizeof(FeBatchMolDev));
  for (int k = 0; k < 2; ++k)
    if (!b->items[k].empty())
      memcpy(h.data() + b->off_item[k], b->items[k].data(), b->items[k].size() * sizeof(FeBatchItem));
  FE_CUDA(cudaMemcpyAsync(d_desc, h.data(), h.size(), cudaMemcpyHostToDevice, st));
  FE_CUDA(cudaStreamSynchronize(st));   // h is a local buffer
  return FE_OK;
}

int fe_batch_run(const fe_batch* b, const void* d_desc, void* d_ws, size_t ws_bytes, cudaStream_t st) {
  if (!b || !d_desc) return fail(FE_ERR_ARG, "fe_batch_run: null argument");
  if (b->n_items() == 0) return FE_OK;
  if (!d_ws || ws_bytes < b->ws_bytes) return fail(FE_ERR_SIZE, "fe_batch_run: workspace too small (need %zu bytes)", b->ws_bytes);
  const void* k0 = nullptr;
  const void* k1 = nullptr;
  {
    const int rc = batch_kernels(b->np, b->stage, k0, k1);
    if (rc != FE_OK) return rc;
  }
  unsigned char* wb = static_cast<unsigned char*>(d_ws);
  unsigned* counter = reinterpret_cast<unsigned*>(wb);
  double* partial = reinterpret_cast<double*>(wb + kBatchCounterBytes);
  const unsigned char* desc = static_cast<const unsigned char*>(d_desc);
  FE_CUDA(cudaMemsetAsync(counter, 0, kBatchCounterBytes, st));
  const int smem = FE_NSTAGE * b->stage;
  unsigned* c1 = counter + 32;
  if (!b->items[0].empty()) {
    void* a0[] = {&desc, &counter, &partial};
    FE_CUDA(cudaLaunchKernel(k0, dim3(b->grid[0]), dim3(128), a0, smem, st));
  }
  if (!b->items[1].empty()) {
    void* a1[] = {&desc, &c1, &partial};
    FE_CUDA(cudaLaunchKernel(k1, dim3(b->grid[1]), dim3(128), a1, smem, st));
  }
  if (b->total_pts > 0)
    fe_batch_reduce_kernel<<<unsigned((b->total_pts + 255) / 256), 256, 0, st>>>(desc, partial);
  FE_CUDA(cudaGetLastError());
  return FE_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Evaluation points
// ---------------------------------------------------------------------------
namespace {

struct PointWs {
  size_t cand, keep, pos, bsum, bytes;
  long long nb;
};

PointWs point_ws(long long ncand) {
  PointWs w{};
  size_t o = 0;
  auto put = [&](size_t bytes) { const size_t at = o; o = align256(o + bytes); return at; };
  w.cand = put(size_t(ncand) * 3 * sizeof(double));
  w.keep = put(size_t(ncand + 1) * sizeof(int));
  w.pos = put(size_t(ncand + 1) * sizeof(int));
  w.nb = (ncand + FE_SCAN_BLOCK - 1) / FE_SCAN_BLOCK;
  w.bsum = put(size_t(w.nb + 1) * sizeof(int));
  w.bytes = std::max<size_t>(o, 256);
  return w;
}

int point_run(const char* who, FePointArgs a, double* d_out, long long cap, int* d_count,
              void* d_ws, size_t ws_bytes, cudaStream_t st) {
  if (a.ncand < 0 || a.ncand >= (1LL << 31)) return fail(FE_ERR_SIZE, "%s: bad candidate count", who);
  if (!d_out || !d_count) return fail(FE_ERR_ARG, "%s: null output", who);
  const PointWs w = point_ws(a.ncand);
  if (!d_ws || ws_bytes < w.bytes) return fail(FE_ERR_SIZE, "%s: workspace %zu < %zu bytes", who, ws_bytes, w.bytes);
  if (a.ncand == 0) {
    FE_CUDA(cudaMemsetAsync(d_count, 0, sizeof(int), st));
    return FE_OK;
  }
  unsigned char* wb = static_cast<unsigned char*>(d_ws);
  a.cand = reinterpret_cast<double*>(wb + w.cand);
  a.keep = reinterpret_cast<int*>(wb + w.keep);
  int* pos = reinterpret_cast<int*>(wb + w.pos);
  int* bsum = reinterpret_cast<int*>(wb + w.bsum);
  const unsigned nblk = unsigned((a.ncand + 255) / 256);
  fe_point_candidates_kernel<<<nblk, 256, 0, st>>>(a);
  fe_scan_sums_kernel<<<unsigned(w.nb), FE_SCAN_BLOCK, 0, st>>>(a.keep, a.ncand, bsum);
  fe_scan_top_kernel<<<1, FE_SCAN_BLOCK, 0, st>>>(bsum, int(w.nb));
  fe_scan_apply_kernel<<<unsigned(w.nb), FE_SCAN_BLOCK, 0, st>>>(a.keep, a.ncand, bsum, pos);
  fe_point_compact_kernel<<<nblk, 256, 0, st>>>(a.cand, a.keep, pos, a.ncand, d_out, cap, d_count);
  FE_CUDA(cudaGetLastError());
  return FE_OK;
}

}  // namespace

extern "C" {

size_t fe_points_ws_bytes(long long ncand) { return ncand < 0 ? 0 : point_ws(ncand).bytes; }

int fe_surface_points(const double* d_xyz, const double* d_rad, int natom, const long long* d_off,
                      long long ncand, double slack, double* d_out, long long cap, int* d_count,
                      void* d_ws, size_t ws_bytes, cudaStream_t st) {
  if (natom <= 0 || !d_xyz || !d_rad || !d_off) return fail(FE_ERR_ARG, "fe_surface_points: bad atoms");
  FePointArgs a{};
  a.xyz = d_xyz;
  a.rad = d_rad;
  a.natom = natom;
  a.slack = slack;
  a.off = d_off;
  a.grid = 0;
  a.ncand = ncand;
  return point_run("fe_surface_points", a, d_out, cap, d_count, d_ws, ws_bytes, st);
}

int fe_grid_points(const double* d_xyz, int natom, double exclude, const long long* d_index,
                   long long ncand, const double* d_axes, long long nx, long long ny, long long nz,
                   double* d_out, long long cap, int* d_count, void* d_ws, size_t ws_bytes,
                   cudaStream_t st) {
  if (natom < 0 || (natom > 0 && !d_xyz) || !d_index || !d_axes || nx <= 0 || ny <= 0 || nz <= 0)
    return fail(FE_ERR_ARG, "fe_grid_points: bad argument");
  FePointArgs a{};
  a.xyz = d_xyz;
  a.natom = natom;
  a.excl = exclude;
  a.index = d_index;
  a.axes = d_axes;
  a.nx = nx;
  a.ny = ny;
  a.nz = nz;
  a.grid = 1;
  a.ncand = ncand;
  return point_run("fe_grid_points", a, d_out, cap, d_count, d_ws, ws_bytes, st);
}

}  // extern "C"
