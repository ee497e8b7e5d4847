/* fastesp_b200 -- C ABI of the B200 exact-ESP library (libfastesp_b200.so).
 *
 * The reference (ZidongS/fastesp) reaches its native code through two
 * executables and files: ``build_pairs basis.bin pairs.bin tol``
 * (fastesp/native/build_pairs.cpp:162-425, called from fastesp/cli.py:143-150)
 * and ``esp_gpu pairs.bin out.txt`` (fastesp/native/esp_gpu.cu:232-326, called
 * from fastesp/cli.py:153-168).  This header replaces both with in-process
 * calls.  The basis description is the reference's ``basis_payload`` dict
 * (fastesp/table.py:268-293) field for field.
 *
 * Conventions
 *  - Every device buffer is allocated by the caller; the library allocates no
 *    device memory.  Sizes come from fe_plan_sizes / fe_eval_ws_bytes.
 *  - Calls are stream-ordered and asynchronous unless stated otherwise.
 *  - Every function returns FE_OK (0) or an FE_ERR_* code and never exits the
 *    process; fe_last_error() gives the message of the calling thread's last
 *    failure.  Kernels report anomalies (a bounded wait that gave up, a
 *    capacity overflow) in a device status word read by fe_status().
 */
#ifndef FASTESP_B200_H
#define FASTESP_B200_H

#include <stddef.h>
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FE_OK 0
#define FE_ERR_ARG 1          /* invalid argument or shape */
#define FE_ERR_CUDA 2         /* a CUDA runtime call failed */
#define FE_ERR_SIZE 3         /* a caller buffer is too small */
#define FE_ERR_UNSUPPORTED 4  /* angular momentum above g, or similar */
#define FE_ERR_DEVICE 5       /* the device status word reports a failure */

#define FE_NCLASS 9           /* angular classes L = la + lb = 0..8 */

#define FE_RULE_NUMPY 0       /* keep unless K*bound/max(dmin, 0.05) < tol (fastesp/table.py:193) */
#define FE_RULE_NATIVE 1      /* drop if K*bound/max(dmin - reff, 0.05) < tol (build_pairs.cpp:326-328) */

/* Host copy of the basis payload (fastesp/table.py:268-293): per Cartesian
 * function its atom, primitive count and offset, Cartesian exponents, shell
 * id and centre; per primitive exponent and coefficient; per atom Z and xyz. */
typedef struct fe_basis {
  int n_func, n_prim, n_atoms;
  const int *fn_atom, *fn_nprim, *fn_off, *fn_lx, *fn_ly, *fn_lz, *fn_shell;
  const double *fc;      /* (n_func, 3) */
  const double *pexp;    /* (n_prim,)  */
  const double *pcoef;   /* (n_prim,)  */
  const double *Z;       /* (n_atoms,) */
  const double *xyz;     /* (n_atoms, 3) */
} fe_basis;

typedef struct fe_plan fe_plan;    /* opaque, host memory */

typedef struct fe_sizes {
  size_t plan_bytes;       /* device bytes of the uploaded plan */
  size_t table_bytes;      /* device bytes of one pair table */
  size_t build_ws_bytes;   /* device workspace of fe_table_build without points (fe_build_ws_bytes) */
  int n_shell, n_shell_pair, n_work;
  int cap[FE_NCLASS];      /* primitive-pair slots per class (upper bound of kept pairs) */
} fe_sizes;

typedef struct fe_table_info {
  int count[FE_NCLASS];    /* kept primitive pairs per class */
  int n_pairs;             /* sum of count */
  int n_atoms;
  double sum_rule;         /* Tr(P S) = sum over pairs K (pi/p)^1.5 etab_0 (build_pairs.cpp:294-296) */
  double tol;
  int rule;
  int has_f32;
  int n_warp_screen;       /* pairs of the last device build whose screen took the warp-parallel search */
} fe_table_info;

/* Version as major*10000 + minor*100 + patch. */
int fe_version(void);

/* Message of the calling thread's last failed call ("" if none). */
const char* fe_last_error(void);

/* Read the device status word of the current device (synchronises the
 * device); clear it when ``clear`` is non-zero.  Bits: 1 a bounded wait gave
 * up, 2 an invalid class, 4 a capacity overflow. */
int fe_status(unsigned* bits, int clear);

/* Group the functions into shells (contiguous runs of fn_shell, as
 * build_pairs.cpp:170-182 does), enumerate the shell pairs si <= sj and their
 * primitive pairs in the reference's order, and size everything.
 * Replaces the set-up half of build_pairs' main (build_pairs.cpp:162-187). */
int fe_plan_create(const fe_basis* basis, fe_plan** out);
void fe_plan_destroy(fe_plan* plan);
int fe_plan_sizes(const fe_plan* plan, fe_sizes* sizes);

/* Copy the plan to the caller's device buffer (plan_bytes, 256-byte aligned). */
int fe_plan_upload(const fe_plan* plan, void* d_plan, cudaStream_t stream);

/* Workspace bytes of fe_table_build with n_pts screening points: the plan's
 * build_ws_bytes plus the bounding boxes of the point blocks. */
size_t fe_build_ws_bytes(const fe_plan* plan, int n_pts);

/* Build the pair table on the GPU: E-coefficients, density-weighted Hermite
 * table, G[alpha, m] contraction, screening bound and point screen, then an
 * order-preserving compaction per class.  ``d_dens`` is the (n_func, n_func)
 * Cartesian density, ``d_pts`` the (n_pts, 3) points (Bohr) used for the
 * screen, ``rule`` FE_RULE_NUMPY or FE_RULE_NATIVE.  Replaces the hot loop and
 * output of build_pairs (build_pairs.cpp:194-421) and build_table
 * (fastesp/table.py:176-259).  Stream-ordered on ``stream``: the per-(la, lb)
 * group kernels and the per-class record kernels run on the library's own
 * side streams of the device, forked from ``stream`` by an event and joined
 * back into it, so they start after the work already on ``stream`` and every
 * later launch on ``stream`` waits for them.  Calls from several host threads
 * take turns on the side streams. */
int fe_table_build(const fe_plan* plan, const void* d_plan, const double* d_dens,
                   const double* d_pts, int n_pts, double tol, int rule,
                   void* d_table, void* d_ws, size_t ws_bytes, cudaStream_t stream);

/* Bytes of a table whose class L holds up to cap[L] pairs (0 on bad input),
 * and the byte offsets of its FP64 records, FP32 records and atom block. */
size_t fe_table_bytes(const int* cap, int n_atoms);
int fe_table_offsets(const int* cap, int n_atoms, size_t* off64, size_t* off32,
                     size_t* off_atoms);

/* Write the header and atom block of a table holding count[L] pairs per class
 * whose FP64 records the caller copies in itself (import of a pairs.bin
 * table, fastesp/table.py:143-170).  Synchronises ``stream``. */
int fe_table_init(void* d_table, const int* count, int n_atoms, const double* Z,
                  const double* xyz, cudaStream_t stream);

/* (Re)derive the FP32 records of the mixed-precision path from the FP64 ones. */
int fe_table_make_f32(void* d_table, cudaStream_t stream);

/* Copy the table header to the host (synchronises ``stream``). */
int fe_table_info_get(const void* d_table, fe_table_info* info, cudaStream_t stream);

/* Workspace bytes of an FP64 evaluation of n_pts points: the per-split
 * partial sums of the pair-split reduction (the minimum; see
 * fe_point_order_bytes). */
size_t fe_eval_ws_bytes(int n_pts);

/* Further workspace bytes with which the evaluators (fe_esp_fp64,
 * fe_electron_fp64, fe_electron_classes at precision 0) take the points in a
 * spatially coherent order -- a stable counting sort by the Morton code of a
 * 16^3 grid of cells over the points' bounding box -- and write every result
 * to its caller's row.  Faster for point sets in any order; the FP64 results
 * are the same bit for bit either way (each point's sum runs over the pairs in
 * table order whatever its neighbours).  fe_eval_ws_bytes_mixed includes them:
 * the mixed path always evaluates in this order. */
size_t fe_point_order_bytes(int n_pts);

/* Workspace bytes of a mixed-precision evaluation of n_pts points of a table
 * holding at most cap[L] pairs of class L (fe_sizes.cap of its plan, or the
 * counts of an imported table): partial sums, the spatial point order
 * (fe_point_order_bytes) and the FP64 routing mask (one bit per pair and warp
 * of points). */
size_t fe_eval_ws_bytes_mixed(int n_pts, const int* cap);

/* V(C) = sum_A Z_A/|C-R_A| - sum_pairs K sum_k G_k R^alpha F_m(p R^2), all FP64,
 * for the (n_pts, 3) points ``d_pts`` into ``d_out`` (n_pts,).  Replaces
 * esp_pairs_kernel + esp_reduce_kernel (fastesp/native/esp_gpu.cu:161-229)
 * and PairTable.esp (fastesp/table.py:102-104). */
int fe_esp_fp64(const void* d_table, const double* d_pts, int n_pts, double* d_out,
                void* d_ws, size_t ws_bytes, cudaStream_t stream);

/* Mixed precision: the Boys vector, monomials and term products in FP32, each
 * pair's contribution accumulated in FP64 per point; a pair is evaluated in
 * FP64 for a warp of points whenever the bound sum_n b_n/|R|^(n+1) on
 * K sum_k |G_k R^alpha F_m| (b_n formed by the table build from G, p and K)
 * reaches ``tau`` (a.u.; <= 0 selects the default) for one of them; the split sums, the
 * nuclear term and the final subtraction are FP64.  Same result as
 * fe_esp_fp64 within 1e-6 a.u. on the tested systems.  ``d_n64`` (nullable)
 * accumulates the number of (pair, warp) evaluations routed to FP64.  No
 * counterpart in the reference, which is FP64 only. */
int fe_esp_mixed(const void* d_table, const double* d_pts, int n_pts, double* d_out,
                 void* d_ws, size_t ws_bytes, double tau, unsigned long long* d_n64,
                 cudaStream_t stream);
int fe_electron_mixed(const void* d_table, const double* d_pts, int n_pts, double* d_out,
                      void* d_ws, size_t ws_bytes, double tau, unsigned long long* d_n64,
                      cudaStream_t stream);

/* The electron part alone, int rho(r)/|r-C| dr (fastesp/table.py:73-93), FP64. */
int fe_electron_fp64(const void* d_table, const double* d_pts, int n_pts, double* d_out,
                     void* d_ws, size_t ws_bytes, cudaStream_t stream);

/* The electron part of the pairs of classes lmin..lmax only (no counterpart in
 * the reference): FP64 (precision 0, workspace fe_eval_ws_bytes) or mixed
 * (precision 1, workspace fe_eval_ws_bytes_mixed, routing threshold tau as in
 * fe_esp_mixed).  The sum over a partition of 0..FE_NCLASS-1 into ranges is the
 * full electron part; used to time and rate each class on its own. */
int fe_electron_classes(const void* d_table, const double* d_pts, int n_pts, double* d_out,
                        void* d_ws, size_t ws_bytes, int precision, double tau, int lmin,
                        int lmax, unsigned long long* d_n64, cudaStream_t stream);

/* The nuclear part alone, sum_A Z_A/|C-R_A| (fastesp/table.py:95-100); the
 * workspace arguments are unused and may be null. */
int fe_nuclear_fp64(const void* d_table, const double* d_pts, int n_pts, double* d_out,
                    void* d_ws, size_t ws_bytes, cudaStream_t stream);

/* Boys function F_0..F_mmax(T) for n arguments into d_F (n, mmax+1), FP64.
 * Same values as fastesp.ints.boys (fastesp/ints.py:35-40). */
int fe_boys_fp64(const double* d_T, int n, int mmax, double* d_F, cudaStream_t stream);

/* fe_esp_fp64 without a caller workspace (no counterpart in the reference).
 * For callers that cannot allocate device memory -- a host framework that
 * owns the device-memory budget and lends only input and output buffers, or a
 * binding of the reference's table-and-points-in / potentials-out interface --
 * the partial sums live in a file-scope device array of
 * fe_noalloc_scratch_bytes() (16 MiB) that every GPU loading the library keeps
 * until the process exits.  A point count n fits when fe_eval_ws_bytes(n) <=
 * fe_noalloc_scratch_bytes(): up to 232,992 points on a 148-SM B200 (large
 * counts need 9 FP64 rows of the padded point count); larger counts are
 * refused with FE_ERR_SIZE before anything is launched.  Allocates nothing: no
 * cudaMalloc, cudaFree or allocating library routine.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) and should
 * come before any stream capture; the address is looked up again after a
 * device reset (a new context).  All calls share the array and every partial
 * sum it holds is rewritten before it is read, so nothing needs clearing: a
 * block whose bounded wait gave up writes NaN for its points, and the status
 * word (fe_status) records it.  Calls whose executions overlap on the GPU
 * (other streams, other host threads) race on the array and must be
 * serialised by the caller. */
int fe_esp_fp64_noalloc(const void* d_table, const double* d_pts, int n_pts, double* d_out,
                        cudaStream_t stream);
size_t fe_noalloc_scratch_bytes(void);

/* Potential and its gradient with respect to the points, FP64 (no counterpart
 * in the reference, which evaluates the potential only).  With R = C - P,
 * dV/dC = sum_A -Z_A (C-R_A)/|C-R_A|^3
 *         - sum_pairs K sum_k G_k (a R^(a-e) F_m - 2p R R^a F_(m+1))(pR^2),
 * i.e. minus the electric field.  d_v (n, nullable) receives V; d_dvdc (n, 3,
 * nullable) receives w_i dV_i/dC_i with w = d_w (n, nullable: w_i = 1).
 * Workspace: fe_field_ws_bytes(n_pts). */
size_t fe_field_ws_bytes(int n_pts);
int fe_esp_field_fp64(const void* d_table, const double* d_pts, int n_pts, const double* d_w,
                      double* d_v, double* d_dvdc, void* d_ws, size_t ws_bytes,
                      cudaStream_t stream);

/* Adjoint of V = table.esp(points) for a loss with dL/dV = d_dLdV (n), FP64
 * (no counterpart in the reference).  d_dLdC (n, 3, nullable) receives
 * dL/dC = dL/dV dV/dC; d_dLdP (n_func, n_func, nullable) receives dL/dP with
 * respect to the Cartesian density given to fe_table_build: the per-pair
 * point-weighted moments sum_i w_i R^a F_m are carried back through
 * G = (2pi/p)(2p)^m M0 etab and etab = sum W c_a c_b Ex Ey Ez (the builder's
 * contraction, fastesp/esp.py:239-250) to the density entries, with the kept
 * pair set held fixed.  dL/dP needs a table built by fe_table_build with this
 * plan; it reads the table header (one synchronising copy).  Deterministic:
 * fixed summation orders, no atomics.  Workspace: fe_adjoint_ws_bytes(plan,
 * n_pts), 256-byte aligned. */
size_t fe_adjoint_ws_bytes(const fe_plan* plan, int n_pts);
int fe_esp_adjoint(const fe_plan* plan, const void* d_plan, const void* d_table,
                   const double* d_pts, int n_pts, const double* d_dLdV, double* d_dLdC,
                   double* d_dLdP, void* d_ws, size_t ws_bytes, cudaStream_t stream);

/* Batched FP64 evaluation (no counterpart in the reference, which runs one
 * molecule per process): V for many molecules, each with its own table and
 * points, in one persistent launch over a flattened queue of
 * (molecule, point block, pair split) work items ordered largest first and
 * claimed by the resident blocks from a global counter.  Same per-point
 * arithmetic as fe_esp_fp64; deterministic.  Use: fe_batch_create (reads
 * every table's header: synchronising), fe_batch_sizes, a caller-allocated
 * descriptor filled by fe_batch_upload, then fe_batch_run any number of times
 * (stream-ordered, no synchronisation or allocation: it can be captured in a
 * CUDA graph) with a workspace of the reported size.  The buffers named in
 * ``mols`` must stay valid while the batch is used. */
typedef struct fe_batch_mol {
  const void* d_table;          /* pair table (fe_table_build / fe_table_init) */
  const double* d_pts;          /* (n_pts, 3) Bohr */
  double* d_out;                /* (n_pts) V */
  int n_pts;
  int reserved;
} fe_batch_mol;

typedef struct fe_batch_shape {
  int points_per_thread;        /* 1 or 2: point block of 128 or 256 points */
  int waves;                    /* work items per resident block, 1..64 */
  int stage_bytes;              /* pair tile: bytes per shared-memory stage, 8192, 16384
                                   or 32768 (0: 16384); a tile holds stage_bytes / record
                                   bytes pairs of a class */
} fe_batch_shape;

typedef struct fe_batch fe_batch;   /* opaque, host memory */

int fe_batch_create(const fe_batch_mol* mols, int n_mol, const fe_batch_shape* shape,
                    fe_batch** out, cudaStream_t stream);
void fe_batch_destroy(fe_batch* batch);
int fe_batch_sizes(const fe_batch* batch, size_t* desc_bytes, size_t* ws_bytes, int* n_items);
int fe_batch_upload(const fe_batch* batch, void* d_desc, size_t desc_bytes, cudaStream_t stream);
int fe_batch_run(const fe_batch* batch, const void* d_desc, void* d_ws, size_t ws_bytes,
                 cudaStream_t stream);

/* Evaluation points on the GPU (the reference does this in NumPy:
 * benchmarks/make_points.py:22-58, examples/vdw_surface_esp.py:38-52).
 * fe_surface_points: atom a contributes d_off[a+1]-d_off[a] Fibonacci points
 * on its sphere (centre d_xyz[a], radius d_rad[a]); the candidates lying on the
 * exposed union of the spheres (distance >= d_rad[b] - slack to every atom b,
 * slack 1e-9 in the reference) are written, in candidate order, to d_out
 * (capacity cap points) and their number to *d_count.  fe_grid_points: the
 * candidates are flat indices d_index (x-major) into the nx*ny*nz grid whose
 * axis coordinates are d_axes = [x(nx), y(ny), z(nz)]; kept when farther than
 * ``exclude`` from every nucleus.  Workspace: fe_points_ws_bytes(ncand). */
size_t fe_points_ws_bytes(long long ncand);
int fe_surface_points(const double* d_xyz, const double* d_rad, int natom, const long long* d_off,
                      long long ncand, double slack, double* d_out, long long cap, int* d_count,
                      void* d_ws, size_t ws_bytes, cudaStream_t stream);
int fe_grid_points(const double* d_xyz, int natom, double exclude, const long long* d_index,
                   long long ncand, const double* d_axes, long long nx, long long ny, long long nz,
                   double* d_out, long long cap, int* d_count, void* d_ws, size_t ws_bytes,
                   cudaStream_t stream);

/* Self-test of the bounded waits (no counterpart in the reference, whose
 * tools exit on errors): one block waits on an mbarrier that nothing arrives on
 * and no copy targets, for at most ``cycles`` SM clocks (1..4e9).  The wait
 * gives up, sets bit 1 (FE_ST_TIMEOUT) of the status word and the kernel
 * returns normally, so the context stays usable; *d_done is 2 (gave up) or
 * 1 (completed).  Synchronises ``stream`` and returns FE_ERR_DEVICE when the
 * status word has the timeout bit, as every caller should treat it.  The bit
 * stays set until fe_status(..., 1) clears it. */
int fe_wait_selftest(long long cycles, int* d_done, cudaStream_t stream);

/* FMA throughput probe (no counterpart in the reference): ``blocks`` blocks of
 * 256 threads each run ``iters`` iterations of 8 independent FMA chains, in
 * FP32 (kind 0), FP64 (kind 1) or packed FP32x2 (kind 2: two lanes per
 * instruction, as the mixed evaluator issues them), writing one value per
 * block to d_out.  Timed by the caller; FLOPs = 16 * iters * 256 * blocks
 * (twice that for kind 2).  Used as the FP64/FP32 roofline. */
int fe_peak_run(int kind, long long iters, int blocks, void* d_out, cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* FASTESP_B200_H */
