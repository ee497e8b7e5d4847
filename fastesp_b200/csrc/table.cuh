// Device pair-table layout, shared by the builder, the evaluators and the host.
//
// One caller-allocated buffer holds the whole table:
//
//   [FeTableHdr][pad to 256][class 0 FP64 records][class 1 ...]...[class 8]
//                           [class 0 FP32 records]...[atoms: Z[n], xyz[3n]]
//                           [sources: int32 per record slot, class 0 first]
//
// Pairs are grouped by angular class L = la + lb.  A class-L FP64 record is
// fe_class_rec64[L] doubles: [p, Px, Py, Pz, K, K*bound, G_0 .. G_(nt-1), pad]
// (K*bound is the screening bound's numerator, +inf when unknown; the G_k are
// stored in the order the class's generated code reads them, fe_gpos_L), so the
// records of a tile are one contiguous, 16-byte-aligned run that a single
// bulk copy moves into shared memory.  Within a class, pairs keep the order of
// the reference builder: shell pairs (si <= sj) in shell order, then
// primitive pairs with the primitive of shell si outer.
//
// Mixed-precision records are fe_class_rec32[L] floats: the pair's centre as
// hi = float(v), lo = float(v - hi) splits, then every coefficient twice, so
// a 16-byte load yields two coefficients each already a {c, c} operand pair
// of the packed FP32x2 arithmetic:
// [p, sqrt(p), Px_hi, Py_hi, Pz_hi, Px_lo, Py_lo, Pz_lo, rfar^2, p^-1/2, 0, 0,
//  c_0, c_0, c_1, c_1, ..., c_(nt-1), c_(nt-1), b_0, .., b_L, pad to 16 bytes]
// with c_k = K G_k s_m p^-(m+1/2) formed in FP64 (s_m the Boys scale factor,
// boys.cuh), in the same consumption order as the FP64 record's G; b_n the
// coefficients of the routing bound sum_n b_n / |R|^(n+1); rfar the radius
// beyond which the pair's FP32 Boys vector is asymptotic and the routing
// bound is below the header's tau_fast (eval_mixed.cuh).
//
// The source section maps every record of a table built on the device back to
// the builder's work item (shell pair and primitive indices), so the adjoint
// can recompute the pair's Hermite coefficients; record i of class L has its
// entry at sum_{L' < L} cap[L'] + i.  Imported tables have none (has_src 0).
#pragma once
#include <cstdint>

#define FE_NCLASS_MAX 16
#define FE_TABLE_MAGIC 0x34364546   // "FE64"

struct FeTableHdr {
  int32_t magic;
  int32_t nclass;
  int32_t n_atoms;
  int32_t rule;                      // screening rule used by the build
  double tol;                        // screening threshold used by the build
  int32_t count[FE_NCLASS_MAX];      // kept pairs per class (device-written)
  int32_t cap[FE_NCLASS_MAX];        // record capacity per class
  int64_t off64[FE_NCLASS_MAX];      // byte offset of the FP64 records of class L
  int64_t off32[FE_NCLASS_MAX];      // byte offset of the FP32 records of class L
  int64_t off_atoms;                 // byte offset of Z[n_atoms] then xyz[3 n_atoms]
  int64_t bytes;                     // total bytes of the table buffer
  double sum_rule;                   // Tr(P S) accumulated by the build
  int32_t has32;                     // FP32 records are current
  int32_t has_src;                   // the source section is filled
  int64_t off_src;                   // byte offset of the source section
  float tau_fast;                    // routing threshold of the FP32 records' far radius
  int32_t n_warp_screen;             // pairs the build's per-thread screen left to the warp screen
};

static_assert(sizeof(FeTableHdr) <= 512, "header must fit its slot");
#define FE_TABLE_HDR_BYTES 512
