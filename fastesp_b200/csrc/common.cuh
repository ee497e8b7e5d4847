// Shared device helpers: status word, bounded mbarrier waits, bulk copies.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define FE_DEV __device__ __forceinline__

// Device status bits (OR-ed into fe_status_word; read back by fe_status()).
#define FE_ST_TIMEOUT 1u      // an mbarrier wait gave up
#define FE_ST_BADCLASS 2u     // a tile named a class outside 0..FE_NCLASS-1
#define FE_ST_OVERFLOW 4u     // a count exceeded its capacity

__device__ unsigned int fe_status_word;

FE_DEV void fe_flag(unsigned bits) { atomicOr(&fe_status_word, bits); }

FE_DEV double fe_fma(double a, double b, double c) { return fma(a, b, c); }
FE_DEV float fe_fma(float a, float b, float c) { return fmaf(a, b, c); }

// Packed FP32x2 arithmetic (two lanes per instruction on sm_100), round to
// nearest, no contraction beyond the explicit fused multiply-add: the same
// results as the scalar operations lane by lane.
FE_DEV float2 fe_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
FE_DEV float2 operator*(float2 a, float2 b) { return __fmul2_rn(a, b); }
FE_DEV float2& operator*=(float2& a, float2 b) { a = __fmul2_rn(a, b); return a; }
FE_DEV float2 operator+(float2 a, float2 b) { return __fadd2_rn(a, b); }
FE_DEV float2 operator-(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
FE_DEV float2 fe_f2(float v) { return make_float2(v, v); }

FE_DEV unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

FE_DEV void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count));
}

FE_DEV void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

FE_DEV void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}

FE_DEV bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
               " selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return ok != 0;
}

// Wait for phase ``parity`` of ``bar`` for at most ``cycles`` SM clocks (and a
// hard iteration cap).  Returns false (and flags FE_ST_TIMEOUT) if it gave up.
FE_DEV bool mbar_wait_limited(uint64_t* bar, unsigned parity, long long cycles) {
  const long long t0 = clock64();
  for (unsigned it = 0; it < (1u << 26); ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (clock64() - t0 > cycles) break;
  }
  fe_flag(FE_ST_TIMEOUT);
  return false;
}

// The evaluators' wait: about 1 s of SM clock.
FE_DEV bool mbar_wait_bounded(uint64_t* bar, unsigned parity) {
  return mbar_wait_limited(bar, parity, 2000000000LL);
}

// A block whose bounded wait gave up has incomplete sums: it writes NaN to its
// points' entries of its partial row (points p0 + j * stride, j < NP), so the
// reduction gives NaN for those points instead of a partial or stale value.
template <int NP>
FE_DEV void fe_poison_row(double* row, int p0, int stride, int npts) {
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    const int p = p0 + j * stride;
    if (p < npts) row[p] = __longlong_as_double(0x7ff8000000000000LL);
  }
}

// 1-D TMA bulk copy global -> shared, completing on ``bar``; the destination is
// this block's own shared memory.  dst/src 16-byte aligned, bytes a multiple
// of 16.
FE_DEV void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

