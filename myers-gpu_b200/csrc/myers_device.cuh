// Device helpers shared by the verification and traceback kernels: window
// sizing, reference loads and PEQ words.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "myers_internal.h"

namespace myers {

#define FULL_MASK 0xFFFFFFFFu

__device__ __forceinline__ uint32_t d_window_bases(uint32_t m, float distance) {
  // (uint32_t)(m * (1 + 2*distance)) in float32, no contraction.
  float f = __fadd_rn(1.0f, __fmul_rn(2.0f, distance));
  return (uint32_t)__fmul_rn((float)m, f);
}

__device__ __forceinline__ uint32_t d_window_words(uint32_t wb) { return wb / 8 + ((wb % 8) ? 2u : 1u); }

// The cut-off bound of a query of m bases: (uint32_t)(m * cutoff) in float32.
__device__ __forceinline__ uint32_t d_cutoff_bound(uint32_t m, float cutoff) {
  return (uint32_t)__fmul_rn((float)m, cutoff);
}

// Rows of the cut-off's first pass for a query of m bases with bound k: k
// times the multiplier (float32, truncated), plus 8, rounded up to whole
// 32-row words, at most m. The same arithmetic as host_prefix_rows.
__device__ __forceinline__ uint32_t d_prefix_rows(uint32_t m, float cutoff, float mult) {
  const uint32_t k = d_cutoff_bound(m, cutoff);
  const float r = __fmul_rn(mult, (float)k);
  const uint32_t rows = r >= 65536.0f ? 0xFFFFFFFFu : (((uint32_t)r + 8u + 31u) & ~31u);
  return rows < m ? rows : m;
}

// Reference codes 5..7 behave as A (code 0) and bit 3 is ignored, as in the
// reference kernel's select (src-api/coreMyersGPU-CC50.cu:82-95, :170).
__device__ __forceinline__ uint32_t sanitize_codes(uint32_t t) {
  uint32_t c = t & 0x77777777u;
  uint32_t bad = (c + 0x33333333u) & 0x88888888u;  // nibbles holding 5..7
  uint32_t mask = bad - (bad >> 3);                 // 0x7 in those nibbles
  return c & ~mask;
}

__device__ __forceinline__ uint32_t ref_load(const uint32_t* __restrict__ ref, long long idx,
                                             unsigned long long nwords) {
  return (idx >= 0 && (unsigned long long)idx < nwords) ? __ldg(ref + idx) : kPadWord;
}

// Word x of the query's bit vector for base c (0 outside the query).
__device__ __forceinline__ uint32_t qword(const uint32_t* __restrict__ peq, uint32_t pos_entry,
                                          int nw, int c, int x) {
  return (x >= 0 && x < nw) ? __ldg(peq + (size_t)(pos_entry + (uint32_t)(x >> 2)) * 20u + c * 4 + (x & 3))
                            : 0u;
}

// Base code of reference base `b` (absolute base index): N past the packed
// words, codes 5..7 as A.
__device__ __forceinline__ uint32_t ref_code(const uint32_t* __restrict__ ref, unsigned long long b,
                                             unsigned long long nwords) {
  return sanitize_codes(ref_load(ref, (long long)(b >> 3), nwords)) >> (4 * (uint32_t)(b & 7)) & 0xFu;
}

}  // namespace myers
