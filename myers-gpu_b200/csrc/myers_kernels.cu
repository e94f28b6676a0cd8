// Myers bit-parallel candidate verification kernels for sm_100a.
//
// One candidate = one query (m bases, as PEQ bitmaps) against one window of
// the 4-bit packed reference; the result is the first column of minimum
// semi-global edit distance and that distance (the reference computes the
// same in src-api/coreMyersGPU-CC50.cu:110-240 and, on the CPU,
// src-integration/myers-reorderBuffer-padding.c:97-176).
//
// Layout of the work:
//  * A candidate's query is a vector of 32*L*W rows held by L lanes, W
//    32-bit words per lane. The query occupies the TOP m rows; the bottom
//    p = 32*L*W - m rows are padding rows that match no base. Padding rows
//    add exactly p to every score of the last row (row p of the DP is the
//    constant p), so the score bit is always bit 31 of the top word and the
//    argmin is unchanged; p is subtracted at the end.
//  * Single-lane shapes (L = 1, W = 1..32): one candidate per lane, no lane
//    exchange at all; the W-word add is one add.cc/addc chain.
//  * Multi-lane shapes (L = 2..32): lane l holds rows [32*W*l, 32*W*(l+1)).
//    Lanes run as a systolic pipeline: at step t lane l processes column
//    t - l, taking the horizontal delta of its bottom row from lane l-1
//    (that lane's top-row Ph/Mh bits of the same column, produced one step
//    earlier) through __shfl_up_sync, with Myers' block rule (Eq |= hin<0,
//    hin shifted into Ph/Mh). One shuffle pair per step; no carry ripple.
//  * The PEQ of each candidate is staged once in shared memory, re-laid so
//    that the W words a lane needs for one base are contiguous 16-byte
//    groups (one LDS.128 per 4 words per column), already shifted to the
//    top-aligned row layout.
//  * The text is streamed per lane with one 32-bit load per 8 columns,
//    prefetched one block ahead; a funnel shift realigns it for the exact
//    window mode and for the per-lane skew of the systolic pipeline.
//  * min(score, column) is tracked as one 32-bit key (score << 16 | column):
//    an unsigned min keeps the smallest score and, among equal scores, the
//    first column -- the reference's strict-< tie-break.
#include <cstdint>
#include <cuda_runtime.h>
#include <utility>

#include "myers_internal.h"
#include "myers_device.cuh"

namespace myers {

// Shared-memory PEQ of one warp. Candidates of the same read share one slot
// (the candidates of a read are adjacent in a tile), so a warp stages one
// copy per distinct read. Layout: [group g][base c][column][4 words], group g
// holding words 4g..4g+3 of a lane's W words and column = slot * L + lane in
// the segment. NCOL (the column count) is 1 mod 8, so the eight lanes of one
// LDS.128 phase that read the same slot with different bases hit different
// 16-byte bank groups.
template <int W, bool MULTI>
struct Layout {
  static constexpr int GW = (W + 3) / 4;
  // single-lane shapes: up to 32 slots (16 for W > 16, which halves the
  // footprint of the widest shapes); multi-lane: one column per lane
  static constexpr int SLOTS = MULTI ? 32 : (W > 16 ? 16 : 32);
  static constexpr int NCOL = ((SLOTS + 7) / 8) * 8 + 1;
  static constexpr int BASE = NCOL * 4;       // words between bases of a group
  static constexpr int GROUP = 5 * NCOL * 4;  // words between groups
  static constexpr int WORDS = GW * GROUP;    // per warp
};

// Stage lane l's W words (of a 32*LW-row top-aligned query) for all five
// bases. `dst` = the warp's region + column * 4.
template <int W, bool MULTI>
__device__ __forceinline__ void stage_lane(uint32_t* __restrict__ dst, const uint32_t* __restrict__ peq,
                                           uint32_t pos_entry, uint32_t m, int LW, int l) {
  using Lay = Layout<W, MULTI>;
  const int nw = (int)((m + 31) >> 5);
  const int p = LW * 32 - (int)m;
  const int pw = p >> 5, ps = p & 31;
#pragma unroll 1
  for (int g = 0; g < Lay::GW; ++g) {
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      uint32_t v[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int a = l * W + 4 * g + j - pw;
        uint32_t hi = qword(peq, pos_entry, nw, c, a);
        uint32_t lo = qword(peq, pos_entry, nw, c, a - 1);
        v[j] = ps ? __funnelshift_r(lo, hi, 32 - ps) : hi;
      }
      *reinterpret_cast<uint4*>(dst + g * Lay::GROUP + c * Lay::BASE) = make_uint4(v[0], v[1], v[2], v[3]);
    }
  }
}

// The W Eq words of one base; `p` points at the lane's words of that base
// in group 0.
template <int W, bool MULTI>
__device__ __forceinline__ void load_eq(const uint32_t* __restrict__ p, uint32_t (&eq)[W]) {
#pragma unroll
  for (int g = 0; g < (W + 3) / 4; ++g) {
    const uint32_t* q = p + g * Layout<W, MULTI>::GROUP;
    if (4 * g + 4 <= W) {
      uint4 v = *reinterpret_cast<const uint4*>(q);
      eq[4 * g] = v.x;
      eq[4 * g + 1] = v.y;
      eq[4 * g + 2] = v.z;
      eq[4 * g + 3] = v.w;
    } else if (W - 4 * g >= 2) {
      uint2 v = *reinterpret_cast<const uint2*>(q);
      eq[4 * g] = v.x;
      eq[4 * g + 1] = v.y;
      if (W - 4 * g == 3) eq[4 * g + 2] = q[2];
    } else {
      eq[4 * g] = q[0];
    }
  }
}

#ifndef MYERS_SHIFT_MODE
#define MYERS_SHIFT_MODE 0
#endif

// Multipliers read from the kernel parameters. ptxas cannot fold them into
// shifts or adds, so multiply-adds by them execute on the FMA pipe, which the
// Myers recurrence leaves idle (it saturates the integer ALU pipe). The
// per-column bookkeeping -- score update, text code extraction, shared
// memory addressing, lane masks -- runs there.
struct Mul {
  uint32_t one, two;   // 1, 2
  uint32_t k16, mk16;  // 1 << 16, -(1 << 16)
  uint32_t p28;        // 1 << 28: umulhi(x, p28) = x >> 4
  uint32_t kb33, kb17; // bytes between bases of a group for 33 / 17 columns
  uint32_t mn16;       // -16
  uint32_t mone;       // -1
};

__device__ __forceinline__ Mul make_mul(const DevInputs& in) {
  return Mul{in.one, in.two, in.k16, in.mk16, in.p28, in.kb33, in.kb17, in.mn16, in.mone};
}

#ifndef MYERS_FMA_KEY
#define MYERS_FMA_KEY 1
#endif

// The next text code (low nibble of t) and t shifted to the following one.
// With MYERS_FMA_KEY both are FMA-pipe ops: the code is t - 16 * (t >> 4),
// equal to t & 7 since sanitised codes are 0..4.
__device__ __forceinline__ uint32_t next_code(uint32_t& t, Mul k) {
#if MYERS_FMA_KEY
  const uint32_t tn = __umulhi(t, k.p28);
  const uint32_t code = tn * k.mn16 + t;
  t = tn;
  return code;
#else
  const uint32_t code = t & 7u;
  t = __umulhi(t, k.p28);
  return code;
#endif
}

// Score key update for one column on the FMA pipe: the top row's Ph / Mh bit
// 31 add +1 / -1 to the score held in bits 16..31 of sc.
__device__ __forceinline__ uint32_t score_step(uint32_t sc, uint32_t tp, uint32_t tm, Mul k) {
  const uint32_t hp = __umulhi(tp, k.two);
  const uint32_t hm = __umulhi(tm, k.two);
  sc = hp * k.k16 + sc;
  return hm * k.mk16 + sc;
}

// The same with the column folded in: sk holds score << 16 plus the column
// and advances by one column per call -- the (score, column) key without an
// ALU add.
__device__ __forceinline__ uint32_t key_step(uint32_t sk, uint32_t tp, uint32_t tm, Mul k) {
  const uint32_t hp = __umulhi(tp, k.two);
  const uint32_t hm = __umulhi(tm, k.two);
  const uint32_t up = hp * k.k16 + k.one;
  sk = hm * k.mk16 + sk;
  return up * k.one + sk;
}

// Bytes between the bases of a PEQ group for shape (W, MULTI).
template <int W, bool MULTI>
__device__ __forceinline__ uint32_t base_bytes(Mul k) {
  static_assert(Layout<W, MULTI>::NCOL == 33 || Layout<W, MULTI>::NCOL == 17, "column count");
  return Layout<W, MULTI>::NCOL == 33 ? k.kb33 : k.kb17;
}

// How the words of the multi-word add are formed: 0 add/addc (ALU pipe);
// 1 every word as a multiply-add by an opaque one with carry (mad.lo.cc /
// madc.lo.cc); 2 the odd words that way.
#ifndef MYERS_MADC_ADD
#define MYERS_MADC_ADD 0
#endif

// s = a + b over W words with the carry rippling through the CC flag.
template <int W>
__device__ __forceinline__ void add_chain(const uint32_t (&a)[W], const uint32_t (&b)[W], uint32_t (&s)[W],
                                          uint32_t one) {
  if constexpr (W == 1) {
    (void)one;
    s[0] = a[0] + b[0];
  } else if constexpr (MYERS_MADC_ADD == 0) {
    (void)one;
    asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(s[0]) : "r"(a[0]), "r"(b[0]));
#pragma unroll
    for (int j = 1; j < W - 1; ++j)
      asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(s[j]) : "r"(a[j]), "r"(b[j]));
    asm volatile("addc.u32 %0, %1, %2;" : "=r"(s[W - 1]) : "r"(a[W - 1]), "r"(b[W - 1]));
  } else {
    constexpr int ALL = MYERS_MADC_ADD == 1;
    if (ALL) asm volatile("mad.lo.cc.u32 %0, %1, %2, %3;" : "=r"(s[0]) : "r"(a[0]), "r"(one), "r"(b[0]));
    else asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(s[0]) : "r"(a[0]), "r"(b[0]));
#pragma unroll
    for (int j = 1; j < W - 1; ++j) {
      if (ALL || (j & 1))
        asm volatile("madc.lo.cc.u32 %0, %1, %2, %3;" : "=r"(s[j]) : "r"(a[j]), "r"(one), "r"(b[j]));
      else
        asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(s[j]) : "r"(a[j]), "r"(b[j]));
    }
    if (ALL || ((W - 1) & 1))
      asm volatile("madc.lo.u32 %0, %1, %2, %3;" : "=r"(s[W - 1]) : "r"(a[W - 1]), "r"(one), "r"(b[W - 1]));
    else
      asm volatile("addc.u32 %0, %1, %2;" : "=r"(s[W - 1]) : "r"(a[W - 1]), "r"(b[W - 1]));
  }
}

#ifndef MYERS_FMA_SHIFT_MAX_W
#define MYERS_FMA_SHIFT_MAX_W 8  // plain-100b +1.7% (measured); no change on wider shapes
#endif
// where the FMA-pipe shifts apply besides the plain single-lane shapes:
// single-lane shapes of the persistent kernel gain too (short reads on the
// batched path, +1.7%); multi-lane shapes lose (8-word lanes of 1000-base
// reads, -1.1%), all measured
#ifndef MYERS_FMA_SHIFT_BATCHED
#define MYERS_FMA_SHIFT_BATCHED 1
#endif
#ifndef MYERS_FMA_SHIFT_MULTI
#define MYERS_FMA_SHIFT_MULTI 0
#endif

// Which of a column's one-bit shifts run on the FMA pipe (a shift policy):
//   0  none (funnel shifts on the ALU pipe)
//   1  all of them
//   2  the Ph shifts of every word, the Mh shifts on the ALU pipe
//   3  both shifts of the odd words
//   4  the Ph shifts of the odd words
// Single-lane shapes of more than MYERS_FMA_SHIFT_MAX_W words use policy
// MYERS_FMA_SHIFT_WIDE.
#ifndef MYERS_FMA_SHIFT_WIDE
#define MYERS_FMA_SHIFT_WIDE 0
#endif

// The shift policy of shape (W, MULTI) in the plain or the persistent kernel.
template <int W, bool MULTI, bool PERSISTENT>
__host__ __device__ constexpr int fma_shift() {
  if (MYERS_SHIFT_MODE == 2) return 1;
  if (PERSISTENT && !MYERS_FMA_SHIFT_BATCHED) return 0;
  if (MULTI) return MYERS_FMA_SHIFT_MULTI ? 1 : 0;
  return W <= MYERS_FMA_SHIFT_MAX_W ? 1 : MYERS_FMA_SHIFT_WIDE;
}

// Whether the Ph (ph = true) or Mh shift of word j runs on the FMA pipe
// under policy FS. j is a constant after unrolling, so this folds away.
template <int FS>
__device__ __forceinline__ bool fma_word(int j, bool ph) {
  return FS == 1 || (FS == 2 && ph) || (FS == 3 && (j & 1)) || (FS == 4 && ph && (j & 1));
}

// (cur << 1) | (prev >> 31): the one-bit shift of a multi-word vector.
// On the ALU pipe: one funnel shift. On the FMA pipe: multiply-high and
// multiply-add by an opaque two -- fewer ALU instructions but more
// instructions and latency in all, which only pays where many warps are
// resident (narrow shapes).
__device__ __forceinline__ uint32_t shl1(uint32_t prev, uint32_t cur, Mul k, bool fma) {
  if (fma) return cur * k.two + __umulhi(prev, k.two);
  return __funnelshift_l(prev, cur, 1);
}

// One text column over W words. With HIN, bit 31 of inP / inM is the
// horizontal delta (+1 / -1) entering the bottom row (Myers' block rule);
// without, it is 0 (semi-global: row 0 of the DP is all zeros).
// topP / topM return the unshifted top words (bit 31 = delta out of the top row).
template <int W, bool HIN, int FS>
__device__ __forceinline__ void myers_column(const uint32_t (&eq)[W], uint32_t (&Pv)[W], uint32_t (&Mv)[W],
                                             uint32_t inP, uint32_t inM, uint32_t& topP, uint32_t& topM, Mul k) {
  uint32_t e0 = eq[0];
  if (HIN) e0 |= __umulhi(inM, k.two);  // inM >> 31
  uint32_t t[W], s[W];
  t[0] = e0 & Pv[0];
#pragma unroll
  for (int j = 1; j < W; ++j) t[j] = eq[j] & Pv[j];
  add_chain<W>(t, Pv, s, k.one);
  uint32_t php = HIN ? inP : 0u, mhp = HIN ? inM : 0u;
#pragma unroll
  for (int j = 0; j < W; ++j) {
    const uint32_t e = (j == 0) ? e0 : eq[j];
    const uint32_t pv = Pv[j], mv = Mv[j];
    const uint32_t xv = eq[j] | mv;
    const uint32_t xh = (s[j] ^ pv) | e;
    const uint32_t ph = mv | ~(xh | pv);
    const uint32_t mh = pv & xh;
    const uint32_t phs = shl1(php, ph, k, fma_word<FS>(j, true));
    const uint32_t mhs = shl1(mhp, mh, k, fma_word<FS>(j, false));
    Pv[j] = mhs | ~(xv | phs);
    Mv[j] = phs & xv;
    php = ph;
    mhp = mh;
  }
  topP = php;
  topM = mhp;
}

// Eight columns of one text word, single-lane shapes. TAIL masks columns >= n.
// Eight columns of one text word (codes 0..4 in its nibbles), single-lane
// shapes. TAIL masks columns >= n.
template <int W, bool TAIL, int UNR, int FS>
__device__ __forceinline__ void block8_single(uint32_t t, const char* __restrict__ slot, uint32_t (&Pv)[W],
                                              uint32_t (&Mv)[W], uint32_t& sc, uint32_t& kmin,
                                              uint32_t colbase, uint32_t n, Mul k) {
  const uint32_t kb = base_bytes<W, false>(k);
#pragma unroll UNR
  for (int u = 0; u < 8; ++u) {
    const uint32_t code = next_code(t, k);
    uint32_t eq[W];
    load_eq<W, false>(reinterpret_cast<const uint32_t*>(slot + code * kb), eq);
    uint32_t tp, tm;
    myers_column<W, false, FS>(eq, Pv, Mv, 0u, 0u, tp, tm, k);
#if MYERS_FMA_KEY
    sc = key_step(sc, tp, tm, k);  // sc: score key plus column
    if (!TAIL || colbase + (uint32_t)u < n) kmin = min(kmin, sc);
#else
    sc = score_step(sc, tp, tm, k);
    const uint32_t key = sc + colbase + (uint32_t)u;
    if (!TAIL || colbase + (uint32_t)u < n) kmin = min(kmin, key);
#endif
  }
}

// Eight systolic steps of a multi-lane shape. CHECKED: some lanes may be
// outside their candidate's columns (pipeline fill and drain, shorter
// candidates); otherwise every lane with work is inside (steady state), and
// lanes without work compute values nobody reads.
template <int W, bool CHECKED, int UNR, int FS>
__device__ __forceinline__ void block8_multi(uint32_t t, const char* __restrict__ slot, uint32_t (&Pv)[W],
                                             uint32_t (&Mv)[W], uint32_t& outP, uint32_t& outM, uint32_t& sc,
                                             uint32_t& kmin, uint32_t jbase, uint32_t n, bool work,
                                             uint32_t segmul, Mul k) {
  const uint32_t kb = base_bytes<W, true>(k);
#pragma unroll UNR
  for (int u = 0; u < 8; ++u) {
    const uint32_t code = next_code(t, k);
    uint32_t eq[W];
    load_eq<W, true>(reinterpret_cast<const uint32_t*>(slot + code * kb), eq);
    // the bottom lane of a segment takes no delta (segmul 0)
    const uint32_t inP = __shfl_up_sync(FULL_MASK, outP, 1) * segmul;
    const uint32_t inM = __shfl_up_sync(FULL_MASK, outM, 1) * segmul;
    const uint32_t j = jbase + (uint32_t)u;  // wraps when negative
#if MYERS_FMA_KEY
    // sc holds the key plus the step's column j; it advances every step
    if (!CHECKED || (work && j < n)) {
      myers_column<W, true, FS>(eq, Pv, Mv, inP, inM, outP, outM, k);
      sc = key_step(sc, outP, outM, k);
      kmin = min(kmin, sc);
    } else {
      sc = sc * k.one + k.one;
    }
#else
    if (!CHECKED || (work && j < n)) {
      myers_column<W, true, FS>(eq, Pv, Mv, inP, inM, outP, outM, k);
      sc = score_step(sc, outP, outM, k);
      kmin = min(kmin, sc + j);
    }
#endif
  }
}

// The result of a verified candidate from its (score << 16 | column) key,
// whose score carries the p padding rows. Under the cut-off contract a
// minimum above the bound is reported as {kNoMatch, kNoMatch}.
__device__ __forceinline__ uint2 result_of(const DevInputs& in, uint32_t kmin, uint32_t p, uint32_t m) {
  const uint32_t score = (kmin >> 16) - p;
  if (in.cut && score > d_cutoff_bound(m, in.cutoff)) return make_uint2(kNoMatch, kNoMatch);
  return make_uint2(kmin & 0xFFFFu, score);
}

// Finish a candidate whose DP ran over rows m of its query of mf bases. On a
// prefix (the cut-off's first pass, m < mf): every path to the query's last
// row crosses row m, at a cost of at least the prefix minimum, so a prefix
// minimum above the bound k settles the candidate as no match (Ukkonen's
// cut-off); otherwise it goes to the second pass, appended to its full shape's
// list.
__device__ __forceinline__ void finish(const DevInputs& in, uint32_t id, uint32_t kmin, uint32_t p, uint32_t m,
                                       uint32_t mf) {
  if (m < mf) {
    if ((kmin >> 16) - p > d_cutoff_bound(mf, in.cutoff)) {
      in.results[id] = make_uint2(kNoMatch, kNoMatch);
    } else {
      const uint32_t cfg = in.esc_cfg ? in.esc_cfg[id] : 0u;
      const uint32_t k = atomicAdd(&in.esc_state->count[cfg], 1u);
      in.esc_ids[in.esc_state->first[cfg] + k] = id;
    }
  } else {
    in.results[id] = result_of(in, kmin, p, m);
  }
}

// Multi-lane shapes: run the pipeline's ramp-up, steady state and drain as
// three loops instead of one loop that picks the checked or unchecked step
// per block of 8 columns.
#ifndef MYERS_MULTI_SPLIT
#define MYERS_MULTI_SPLIT 0
#endif

struct CandSetup {
  uint32_t id;
  uint32_t query;
  unsigned long long pos;
  uint32_t m;     // rows of the DP: the query's length, or the cut-off's first-pass prefix of it
  uint32_t mf;    // the query's length
  uint32_t pos_entry;
  uint32_t n;     // columns
  bool has;       // the segment holds a candidate
  bool qok;       // ... whose query can be staged (valid indices, 0 < m <= rows)
  bool work;      // ... that needs the DP
};

// Checks that keep every device read of a candidate inside its buffers.
// Returns 0 if the candidate can be verified, else the flag to raise.
__device__ __forceinline__ uint32_t check_query(const DevInputs& in, uint32_t query, uint2 q) {
  if (query >= in.num_queries) return kFlagBadQuery;
  if ((unsigned long long)q.x + ((q.y + 127u) >> 7) > in.num_entries) return kFlagBadEntry;
  return 0u;
}

// Resolve the candidate of this segment and write the result of candidates
// that need no DP (window out of range, empty query, unsupported size,
// invalid indices).
__device__ __forceinline__ CandSetup setup_candidate(const DevInputs& in, const uint32_t* __restrict__ ids,
                                                     uint32_t first, uint32_t cnt, int seg, int nseg,
                                                     int l, int rows) {
  CandSetup c;
  c.has = seg < nseg && (uint32_t)seg < cnt;
  c.id = 0;
  c.pos = 0;
  c.m = 0;
  c.mf = 0;
  c.pos_entry = 0;
  c.n = 0;
  c.query = 0;
  c.qok = false;
  c.work = false;
  if (c.has) {
    c.id = ids ? __ldg(ids + first + seg) : first + (uint32_t)seg;
    const Cand cd = in.cands[c.id];
    uint2 q = make_uint2(0u, 0u);
    uint32_t bad = 0u;
    if (cd.query < in.num_queries) q = __ldg(in.qinfo + cd.query);
    bad = check_query(in, cd.query, q);
    c.query = cd.query;
    c.pos = cd.position;
    c.pos_entry = q.x;
    c.mf = q.y;
    c.m = in.prefix ? d_prefix_rows(c.mf, in.cutoff, in.prefix_mult) : c.mf;
    const uint32_t wb = d_window_bases(c.mf, in.distance);
    const bool valid = bad == 0u && c.pos < in.ref_size && (in.ref_size - c.pos) > (unsigned long long)wb;
    c.n = in.exact ? wb : 8u * d_window_words(wb);
    const bool fits = c.m <= (uint32_t)rows && c.n <= kMaxColumns;
    c.qok = bad == 0u && c.m > 0 && c.m <= (uint32_t)rows;
    c.work = valid && c.m > 0 && fits;
    if (!c.work && l == 0) {
      in.results[c.id] = (valid && c.m == 0) ? make_uint2(0u, 0u) : make_uint2(0u, kNoResult);
      if (bad) atomicOr(in.flags, bad);
      else if (valid && c.m > 0 && !fits) atomicOr(in.flags, kFlagUnsupported);
    }
  }
  return c;
}

// UNR: how far the 8 columns of a text word are unrolled -- fully for the
// one-shape plain kernels; partly in the persistent kernel, whose code holds
// every shape and would otherwise overflow the instruction cache.
template <int W, bool MULTI, int UNR = 8, int FS = 0>
__device__ __forceinline__ void process_tile(const DevInputs& in, const uint32_t* __restrict__ ids, uint32_t first,
                                             uint32_t cnt, int L, uint32_t* __restrict__ wsmem, int lane) {
  using Lay = Layout<W, MULTI>;
  const int Lr = MULTI ? L : 1;
  const int nseg = MULTI ? 32 / L : 32;
  const int seg = MULTI ? lane / L : lane;
  const int l = MULTI ? lane - seg * L : 0;
  const int LW = Lr * W;
  const int rows = 32 * LW;

  const CandSetup c = setup_candidate(in, ids, first, cnt, seg, nseg, l, rows);

  // One slot per run of segments with the same read: a run starts where the
  // read differs from the previous segment's.
  const uint32_t qkey = c.has ? c.query : 0xFFFFFFFFu;
  const uint32_t qprev = __shfl_up_sync(FULL_MASK, qkey, Lr);
  const bool starts = c.has && (seg == 0 || qprev != qkey);
  const unsigned run_starts = __ballot_sync(FULL_MASK, starts && l == 0);
  const int my_bit = seg * Lr;
  const int run = __popc(run_starts & (my_bit >= 31 ? FULL_MASK : ((2u << my_bit) - 1u))) - 1;
  const int distinct = __popc(run_starts);
  // more distinct reads than slots (single-lane wide shapes only): rounds
  const int rounds = (distinct + Lay::SLOTS / Lr - 1) / (Lay::SLOTS / Lr);

  const uint32_t p = (uint32_t)rows - c.m;
  const long long q0 = (long long)(in.exact ? c.pos : (c.pos & ~7ull)) - l;
  const long long b0 = q0 >> 3;
  const uint32_t sh = 4u * (uint32_t)(q0 & 7);
  const Mul k = make_mul(in);

  for (int r = 0; r < rounds; ++r) {
    const int slot = run - r * (Lay::SLOTS / Lr);
    const bool in_round = c.has && slot >= 0 && slot < Lay::SLOTS / Lr;
    const int col = in_round ? slot * Lr + l : l;
    uint32_t* lane_part = wsmem + col * 4;
    if (in_round && starts && c.qok) stage_lane<W, MULTI>(lane_part, in.peq, c.pos_entry, c.m, LW, l);
    __syncwarp();
    const bool work = c.work && in_round;
    const char* slotp = reinterpret_cast<const char*>(lane_part);

    uint32_t Pv[W], Mv[W];
#pragma unroll
    for (int j = 0; j < W; ++j) {
      Pv[j] = 0xFFFFFFFFu;
      Mv[j] = 0u;
    }
    uint32_t sc = (uint32_t)rows << 16;  // score + p = rows at column -1
    uint32_t kmin = sc;                  // (score, column) = (m, 0) before any column
#if MYERS_FMA_KEY
    // the key counter: score << 16 plus the column, one column before the
    // first (the lane's first step is column -l on multi-lane shapes)
    sc -= 1u + (uint32_t)l;
#endif

    if constexpr (!MULTI) {
      if (work) {
        uint32_t lo = ref_load(in.ref, b0, in.ref_words);
        uint32_t hi = ref_load(in.ref, b0 + 1, in.ref_words);
        const uint32_t nfull = c.n >> 3;
        uint32_t i = 0;
        for (; i < nfull; ++i) {
          const uint32_t t = sanitize_codes(__funnelshift_r(lo, hi, sh));
          lo = hi;
          hi = ref_load(in.ref, b0 + (long long)i + 2, in.ref_words);
          block8_single<W, false, UNR, FS>(t, slotp, Pv, Mv, sc, kmin, 8u * i, c.n, k);
        }
        if (c.n & 7u) {
          const uint32_t t = sanitize_codes(__funnelshift_r(lo, hi, sh));
          block8_single<W, true, UNR, FS>(t, slotp, Pv, Mv, sc, kmin, 8u * i, c.n, k);
        }
        finish(in, c.id, kmin, p, c.m, c.mf);
      }
    } else {
      uint32_t steps = work ? c.n + (uint32_t)L - 1u : 0u;
      steps = __reduce_max_sync(FULL_MASK, steps);
      // steps [L-1, n_min) have every lane with work inside its columns
      const uint32_t n_min = __reduce_min_sync(FULL_MASK, work ? c.n : 0xFFFFFFFFu);
      const uint32_t nblk = (steps + 7u) >> 3;
      uint32_t lo = ref_load(in.ref, b0, in.ref_words);
      uint32_t hi = ref_load(in.ref, b0 + 1, in.ref_words);
      uint32_t outP = 0u, outM = 0u;
      const uint32_t segmul = (uint32_t)min(l, 1);
#if MYERS_MULTI_SPLIT
      // blocks [i_lo, i_hi) have every lane with work inside its columns:
      // 8i + 1 >= L and 8i + 8 <= n_min. The ramp-up, the steady state and the
      // drain run as separate loops, so no block tests which one it is in.
      const uint32_t i_lo = min(((uint32_t)L + 6u) >> 3, nblk);
      const uint32_t i_hi = max(min(n_min >> 3, nblk), i_lo);
      uint32_t i = 0;
      for (; i < i_lo; ++i) {
        const uint32_t t = sanitize_codes(__funnelshift_r(lo, hi, sh));
        lo = hi;
        hi = ref_load(in.ref, b0 + (long long)i + 2, in.ref_words);
        block8_multi<W, true, UNR, FS>(t, slotp, Pv, Mv, outP, outM, sc, kmin, 8u * i - (uint32_t)l, c.n, work,
                                       segmul, k);
      }
      for (; i < i_hi; ++i) {
        const uint32_t t = sanitize_codes(__funnelshift_r(lo, hi, sh));
        lo = hi;
        hi = ref_load(in.ref, b0 + (long long)i + 2, in.ref_words);
        block8_multi<W, false, UNR, FS>(t, slotp, Pv, Mv, outP, outM, sc, kmin, 8u * i - (uint32_t)l, c.n, work,
                                        segmul, k);
      }
      for (; i < nblk; ++i) {
        const uint32_t t = sanitize_codes(__funnelshift_r(lo, hi, sh));
        lo = hi;
        hi = ref_load(in.ref, b0 + (long long)i + 2, in.ref_words);
        block8_multi<W, true, UNR, FS>(t, slotp, Pv, Mv, outP, outM, sc, kmin, 8u * i - (uint32_t)l, c.n, work,
                                       segmul, k);
      }
#else
      for (uint32_t i = 0; i < nblk; ++i) {
        const uint32_t t = sanitize_codes(__funnelshift_r(lo, hi, sh));
        lo = hi;
        hi = ref_load(in.ref, b0 + (long long)i + 2, in.ref_words);
        const uint32_t jbase = 8u * i - (uint32_t)l;
        if (8u * i + 1u >= (uint32_t)L && 8u * i + 8u <= n_min)
          block8_multi<W, false, UNR, FS>(t, slotp, Pv, Mv, outP, outM, sc, kmin, jbase, c.n, work, segmul, k);
        else
          block8_multi<W, true, UNR, FS>(t, slotp, Pv, Mv, outP, outM, sc, kmin, jbase, c.n, work, segmul, k);
      }
#endif
      if (work && l == L - 1) finish(in, c.id, kmin, p, c.m, c.mf);
    }
    __syncwarp();
  }
}

template <int W, bool MULTI>
__host__ __device__ constexpr uint32_t warp_words() {
  return (uint32_t)Layout<W, MULTI>::WORDS;
}

// Plain launch: one shape over a contiguous range of (sorted) candidates.
// Warps take warp tiles from a device counter (`next`, zero at launch), so
// SMs that run ahead take more tiles and the launch ends evenly.
template <int W, bool MULTI>
__global__ void __launch_bounds__(128) k_plain(DevInputs in, const uint32_t* __restrict__ ids,
                                               const BucketState* __restrict__ st, int cfg, uint32_t first,
                                               uint32_t count, int L, uint32_t* __restrict__ next) {
  extern __shared__ __align__(16) uint32_t smem[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  if (st != nullptr) {
    first = st->first[cfg];
    count = st->count[cfg];
  }
  const int nseg = MULTI ? 32 / L : 32;
  uint32_t* wsmem = smem + wib * warp_words<W, MULTI>();
  const uint32_t tiles = (count + nseg - 1) / nseg;
  while (true) {
    uint32_t t = 0;
    if (lane == 0) t = atomicAdd(next, 1u);
    t = __shfl_sync(FULL_MASK, t, 0);
    if (t >= tiles) break;
    const uint32_t f = t * nseg;
    const uint32_t cnt = min((uint32_t)nseg, count - f);
    process_tile<W, MULTI, 8, fma_shift<W, MULTI, false>()>(in, ids, first + f, cnt, L, wsmem, lane);
  }
}

// ---- length bucketing on the device ----

// With TWO (the cut-off's first pass) a candidate is classified by its
// prefix's word count under `plan`, and, when the prefix covers only part of
// its query, by its full word count under `plan2` into in.esc_cfg, counted in
// in.esc_state->cursor (the second pass's layout).
template <bool TWO>
__global__ void k_classify(DevInputs in, const __grid_constant__ PlanTable plan,
                           const __grid_constant__ PlanTable plan2, BucketState* st,
                           uint8_t* __restrict__ cfg_of_cand) {
  const int lane = threadIdx.x & 31;
  const uint32_t n = in.num_cands;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; base < n; base += stride) {
    const uint32_t i = base + lane;
    uint32_t cfg = kNoCfg;
    if (i < n) {
      const Cand cd = in.cands[i];
      uint2 q = make_uint2(0u, 0u);
      if (cd.query < in.num_queries) q = __ldg(in.qinfo + cd.query);
      const uint32_t bad = check_query(in, cd.query, q);
      const uint32_t mf = q.y;
      const uint32_t m = TWO ? d_prefix_rows(mf, in.cutoff, in.prefix_mult) : mf;
      const uint32_t wb = d_window_bases(mf, in.distance);
      const bool valid = bad == 0u && cd.position < in.ref_size &&
                         (in.ref_size - cd.position) > (unsigned long long)wb;
      const uint32_t ncol = in.exact ? wb : 8u * d_window_words(wb);
      if (bad) {
        in.results[i] = make_uint2(0u, kNoResult);
        atomicOr(in.flags, bad);
      } else if (!valid) {
        in.results[i] = make_uint2(0u, kNoResult);
      } else if (m == 0) {
        in.results[i] = make_uint2(0u, 0u);
      } else if (mf > kMaxWords * 32 || ncol > kMaxColumns || plan.cfg_of_words[(m + 31) >> 5] == kNoCfg ||
                 (TWO && m < mf && plan2.cfg_of_words[(mf + 31) >> 5] == kNoCfg)) {
        in.results[i] = make_uint2(0u, kNoResult);
        atomicOr(in.flags, kFlagUnsupported);
      } else {
        cfg = plan.cfg_of_words[(m + 31) >> 5];
        if (TWO && m < mf) {
          const uint32_t c2 = plan2.cfg_of_words[(mf + 31) >> 5];
          in.esc_cfg[i] = (uint8_t)c2;
          atomicAdd(&in.esc_state->cursor[c2], 1u);
        }
      }
      cfg_of_cand[i] = (uint8_t)cfg;
    }
    const unsigned peers = __match_any_sync(FULL_MASK, cfg);
    if (cfg != kNoCfg && lane == __ffs(peers) - 1) atomicAdd(&st->count[cfg], (uint32_t)__popc(peers));
  }
}

// The second pass's layout: each full-length shape's list starts where the
// candidates counted for it in the classification end up at most; the lists
// fill as the first pass appends to them.
__global__ void k_plan_escalation(const __grid_constant__ PlanTable plan2, BucketState* esc) {
  if (threadIdx.x != 0) return;
  uint32_t acc = 0;
  for (uint32_t c = 0; c < plan2.num_cfg; ++c) {
    esc->first[c] = acc;
    acc += esc->cursor[c];
    esc->count[c] = 0;
    esc->next[c] = 0;
  }
}

// The second pass's tiles on the persistent path, once the first pass has
// filled the lists: each shape's tiles from its list length, the persistent
// kernel's tile count and a fresh work counter.
__global__ void k_plan_tiles(const __grid_constant__ PlanTable plan2, BucketState* esc) {
  if (threadIdx.x != 0) return;
  uint32_t tiles = 0;
  for (uint32_t c = 0; c < plan2.num_cfg; ++c) {
    const Shape s = plan2.shape[c];
    const uint32_t nseg = (s.variant >= kNumSingle) ? 32u / s.L : 32u;
    if (c == plan2.num_batched) esc->total_tiles = tiles;
    esc->tile_start[c] = tiles;
    tiles += (esc->count[c] + nseg - 1) / nseg;
  }
  esc->tile_start[plan2.num_cfg] = tiles;
  if (plan2.num_batched >= plan2.num_cfg) esc->total_tiles = tiles;
  esc->queue = 0;
}

__global__ void k_plan(const __grid_constant__ PlanTable plan, BucketState* st) {
  if (threadIdx.x != 0) return;
  uint32_t acc = 0, tiles = 0;
  for (uint32_t c = 0; c < plan.num_cfg; ++c) {
    const Shape s = plan.shape[c];
    const uint32_t nseg = (s.variant >= kNumSingle) ? 32u / s.L : 32u;
    if (c == plan.num_batched) st->total_tiles = tiles;
    st->first[c] = acc;
    st->cursor[c] = 0;
    st->tile_start[c] = tiles;
    tiles += (st->count[c] + nseg - 1) / nseg;
    acc += st->count[c];
  }
  st->tile_start[plan.num_cfg] = tiles;
  if (plan.num_batched >= plan.num_cfg) st->total_tiles = tiles;
  st->queue = 0;
}

// Stable within each warp's 32 consecutive candidates, so the candidates of
// one read (adjacent in the input) mostly stay adjacent.
__global__ void k_scatter(uint32_t n, const uint8_t* __restrict__ cfg_of_cand, BucketState* st,
                          uint32_t* __restrict__ ids) {
  const int lane = threadIdx.x & 31;
  const uint32_t stride = gridDim.x * blockDim.x;
  for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; base < n; base += stride) {
    const uint32_t i = base + lane;
    const uint32_t cfg = i < n ? cfg_of_cand[i] : kNoCfg;
    const unsigned peers = __match_any_sync(FULL_MASK, cfg);
    const int leader = __ffs(peers) - 1;
    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    uint32_t b = 0;
    if (cfg != kNoCfg && lane == leader) b = atomicAdd(&st->cursor[cfg], (uint32_t)__popc(peers));
    b = __shfl_sync(FULL_MASK, b, leader);
    if (cfg != kNoCfg) ids[st->first[cfg] + b + rank] = i;
  }
}

// ---- the persistent batched kernel ----

constexpr uint32_t cmax(uint32_t a, uint32_t b) { return a > b ? a : b; }
// the largest batched shape's footprint
constexpr uint32_t kBatchedWarpWords =
    cmax(cmax(warp_words<32, false>(), warp_words<16, false>()), warp_words<kBatchedMaxMultiW, true>());

#ifndef MYERS_BATCHED_UNROLL
#define MYERS_BATCHED_UNROLL 2
#endif

template <int V>
__device__ __forceinline__ void dispatch_one(const DevInputs& in, const uint32_t* ids, uint32_t f, uint32_t cnt,
                                             int L, uint32_t* wsmem, int lane) {
  if constexpr (V < kNumSingle) {
    process_tile<V + 1, false, MYERS_BATCHED_UNROLL, fma_shift<V + 1, false, true>()>(in, ids, f, cnt, L, wsmem,
                                                                                       lane);
  } else {
    if constexpr (kMultiW[V - kNumSingle] <= kBatchedMaxMultiW)
      process_tile<kMultiW[V - kNumSingle], true, MYERS_BATCHED_UNROLL,
                   fma_shift<kMultiW[V - kNumSingle], true, true>()>(in, ids, f, cnt, L, wsmem, lane);
  }
}

template <int... Vs>
__device__ __forceinline__ void dispatch(int v, const DevInputs& in, const uint32_t* ids, uint32_t f, uint32_t cnt,
                                         int L, uint32_t* wsmem, int lane, std::integer_sequence<int, Vs...>) {
  ((v == Vs ? (dispatch_one<Vs>(in, ids, f, cnt, L, wsmem, lane), 0) : 0), ...);
}

// Each warp pulls the next tile index from the device queue; tiles are
// ordered by shape, most expensive shape first, so the long candidates start
// early and the short ones fill the tail.
// At least three blocks of four warps per SM. ptxas then takes 159
// registers (three blocks fit); a bound of four holds it at 115 without a
// spill, and measured 0.2-0.4% slower on long and mixed reads.
#ifndef MYERS_BATCHED_MIN_BLOCKS
#define MYERS_BATCHED_MIN_BLOCKS 3
#endif
__global__ void __launch_bounds__(128, MYERS_BATCHED_MIN_BLOCKS) k_batched(DevInputs in, const uint32_t* __restrict__ ids,
                                                 const __grid_constant__ PlanTable plan, BucketState* st) {
  extern __shared__ __align__(16) uint32_t smem[];
  __shared__ uint32_t s_tile_start[kMaxCfg + 1];
  __shared__ uint32_t s_first[kMaxCfg];
  __shared__ uint32_t s_count[kMaxCfg];
  __shared__ Shape s_shape[kMaxCfg];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t ncfg = plan.num_batched;
  for (uint32_t c = threadIdx.x; c < ncfg; c += blockDim.x) {
    s_tile_start[c] = st->tile_start[c];
    s_first[c] = st->first[c];
    s_count[c] = st->count[c];
    s_shape[c] = plan.shape[c];
  }
  __syncthreads();
  const uint32_t total = st->total_tiles;
  uint32_t* wsmem = smem + wib * kBatchedWarpWords;
  while (true) {
    uint32_t t = 0;
    if (lane == 0) t = atomicAdd(&st->queue, 1u);
    t = __shfl_sync(FULL_MASK, t, 0);
    if (t >= total) break;
    // last shape whose first tile is <= t
    uint32_t lo = 0, hi = ncfg - 1;
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (s_tile_start[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    const Shape s = s_shape[lo];
    const int L = s.L;
    const uint32_t nseg = (s.variant >= kNumSingle) ? 32u / (uint32_t)L : 32u;
    const uint32_t f = (t - s_tile_start[lo]) * nseg;
    const uint32_t cnt = min(nseg, s_count[lo] - f);
    dispatch(s.variant, in, ids, s_first[lo] + f, cnt, L, wsmem, lane,
             std::make_integer_sequence<int, kNumVariants>{});
  }
}

// Integer-ALU peak probe: eight independent chains of 3-input logic ops per
// thread (the instruction class of the Myers column), written out so the
// work cannot be removed.
__global__ void k_lop3_probe(uint32_t* out, int iters) {
  uint32_t a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = threadIdx.x * (k + 3) + blockIdx.x;
  uint32_t b = threadIdx.x ^ 0x5A5A5A5Au;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
#pragma unroll
      for (int k = 0; k < 8; ++k)
        asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(a[k]) : "r"(a[(k + 1) & 7]), "r"(b));
    }
  }
  uint32_t x = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) x ^= a[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = x;
}

// ---- host-side launchers ----

using PlainFn = void (*)(DevInputs, const uint32_t*, const BucketState*, int, uint32_t, uint32_t, int, uint32_t*);

template <int V>
constexpr PlainFn plain_fn() {
  if constexpr (V < kNumSingle) return &k_plain<V + 1, false>;
  else return &k_plain<kMultiW[V - kNumSingle], true>;
}

template <int... Vs>
constexpr auto make_plain_table(std::integer_sequence<int, Vs...>) {
  struct T { PlainFn f[sizeof...(Vs)]; };
  return T{{plain_fn<Vs>()...}};
}

static const auto kPlainTable = make_plain_table(std::make_integer_sequence<int, kNumVariants>{});

uint32_t warp_smem_bytes(int v, int) {
  const int W = variant_W(v);
  const int slots = variant_multi(v) ? 32 : (W > 16 ? 16 : 32);
  const int ncol = ((slots + 7) / 8) * 8 + 1;
  return (uint32_t)(((W + 3) / 4) * 5 * ncol * 4 * 4);
}

static int blocks_per_sm(const void* fn, int threads, size_t smem) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, threads, smem) != cudaSuccess || nb < 1) nb = 1;
  return nb;
}

cudaError_t launch_plain(int v, int L, const DevInputs& in, const uint32_t* d_ids, const BucketState* d_state,
                         int cfg, uint32_t first, uint32_t count, uint32_t* d_next, cudaStream_t s, int num_sms) {
  const PlainFn fn = kPlainTable.f[v];
  const int threads = 128;
  const int Lr = variant_multi(v) ? L : 1;
  const size_t smem = (size_t)warp_smem_bytes(v, Lr) * (threads / 32);
  cudaError_t e = cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  const int nb = blocks_per_sm((const void*)fn, threads, smem);
  uint32_t grid = (uint32_t)(num_sms * nb);
  if (d_state == nullptr) {
    const uint32_t nseg = variant_multi(v) ? 32u / (uint32_t)L : 32u;
    const uint32_t tiles = (count + nseg - 1) / nseg;
    const uint32_t need = (tiles + threads / 32 - 1) / (threads / 32);
    if (need < grid) grid = need;
    if (grid == 0) return cudaSuccess;
  }
  fn<<<grid, threads, smem, s>>>(in, d_ids, d_state, cfg, first, count, Lr, d_next);
  return cudaGetLastError();
}

int launch_bucketing(const DevInputs& in, const PlanTable& plan, BucketState* d_state, uint8_t* d_cfg_of_cand,
                     uint32_t* d_ids, cudaStream_t s, int num_sms, cudaError_t* err) {
  const int threads = 256;
  const uint32_t need = (in.num_cands + threads - 1) / threads;
  uint32_t grid = (uint32_t)num_sms * 8;
  if (need < grid) grid = need > 0 ? need : 1;
  k_classify<false><<<grid, threads, 0, s>>>(in, plan, plan, d_state, d_cfg_of_cand);
  k_plan<<<1, 32, 0, s>>>(plan, d_state);
  k_scatter<<<grid, threads, 0, s>>>(in.num_cands, d_cfg_of_cand, d_state, d_ids);
  *err = cudaGetLastError();
  return 3;
}

int launch_bucketing_cutoff(const DevInputs& in, const PlanTable& plan, const PlanTable& plan2,
                            BucketState* d_state, uint8_t* d_cfg_of_cand, uint32_t* d_ids, cudaStream_t s,
                            int num_sms, cudaError_t* err) {
  const int threads = 256;
  const uint32_t need = (in.num_cands + threads - 1) / threads;
  uint32_t grid = (uint32_t)num_sms * 8;
  if (need < grid) grid = need > 0 ? need : 1;
  k_classify<true><<<grid, threads, 0, s>>>(in, plan, plan2, d_state, d_cfg_of_cand);
  k_plan<<<1, 32, 0, s>>>(plan, d_state);
  k_plan_escalation<<<1, 32, 0, s>>>(plan2, in.esc_state);
  k_scatter<<<grid, threads, 0, s>>>(in.num_cands, d_cfg_of_cand, d_state, d_ids);
  *err = cudaGetLastError();
  return 4;
}

cudaError_t launch_plan_tiles(const PlanTable& plan2, BucketState* d_esc_state, cudaStream_t s) {
  k_plan_tiles<<<1, 32, 0, s>>>(plan2, d_esc_state);
  return cudaGetLastError();
}

cudaError_t launch_batched(const DevInputs& in, const uint32_t* d_ids, const PlanTable& plan,
                           BucketState* d_state, cudaStream_t s, int num_sms, uint32_t max_tiles) {
  const int threads = 128;
  const size_t smem = (size_t)kBatchedWarpWords * 4 * (threads / 32);
  cudaError_t e = cudaFuncSetAttribute((const void*)k_batched, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  const int nb = blocks_per_sm((const void*)k_batched, threads, smem);
  uint32_t grid = (uint32_t)(num_sms * nb);
  const uint32_t need = (max_tiles + threads / 32 - 1) / (threads / 32);
  if (need < grid) grid = need > 0 ? need : 1;
  k_batched<<<grid, threads, smem, s>>>(in, d_ids, plan, d_state);
  return cudaGetLastError();
}

cudaError_t load_batched_path_kernels() {
  cudaFuncAttributes a;
  const void* fns[] = {(const void*)k_classify<false>, (const void*)k_plan, (const void*)k_scatter,
                       (const void*)k_batched};
  for (const void* f : fns) {
    const cudaError_t e = cudaFuncGetAttributes(&a, f);
    if (e != cudaSuccess) return e;
  }
  for (int v = 0; v < kNumVariants; ++v) {
    if (batched_supports(v)) continue;  // shapes the persistent kernel does not carry get plain launches
    const cudaError_t e = cudaFuncGetAttributes(&a, (const void*)kPlainTable.f[v]);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_lop3_probe(uint32_t* d_out, int blocks, int threads, int iters, cudaStream_t s) {
  k_lop3_probe<<<blocks, threads, 0, s>>>(d_out, iters);
  return cudaGetLastError();
}

}  // namespace myers

// ---- packers on the device ----

namespace myers {

// ASCII base -> code: A0 C1 G2 T3 (either case), anything else 4
// (src-api/genReference-4bits.c:21-40, genCandidate-reorder.c:237-256).
__device__ __forceinline__ uint32_t ascii_code(uint32_t b) {
  const uint32_t u = b & 0xDFu;  // upper case
  return u == 'A' ? 0u : u == 'C' ? 1u : u == 'G' ? 2u : u == 'T' ? 3u : 4u;
}

// One thread per 32-base word of a read: the five 32-bit bitmaps of that
// word. Bits past the read's end are 0 (src-api/genCandidate-reorder.c:258-317).
__global__ void k_pack_peq(const uint8_t* __restrict__ ascii, unsigned long long ascii_bytes,
                           const unsigned long long* __restrict__ offsets, const uint2* __restrict__ qinfo,
                           uint32_t num_reads, uint32_t* __restrict__ peq, uint32_t num_entries,
                           uint32_t* __restrict__ flags) {
  const uint32_t stride = gridDim.x * (blockDim.x / 32);
  const int lane = threadIdx.x & 31;
  for (uint32_t r = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); r < num_reads; r += stride) {
    const uint2 q = qinfo[r];
    const unsigned long long o = offsets[r];
    const uint32_t m = q.y;
    const uint32_t nwords = ((m + 127) / 128) * 4;  // whole entries, padding words zeroed
    const unsigned long long o1 = offsets[r + 1];
    if ((unsigned long long)q.x + nwords / 4 > num_entries || o1 < o || o1 - o < m || o1 > ascii_bytes) {
      if (lane == 0) atomicOr(flags, kFlagBadEntry);
      continue;
    }
    for (uint32_t w = lane; w < nwords; w += 32) {
      uint32_t bm[5] = {0u, 0u, 0u, 0u, 0u};
      const uint32_t b0 = w * 32;
      for (uint32_t i = 0; i < 32 && b0 + i < m; ++i) bm[ascii_code(ascii[o + b0 + i])] |= 1u << i;
      uint32_t* e = peq + (size_t)(q.x + w / 4) * 20;
#pragma unroll
      for (int c = 0; c < 5; ++c) e[c * 4 + (w & 3)] = bm[c];
    }
  }
}

// One thread per packed word: eight bases, base i in bits 4*(i%8); bases at
// or past n are N (src-api/genReference-4bits.c:43-72).
__global__ void k_pack_reference(const uint8_t* __restrict__ ascii, unsigned long long n, uint32_t* __restrict__ words,
                                 unsigned long long nwords) {
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long w = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; w < nwords; w += stride) {
    uint32_t v = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const unsigned long long i = w * 8 + k;
      v |= (i < n ? ascii_code(ascii[i]) : 4u) << (4 * k);
    }
    words[w] = v;
  }
}

cudaError_t launch_pack_peq(const uint8_t* ascii, unsigned long long ascii_bytes, const unsigned long long* offsets,
                            const uint2* qinfo, uint32_t num_reads, uint32_t* peq, uint32_t num_entries,
                            uint32_t* flags, cudaStream_t s, int num_sms) {
  if (num_reads == 0) return cudaSuccess;
  uint32_t grid = (num_reads + 7) / 8;
  if (grid > (uint32_t)num_sms * 16) grid = (uint32_t)num_sms * 16;
  k_pack_peq<<<grid, 256, 0, s>>>(ascii, ascii_bytes, offsets, qinfo, num_reads, peq, num_entries, flags);
  return cudaGetLastError();
}

cudaError_t launch_pack_reference(const uint8_t* ascii, unsigned long long n, uint32_t* words,
                                  unsigned long long nwords, cudaStream_t s, int num_sms) {
  if (nwords == 0) return cudaSuccess;
  unsigned long long grid = (nwords + 255) / 256;
  if (grid > (unsigned long long)num_sms * 32) grid = (unsigned long long)num_sms * 32;
  k_pack_reference<<<(unsigned)grid, 256, 0, s>>>(ascii, n, words, nwords);
  return cudaGetLastError();
}

}  // namespace myers
