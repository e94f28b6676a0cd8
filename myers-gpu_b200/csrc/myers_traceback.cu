// Traceback of accepted candidates: the alignment (start column and
// run-length CIGAR) behind a verification result. No counterpart in the
// reference, which returns (column, score) only.
//
// Definition (the oracle states the same): for a candidate with result
// (column c, score s), s <= maxScore, the alignment is the path through the
// semi-global edit-distance matrix from (m, c+1) back to row 0 that takes, at
// each cell, the first of: the diagonal ('=' or 'X'), the query base alone
// ('I'), the text base alone ('D') that is consistent with the matrix.
//
// Two passes per chunk of traced candidates:
//  * k_tb_forward: a candidate's rows are spread over L lanes of W words (W
//    >= 8, one choice per call), a warp holding 32/S candidates in segments
//    of S lanes. Lanes run as a systolic pipeline (lane r processes column
//    t - r at step t, taking the horizontal delta of its bottom row from
//    lane r-1 through a shuffle). The pass recomputes the window's columns
//    1..c+1 and stores, for each column, the words of the diagonal band the
//    path can use: Pv/Mv (vertical deltas) and Ph/Mh (horizontal deltas into
//    the column). A path of cost s from (0, a) to (m, c+1) has j - i within
//    s of (c+1) - m at every cell, and consumes at most m + s text bases, so
//    columns before c+1-m-s and rows outside that band are never read back.
//  * k_tb_walk: one thread per candidate walks back with bit lookups: the
//    diagonal is consistent iff h(i,j) + v(i,j-1) equals the mismatch cost,
//    the query base alone iff v(i,j) = +1. The columns to the left are
//    fetched four ahead, the PEQ words once per 32 rows and the text once
//    per 8 columns, so a step rarely waits on a load it has just issued.
// Each traced candidate reserves its own band store (256-byte units) when it
// is selected: one 64-bit atomic per warp takes both its place in the list
// and its offset, so offsets rise with list order. A chunk is the range of
// the list whose offsets fall in one window of half the scratch (found by
// binary search); chunks alternate between the two halves, the walk of one
// (latency-bound) running on a second stream beside the forward pass of the
// next (ALU-bound).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <cuda_runtime.h>

#include "myers-interface.h"
#include "myers_device.cuh"
#include "myers_internal.h"

namespace myers {

static constexpr uint32_t kTbNotTraced = 0xFFFFFFFFu;
static constexpr uint32_t kTbInconsistent = 0xFFFFFFFEu;
static constexpr uint32_t kOpEq = 7, kOpX = 8, kOpI = 1, kOpD = 2;  // SAM codes

// Columns the walk fetches ahead of the one it is in.
#ifndef MYERS_TB_AHEAD
#define MYERS_TB_AHEAD 4
#endif
// The walk's band loads: 0 through L2 only (ld.global.cg); 1 through the
// read-only path, cached in L1 as well (the bands are written by the forward
// pass, an earlier kernel).
#ifndef MYERS_TB_LDG
#define MYERS_TB_LDG 0
#endif

// packed = traced count << 36 | their band stores in 256-byte units
static constexpr unsigned kTbUnitShift = 8;
static constexpr unsigned kTbCountShift = 36;
static constexpr unsigned long long kTbUnitMask = (1ull << kTbCountShift) - 1ull;

struct TbState {
  unsigned long long packed;
  unsigned int max_words;  // longest query among them (32-bit words)
  unsigned int max_units;  // largest band store (256-byte units), for any words per lane
  unsigned int max_inv_words;  // ~(shortest query's words): zero-initialised like the rest
  unsigned int next[2][2];  // per scratch half: work counters of the forward pass and the walk
};

struct TbArgs {
  const uint32_t* peq;
  const uint2* qinfo;
  const Cand* cands;
  const uint2* results;
  const uint32_t* ref;
  unsigned long long ref_size;
  unsigned long long ref_words;
  uint32_t num_cands, num_queries, num_entries;
  float distance;
  int exact;
  uint32_t max_score;
  uint32_t* ops;
  uint32_t max_ops;
  uint4* alns;  // {startColumn, numOps, score, endColumn}
  const uint32_t* ids;             // traced candidates, in reservation order
  const unsigned long long* offs;  // their band stores' offsets (units), rising
  uint32_t count;                  // traced candidates
  TbState* st;
  unsigned char* scratch;          // this chunk's half
  unsigned long long unit_lo, unit_hi;  // this chunk: offsets in [unit_lo, unit_hi)
  unsigned int* next;              // this chunk's counters: [0] forward groups, [1] walk candidates
  int fwd_counter;                 // the forward pass takes groups from next[0] (else a static share)
  uint32_t wl;   // words per lane of this call
  uint32_t seg;  // lanes per candidate segment (power of two)
};

// Geometry of one traced candidate (identical in all three kernels).
struct TbGeom {
  uint32_t m, pos_entry, s, c1;  // c1 = end column + 1 (1-based)
  uint32_t L, tw, p;             // lanes, L*wl words, padding rows
  uint32_t a0, B;                // first kept column, band words per column
  int off;                       // c1 - m: the path's final diagonal
  unsigned long long start;      // window start (bases)
};

// Words per lane for queries of up to `words` words: 8 up to 256 words
// (8192 bases), then doubling, so that a query takes at most 32 lanes.
static inline uint32_t tb_words_per_lane(uint32_t words) {
  uint32_t wl = 8;
  while (32u * wl < words) wl <<= 1;
  return wl;
}

// Band words per column for score s, before the cap at the query's words.
__device__ __forceinline__ uint32_t tb_band_words(uint32_t s) { return (2u * s + 3u + 31u) / 32u + 1u; }

// Band: the first stored word of column j1 (1-based).
__device__ __forceinline__ uint32_t tb_xlo(const TbGeom& g, uint32_t j1) {
  const int row_lo = (int)j1 - g.off - (int)g.s - 1;  // lowest query row the path can use, minus one
  const int bit = (int)g.p + (row_lo < 1 ? 1 : row_lo) - 1;
  const uint32_t x = (uint32_t)bit >> 5;
  return x + g.B > g.tw ? g.tw - g.B : x;
}

// Returns 0 and fills g when the candidate is traced; else the numOps code
// of its record (not traced / inconsistent), or 1 for an empty query. With
// wl = 0 the lane layout (L, tw, p, B) is left out (the selection pass).
__device__ __forceinline__ uint32_t tb_setup(const TbArgs& a, uint32_t id, uint2 res, uint32_t wl, TbGeom& g) {
  if (res.y == kNoResult || res.y > a.max_score) return kTbNotTraced;
  const Cand cd = a.cands[id];
  if (cd.query >= a.num_queries) return kTbInconsistent;
  const uint2 q = __ldg(a.qinfo + cd.query);
  if ((unsigned long long)q.x + ((q.y + 127u) >> 7) > a.num_entries) return kTbInconsistent;
  const uint32_t wb = d_window_bases(q.y, a.distance);
  if (!(cd.position < a.ref_size && a.ref_size - cd.position > (unsigned long long)wb)) return kTbInconsistent;
  const uint32_t n = a.exact ? wb : 8u * d_window_words(wb);
  g.m = q.y;
  g.pos_entry = q.x;
  g.s = res.y;
  g.c1 = res.x + 1u;
  if (g.c1 > n || n > kMaxColumns || g.m > kMaxWords * 32u) return kTbInconsistent;
  if (g.m == 0) return (res.x == 0 && res.y == 0) ? 1u : kTbInconsistent;
  if (g.s > g.m) return kTbInconsistent;  // D[m][j] <= m for every column
  g.off = (int)g.c1 - (int)g.m;
  g.a0 = g.c1 > g.m + g.s ? g.c1 - g.m - g.s : 0u;
  g.start = a.exact ? cd.position : (cd.position & ~7ull);
  if (wl) {
    const uint32_t words = (g.m + 31u) >> 5;
    g.L = (words + wl - 1u) / wl;
    g.tw = g.L * wl;
    g.p = 32u * g.tw - g.m;
    const uint32_t b = tb_band_words(g.s);
    g.B = b < g.tw ? b : g.tw;
  }
  return 0u;
}

// Bytes of a candidate's band store for any words per lane (the cap uses
// the largest possible L*wl, words + 31).
__device__ __forceinline__ unsigned long long tb_slot_bound(const TbGeom& g) {
  const uint32_t words = (g.m + 31u) >> 5, b = tb_band_words(g.s);
  const uint32_t B = b < words + 31u ? b : words + 31u;
  return (unsigned long long)(g.c1 - g.a0 + 1u) * B * 16ull;
}

// Pick the candidates to trace; write the records of the others.
__global__ void k_tb_select(TbArgs a, uint32_t* ids, unsigned long long* offs) {
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t base = blockIdx.x * blockDim.x; base < a.num_cands; base += gridDim.x * blockDim.x) {
    const uint32_t id = base + threadIdx.x;
    bool traced = false;
    uint32_t units = 0;
    TbGeom g;
    if (id < a.num_cands) {
      const uint2 res = a.results[id];
      const uint32_t why = tb_setup(a, id, res, 0u, g);
      uint4 rec = make_uint4(kTbNotTraced, why, res.y, res.x);
      if (why == 1u) rec = make_uint4(res.x + 1u, 0u, res.y, res.x);  // empty query: empty alignment
      if (why == 0u) {
        traced = true;
        rec.y = 0u;
        units = (uint32_t)((tb_slot_bound(g) + (1ull << kTbUnitShift) - 1ull) >> kTbUnitShift);
        atomicMax(&a.st->max_words, (g.m + 31u) >> 5);
        atomicMax(&a.st->max_inv_words, ~((g.m + 31u) >> 5));
        atomicMax(&a.st->max_units, units);
      }
      a.alns[id] = rec;
    }
    // warp-aggregated append: list places and band offsets in one atomic
    const uint32_t mask = __ballot_sync(FULL_MASK, traced);
    unsigned long long incl = units;  // inclusive prefix of the units over the warp
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const unsigned long long v = __shfl_up_sync(FULL_MASK, incl, d);
      if ((int)lane >= d) incl += v;
    }
    const unsigned long long total = __shfl_sync(FULL_MASK, incl, 31);
    unsigned long long old = 0;
    if (lane == 0 && mask)
      old = atomicAdd(&a.st->packed, ((unsigned long long)__popc(mask) << kTbCountShift) + total);
    old = __shfl_sync(FULL_MASK, old, 0);
    if (traced) {
      const uint32_t pos = (uint32_t)(old >> kTbCountShift) + __popc(mask & ((1u << lane) - 1u));
      ids[pos] = id;
      offs[pos] = (old & kTbUnitMask) + incl - units;
    }
  }
}

// One column over a lane's W words with the horizontal delta hin entering
// its bottom row; keeps the unshifted Ph/Mh words (the deltas into this
// column) and returns the delta out of the top row.
template <int W>
__device__ __forceinline__ int tb_column(const uint32_t* __restrict__ eq, uint32_t (&Pv)[W], uint32_t (&Mv)[W],
                                         int hin, uint32_t (&ph)[W], uint32_t (&mh)[W]) {
  uint32_t e[W], t[W], s[W];
#pragma unroll
  for (int k = 0; k < W; k += 4) {
    const uint4 v = *reinterpret_cast<const uint4*>(eq + k);
    e[k] = v.x;
    e[k + 1] = v.y;
    e[k + 2] = v.z;
    e[k + 3] = v.w;
  }
  const uint32_t e0 = e[0] | (hin < 0 ? 1u : 0u);
  t[0] = e0 & Pv[0];
#pragma unroll
  for (int k = 1; k < W; ++k) t[k] = e[k] & Pv[k];
  // multi-word add t + Pv as one carry chain
  asm volatile("add.cc.u32 %0, %1, %2;" : "=r"(s[0]) : "r"(t[0]), "r"(Pv[0]));
#pragma unroll
  for (int k = 1; k < W - 1; ++k) asm volatile("addc.cc.u32 %0, %1, %2;" : "=r"(s[k]) : "r"(t[k]), "r"(Pv[k]));
  asm volatile("addc.u32 %0, %1, %2;" : "=r"(s[W - 1]) : "r"(t[W - 1]), "r"(Pv[W - 1]));
  uint32_t pin = hin > 0 ? 1u : 0u, min_ = hin < 0 ? 1u : 0u;
#pragma unroll
  for (int k = 0; k < W; ++k) {
    const uint32_t ek = k == 0 ? e0 : e[k];
    const uint32_t pv = Pv[k], mv = Mv[k];
    const uint32_t xv = e[k] | mv;
    const uint32_t xh = (s[k] ^ pv) | ek;
    const uint32_t hp = mv | ~(xh | pv);
    const uint32_t hm = pv & xh;
    ph[k] = hp;
    mh[k] = hm;
    const uint32_t phs = (hp << 1) | pin;
    const uint32_t mhs = (hm << 1) | min_;
    pin = hp >> 31;
    min_ = hm >> 31;
    Pv[k] = mhs | ~(xv | phs);
    Mv[k] = phs & xv;
  }
  return (int)pin - (int)min_;
}

// First list place whose band offset is >= v.
__device__ __forceinline__ uint32_t tb_lower(const unsigned long long* __restrict__ offs, uint32_t n,
                                             unsigned long long v) {
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(offs + mid) < v) lo = mid + 1u;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ unsigned char* tb_slot(const TbArgs& a, uint32_t k) {
  return a.scratch + ((__ldg(a.offs + k) - a.unit_lo) << kTbUnitShift);
}

// Shared memory per warp: 32 lanes x 5 bases x W words.
template <int W>
__global__ void __launch_bounds__(128) k_tb_forward(TbArgs a) {
  extern __shared__ __align__(16) uint32_t tb_smem[];
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t S = a.seg, G = 32u / S;
  const uint32_t seg = lane / S, r = lane % S;
  uint32_t* sm = tb_smem + (warp * 32u + lane) * 5u * W;  // this lane's [base][W]
  const uint32_t klo = tb_lower(a.offs, a.count, a.unit_lo), khi = tb_lower(a.offs, a.count, a.unit_hi);
  // Groups of G candidates: with fwd_counter, warps take them from the
  // chunk's counter (queries of mixed lengths: uneven groups); else warp w
  // takes groups w, w + warps, ... (one query length: even groups, and blocks
  // that exit early leave room for the previous chunk's walk).
  const uint32_t nwarps = gridDim.x * 4u;
  uint32_t gi = blockIdx.x * 4u + warp;
  while (true) {
    if (a.fwd_counter) {
      uint32_t v = 0;
      if (lane == 0) v = atomicAdd(&a.next[0], 1u);
      gi = __shfl_sync(FULL_MASK, v, 0);
    }
    const uint32_t base = klo + gi * G;
    if (base >= khi) break;
    if (!a.fwd_counter) gi += nwarps;
    const uint32_t k = base + seg;
    TbGeom g;
    uint32_t id = 0;
    bool have = false;
    if (k < khi) {
      id = a.ids[k];
      have = tb_setup(a, id, a.results[id], W, g) == 0u;
    }
    const bool on = have && r < g.L;
    const uint32_t steps = __reduce_max_sync(FULL_MASK, have ? g.c1 + g.L - 1u : 0u);
    uint4* slot = have ? reinterpret_cast<uint4*>(tb_slot(a, k)) : nullptr;
    if (on) {
      // the lane's W words of the top-aligned query, all five bases
      const int nw = (int)((g.m + 31u) >> 5);
      const int pw = (int)(g.p >> 5), ps = (int)(g.p & 31u);
      for (int c = 0; c < 5; ++c)
#pragma unroll
        for (int kk = 0; kk < W; ++kk) {
          const int x = (int)r * W + kk - pw;
          const uint32_t hi = qword(a.peq, g.pos_entry, nw, c, x);
          const uint32_t lo = qword(a.peq, g.pos_entry, nw, c, x - 1);
          sm[c * W + kk] = ps ? __funnelshift_r(lo, hi, 32 - ps) : hi;
        }
    }
    __syncwarp();
    uint32_t Pv[W], Mv[W], ph[W], mh[W];
#pragma unroll
    for (int kk = 0; kk < W; ++kk) {
      Pv[kk] = FULL_MASK;
      Mv[kk] = 0u;
    }
    int hout = 0;
    uint32_t top = on ? 32u * g.tw : 0u;  // D at the top row, column 0 (last lane of the segment)
    const uint32_t x0 = r * W;            // the lane's first word
    // The lane's text: its columns are consecutive bases from the window
    // start, read one sanitised word at a time (the next word fetched ahead).
    long long widx = on ? (long long)(g.start >> 3) : 0;
    uint32_t nib = on ? (uint32_t)(g.start & 7ull) : 0u;
    uint32_t tw = on ? sanitize_codes(ref_load(a.ref, widx, a.ref_words)) : 0u;
    uint32_t tw_next = on ? ref_load(a.ref, widx + 1, a.ref_words) : 0u;
    for (uint32_t t = 0; t < steps; ++t) {
      int hin = __shfl_up_sync(FULL_MASK, hout, 1, S);
      if (r == 0) hin = 0;
      const int j = (int)t - (int)r;  // 0-based text base of this lane's column
      hout = 0;
      if (on && j >= 0 && (uint32_t)j < g.c1) {
        const uint32_t code = (tw >> (4u * nib)) & 0xFu;
        if (++nib == 8u) {
          nib = 0u;
          ++widx;
          tw = sanitize_codes(tw_next);
          tw_next = ref_load(a.ref, widx + 1, a.ref_words);
        }
        hout = tb_column<W>(sm + code * W, Pv, Mv, hin, ph, mh);
        const uint32_t j1 = (uint32_t)j + 1u;
        if (r == g.L - 1u) top += (uint32_t)hout;
        if (j1 >= g.a0) {
          const uint32_t xlo = tb_xlo(g, j1);
          if (x0 < xlo + g.B && xlo < x0 + W) {  // the lane's words meet the band
            // The entry of the lane's first word, which lies outside the column
            // when that word is outside the band (no such entry is written).
            // One base address with constant offsets per word: the per-word
            // indexing of the column cost 4% of the call (measured).
            const long long e0 = (long long)(j1 - g.a0) * g.B + (long long)x0 - (long long)xlo;
            uint4* base = reinterpret_cast<uint4*>(reinterpret_cast<uintptr_t>(slot) + (uintptr_t)(e0 * 16));
            const uint32_t c = x0 - xlo;
#pragma unroll
            for (int kk = 0; kk < W; ++kk)
              if (c + (uint32_t)kk < g.B) base[kk] = make_uint4(Pv[kk], Mv[kk], ph[kk], mh[kk]);  // wraps above B below the band
          }
        }
      }
    }
    // the recomputed score at the end column must be the result's
    if (on && r == g.L - 1u && top - g.p != g.s) a.alns[id].y = kTbInconsistent;
    __syncwarp();
  }
}

__device__ __forceinline__ int tb_delta(uint32_t p, uint32_t m, uint32_t sh) {
  return (int)((p >> sh) & 1u) - (int)((m >> sh) & 1u);
}

// Word x of column j1's band, tagged with x; a zero word tagged 0xFFFFFFFF
// when the column is not kept (outside [max(1, a0), c1]; a column index that
// wrapped below zero lands above c1) or x lies outside its band.
struct TbCol {
  uint4 v;
  uint32_t x;
};


__device__ __forceinline__ TbCol tb_fetch(const uint4* __restrict__ slot, const TbGeom& g, uint32_t j1, uint32_t x) {
  TbCol c;
  c.v = make_uint4(0u, 0u, 0u, 0u);
  c.x = 0xFFFFFFFFu;
  if (j1 >= 1u && j1 >= g.a0 && j1 <= g.c1) {
    const uint32_t xa = tb_xlo(g, j1);
    if (x >= xa && x < xa + g.B) {
      const uint4* e = slot + (size_t)(j1 - g.a0) * g.B + (x - xa);
#if MYERS_TB_LDG
      c.v = __ldg(e);
#else
      c.v = __ldcg(e);
#endif
      c.x = x;
    }
  }
  return c;
}

// The walk of list place k (a traced candidate of this chunk).
__device__ void tb_walk_one(const TbArgs& a, uint32_t k) {
  const uint32_t id = a.ids[k];
  TbGeom g;
  if (tb_setup(a, id, a.results[id], a.wl, g) != 0u) return;
  if (a.alns[id].y == kTbInconsistent) return;
  const uint4* slot = reinterpret_cast<const uint4*>(tb_slot(a, k));
  uint32_t* out = a.ops + (size_t)id * a.max_ops;
  const int nw = (int)((g.m + 31u) >> 5);
  uint32_t i = g.m, j1 = g.c1;
  uint32_t nruns = 0, cur = 0, len = 0;
  bool bad = false;
  // cw[0]: column j1; cw[d]: column j1-d (fetched ahead); all at word xw
  constexpr int D = MYERS_TB_AHEAD;
  uint32_t xw = 0xFFFFFFFFu;
  TbCol cw[D + 1];
  // PEQ words of query word qw (five bases); text word twi
  uint32_t qw = 0xFFFFFFFFu, q0 = 0, q1 = 0, q2 = 0, q3 = 0, q4 = 0;
  unsigned long long twi = ~0ull;
  uint32_t twv = 0;
  // every step lowers i or j1: at most m + c1 steps
  while (i > 0u) {
    uint32_t op;
    if (j1 <= g.a0) {
      op = kOpI;  // only the query base alone is left (column 0, or the first kept column)
      --i;
    } else {
      const uint32_t bit = g.p + i - 1u, x = bit >> 5, sh = bit & 31u;
      if (x != xw) {
        xw = x;
#pragma unroll
        for (int d = 0; d <= D; ++d) cw[d] = tb_fetch(slot, g, j1 - (uint32_t)d, x);
      }
      if (cw[0].x != x) cw[0] = tb_fetch(slot, g, j1, x);
      if (cw[0].x != x) {  // the path left the stored band: the data is inconsistent
        bad = true;
        break;
      }
      const uint32_t q = i - 1u;
      if ((q >> 5) != qw) {
        qw = q >> 5;
        q0 = qword(a.peq, g.pos_entry, nw, 0, (int)qw);
        q1 = qword(a.peq, g.pos_entry, nw, 1, (int)qw);
        q2 = qword(a.peq, g.pos_entry, nw, 2, (int)qw);
        q3 = qword(a.peq, g.pos_entry, nw, 3, (int)qw);
        q4 = qword(a.peq, g.pos_entry, nw, 4, (int)qw);
      }
      const unsigned long long b = g.start + j1 - 1u;
      if ((b >> 3) != twi) {
        twi = b >> 3;
        twv = sanitize_codes(ref_load(a.ref, (long long)twi, a.ref_words));
      }
      const uint32_t code = (twv >> (4u * (uint32_t)(b & 7u))) & 0xFu;
      const uint32_t pq = code == 0 ? q0 : code == 1 ? q1 : code == 2 ? q2 : code == 3 ? q3 : q4;
      const uint32_t match = (pq >> (q & 31u)) & 1u;
      const int h = tb_delta(cw[0].v.z, cw[0].v.w, sh), v = tb_delta(cw[0].v.x, cw[0].v.y, sh);
      int vl = 1;  // column 0: D[i][0] = i
      if (j1 - 1u > 0u) {
        if (cw[1].x != x) cw[1] = tb_fetch(slot, g, j1 - 1u, x);
        if (cw[1].x != x) {
          bad = true;
          break;
        }
        vl = tb_delta(cw[1].v.x, cw[1].v.y, sh);
      }
      if (h + vl == (int)(1u - match)) {
        op = match ? kOpEq : kOpX;
        --i;
        --j1;
      } else if (v == 1) {
        op = kOpI;
        --i;
      } else {
        op = kOpD;
        --j1;
      }
      if (op != kOpI) {  // one column to the left: shift the window, fetch one more
#pragma unroll
        for (int d = 0; d < D; ++d) cw[d] = cw[d + 1];
        cw[D] = tb_fetch(slot, g, j1 >= (uint32_t)D ? j1 - (uint32_t)D : 0u, xw);
      }
    }
    if (len && op == cur) {
      ++len;
    } else {
      if (len) {
        if (nruns < a.max_ops) out[a.max_ops - 1u - nruns] = (len << 4) | cur;
        ++nruns;
      }
      cur = op;
      len = 1;
    }
  }
  if (bad) {
    a.alns[id].y = kTbInconsistent;
    return;
  }
  if (len) {
    if (nruns < a.max_ops) out[a.max_ops - 1u - nruns] = (len << 4) | cur;
    ++nruns;
  }
  // runs were written last first at the end of the region: move them to the front
  if (nruns <= a.max_ops) {
    const uint32_t src = a.max_ops - nruns;
    for (uint32_t r = 0; r < nruns; ++r) out[r] = out[src + r];
  }
  a.alns[id] = make_uint4(j1, nruns, g.s, g.c1 - 1u);
}

__global__ void __launch_bounds__(128) k_tb_walk(TbArgs a) {
  const uint32_t klo = tb_lower(a.offs, a.count, a.unit_lo), khi = tb_lower(a.offs, a.count, a.unit_hi);
  const uint32_t lane = threadIdx.x & 31u;
  while (true) {
    // warps take 32 candidates at a time from the chunk's counter
    uint32_t w0 = 0;
    if (lane == 0) w0 = atomicAdd(&a.next[1], 32u);
    const uint32_t base = klo + __shfl_sync(FULL_MASK, w0, 0);
    if (base >= khi) break;
    if (base + lane < khi) tb_walk_one(a, base + lane);
    __syncwarp();
  }
}

}  // namespace myers

using namespace myers;

struct myersTraceback {
  int device;
  int num_sms;
  uint64_t capacity;
  uint64_t scratch_bytes;
  unsigned char* d_scratch;
  uint32_t* d_ids;
  unsigned long long* d_offs;
  TbState* d_state;
  TbState* h_state;
  cudaStream_t walk_stream;
  cudaEvent_t fwd_done[2], walk_done[2];
  uint32_t last_count;
  uint32_t last_chunks;
};

static void tb_release(myersTraceback_t* t) {
  cudaFree(t->d_scratch);
  cudaFree(t->d_ids);
  cudaFree(t->d_offs);
  cudaFree(t->d_state);
  cudaFreeHost(t->h_state);
  for (int h = 0; h < 2; ++h) {
    if (t->fwd_done[h]) cudaEventDestroy(t->fwd_done[h]);
    if (t->walk_done[h]) cudaEventDestroy(t->walk_done[h]);
  }
  if (t->walk_stream) cudaStreamDestroy(t->walk_stream);
  delete t;
}

extern "C" int myersTracebackCreate(myersTraceback_t** tb, uint64_t maxCandidates, uint64_t scratchBytes) {
  if (tb == nullptr || maxCandidates == 0 || maxCandidates >= (1ull << (64 - kTbCountShift)) ||
      scratchBytes < (1u << 20))
    return MYERS_E_INVALID_ARGUMENT;
  *tb = nullptr;
  myersTraceback_t* t = new myersTraceback_t();
  memset(t, 0, sizeof(*t));
  cudaError_t e = cudaGetDevice(&t->device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&t->num_sms, cudaDevAttrMultiProcessorCount, t->device);
  t->capacity = maxCandidates;
  t->scratch_bytes = scratchBytes & ~511ull;
  if (e == cudaSuccess) e = cudaMalloc((void**)&t->d_scratch, t->scratch_bytes);
  if (e == cudaSuccess) e = cudaMalloc((void**)&t->d_ids, maxCandidates * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc((void**)&t->d_offs, maxCandidates * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc((void**)&t->d_state, sizeof(TbState));
  if (e == cudaSuccess) e = cudaHostAlloc((void**)&t->h_state, sizeof(TbState), cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&t->walk_stream, cudaStreamNonBlocking);
  for (int h = 0; h < 2 && e == cudaSuccess; ++h) {
    e = cudaEventCreateWithFlags(&t->fwd_done[h], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t->walk_done[h], cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    tb_release(t);
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? MYERS_E_INSUFFICIENT_MEM_GPU : cuda_fail(e, "myersTracebackCreate");
  }
  *tb = t;
  return MYERS_SUCCESS;
}

extern "C" int myersTracebackDestroy(myersTraceback_t* tb) {
  if (tb == nullptr) return MYERS_E_INVALID_ARGUMENT;
  cudaSetDevice(tb->device);
  cudaDeviceSynchronize();
  tb_release(tb);
  return MYERS_SUCCESS;
}

extern "C" uint32_t myersTracebackLastCount(const myersTraceback_t* tb) { return tb ? tb->last_count : 0u; }
extern "C" uint32_t myersTracebackLastChunks(const myersTraceback_t* tb) { return tb ? tb->last_chunks : 0u; }

template <int W>
static cudaError_t launch_tb_forward(const TbArgs& a, uint32_t cnt, int num_sms, cudaStream_t s) {
  // cnt: an upper estimate of the chunk's candidates (the kernel finds its range)
  const size_t smem = 4u * 32u * 5u * W * sizeof(uint32_t);
  if (smem > 48u * 1024u) {  // per function and device; cheap to repeat
    cudaError_t e = cudaFuncSetAttribute(k_tb_forward<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  const uint32_t per_block = 4u * (32u / a.seg);
  uint32_t blocks = (cnt + per_block - 1u) / per_block;
  const uint32_t cap = (uint32_t)num_sms * 16u;
  if (blocks > cap) blocks = cap;
  k_tb_forward<W><<<blocks, 128, smem, s>>>(a);
  return cudaGetLastError();
}

extern "C" int myersTraceback(myersTraceback_t* tb, const myersReference_t* ref, const qryEntry_t* d_peq,
                              uint32_t numPEQEntries, const qryInfo_t* d_qinfo, uint32_t numQueries,
                              const candInfo_t* d_cands, const resEntry_t* d_results, uint32_t numCandidates,
                              float distance, int windowMode, uint32_t maxScore, uint32_t* d_ops,
                              uint32_t maxOpsPerCandidate, myersAlignment_t* d_alignments, void* stream) {
  if (tb == nullptr || ref == nullptr || !(distance >= 0.0f) || !std::isfinite(distance) ||
      (windowMode != MYERS_WINDOW_ALIGNED && windowMode != MYERS_WINDOW_EXACT) || maxOpsPerCandidate == 0)
    return MYERS_E_INVALID_ARGUMENT;
  tb->last_count = 0;
  tb->last_chunks = 0;
  if (numCandidates == 0) return MYERS_SUCCESS;
  if (d_peq == nullptr || d_qinfo == nullptr || d_cands == nullptr || d_results == nullptr || d_ops == nullptr ||
      d_alignments == nullptr)
    return MYERS_E_INVALID_ARGUMENT;
  if (numCandidates > tb->capacity) return MYERS_E_CAPACITY;
  if (ref->device != tb->device) return MYERS_E_INVALID_ARGUMENT;
  NvtxRange range("myers: traceback (select, count, passes)");
  cudaError_t e = cudaSetDevice(tb->device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  cudaStream_t s = (cudaStream_t)stream;
  TbArgs a;
  memset(&a, 0, sizeof(a));
  a.peq = reinterpret_cast<const uint32_t*>(d_peq);
  a.qinfo = reinterpret_cast<const uint2*>(d_qinfo);
  a.cands = reinterpret_cast<const Cand*>(d_cands);
  a.results = reinterpret_cast<const uint2*>(d_results);
  a.ref = ref->d_words;
  a.ref_size = ref->size;
  a.ref_words = ref->words + kRefPadWords;
  a.num_cands = numCandidates;
  a.num_queries = numQueries;
  a.num_entries = numPEQEntries;
  a.distance = distance;
  a.exact = windowMode == MYERS_WINDOW_EXACT;
  a.max_score = maxScore;
  a.ops = d_ops;
  a.max_ops = maxOpsPerCandidate;
  a.alns = reinterpret_cast<uint4*>(d_alignments);
  a.st = tb->d_state;
  if ((e = cudaMemsetAsync(tb->d_state, 0, sizeof(TbState), s)) != cudaSuccess) return cuda_fail(e, "memset");
  uint32_t blocks = (numCandidates + 255u) / 256u;
  if (blocks > (uint32_t)tb->num_sms * 8u) blocks = (uint32_t)tb->num_sms * 8u;
  k_tb_select<<<blocks, 256, 0, s>>>(a, tb->d_ids, tb->d_offs);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "k_tb_select");
  // the pass count depends on how many candidates are traced and their band sizes
  if ((e = cudaMemcpyAsync(tb->h_state, tb->d_state, sizeof(TbState), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return cuda_fail(e, "traceback count");
  const TbState st = *tb->h_state;
  const uint32_t count = (uint32_t)(st.packed >> kTbCountShift);
  const unsigned long long total = st.packed & kTbUnitMask;
  tb->last_count = count;
  if (count == 0) return MYERS_SUCCESS;
  a.wl = tb_words_per_lane(st.max_words);
  a.fwd_counter = (~st.max_inv_words) != st.max_words;  // more than one query length
  const uint32_t lanes = (st.max_words + a.wl - 1u) / a.wl;
  a.seg = 1;
  while (a.seg < lanes) a.seg <<= 1;
  a.ids = tb->d_ids;
  a.offs = tb->d_offs;
  a.count = count;
  // a chunk holds the candidates whose offsets start in a window of H units;
  // the last of them ends within H + max_units <= half the scratch
  const unsigned long long half_units = (tb->scratch_bytes / 2) >> kTbUnitShift;
  if (half_units <= st.max_units) return MYERS_E_CAPACITY;  // one band does not fit half the scratch
  const unsigned long long H = half_units - st.max_units;
  const unsigned long long chunks = (total + H - 1ull) / H;
  const uint32_t est = (uint32_t)((unsigned long long)count * (H < total ? H : total) / total) + 1u;
  for (uint32_t c = 0; c < chunks; ++c) {
    const int h = (int)(c & 1u);
    TbArgs ca = a;
    ca.unit_lo = c * H;
    ca.unit_hi = ca.unit_lo + H;
    ca.scratch = tb->d_scratch + (size_t)h * (half_units << kTbUnitShift);
    ca.next = tb->d_state->next[h];
    if (c >= 2 && (e = cudaStreamWaitEvent(s, tb->walk_done[h], 0)) != cudaSuccess) return cuda_fail(e, "wait");
    // the half's walk of two chunks ago has finished: its counters may start again
    if ((e = cudaMemsetAsync(ca.next, 0, 2 * sizeof(unsigned int), s)) != cudaSuccess) return cuda_fail(e, "memset");
    switch (a.wl) {
      case 8: e = launch_tb_forward<8>(ca, est, tb->num_sms, s); break;
      case 16: e = launch_tb_forward<16>(ca, est, tb->num_sms, s); break;
      default: e = launch_tb_forward<32>(ca, est, tb->num_sms, s); break;
    }
    if (e != cudaSuccess) return cuda_fail(e, "k_tb_forward");
    if ((e = cudaEventRecord(tb->fwd_done[h], s)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(tb->walk_stream, tb->fwd_done[h], 0)) != cudaSuccess)
      return cuda_fail(e, "event");
    uint32_t wb = (est + 127u) / 128u;
    if (wb > (uint32_t)tb->num_sms * 16u) wb = (uint32_t)tb->num_sms * 16u;
    k_tb_walk<<<wb, 128, 0, tb->walk_stream>>>(ca);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "k_tb_walk");
    if ((e = cudaEventRecord(tb->walk_done[h], tb->walk_stream)) != cudaSuccess) return cuda_fail(e, "event");
  }
  const uint32_t c = (uint32_t)chunks;
  tb->last_chunks = c;
  // the caller's stream resumes after the last walk
  if ((e = cudaStreamWaitEvent(s, tb->walk_done[(c - 1u) & 1u], 0)) != cudaSuccess) return cuda_fail(e, "wait");
  return MYERS_SUCCESS;
}
