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
//  * k_tb_forward: one candidate per warp, its rows spread over L lanes of W
//    words (the systolic layout of the multi-lane verification shapes: lane
//    l processes column t - l at step t, taking the horizontal delta of its
//    bottom row from lane l-1 through a shuffle). It recomputes the window's
//    columns 1..c+1 and stores, for each column, the words of the diagonal
//    band the path can use: Pv/Mv (vertical deltas) and Ph/Mh (horizontal
//    deltas into the column). A path of cost s from (0, a) to (m, c+1) has
//    j - i within s of (c+1) - m at every cell, and consumes at most m + s
//    text bases, so columns before c+1-m-s and rows outside that band are
//    never read back.
//  * k_tb_walk: one thread per candidate walks back with three bit lookups
//    per step: the diagonal is consistent iff h(i,j) + v(i,j-1) equals the
//    mismatch cost, the query base alone iff v(i,j) = +1.
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

struct TbState {
  unsigned int count;               // candidates to trace
  unsigned int max_wl;              // widest words-per-lane among them
  unsigned long long max_slot;      // largest band store (bytes)
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
  uint32_t* ids;
  TbState* st;
  unsigned char* scratch;
  unsigned long long slot_bytes;
};

// Geometry of one traced candidate (identical in all three kernels).
struct TbGeom {
  uint32_t m, pos_entry, s, c1;  // c1 = end column + 1 (1-based)
  uint32_t wl, L, tw, p;         // words per lane, lanes, L*wl, padding rows
  uint32_t a0, B;                // first kept column, band words per column
  int off;                       // c1 - m: the path's final diagonal
  unsigned long long start;      // window start (bases)
};

__host__ __device__ __forceinline__ uint32_t tb_words_per_lane(uint32_t words) {
  uint32_t wl = 1;
  while (32u * wl < words) wl <<= 1;
  return wl;
}

// Band: the first stored word of column j1 (1-based).
__device__ __forceinline__ uint32_t tb_xlo(const TbGeom& g, uint32_t j1) {
  const int row_lo = (int)j1 - g.off - (int)g.s - 1;  // lowest query row the path can use, minus one
  const int bit = (int)g.p + (row_lo < 1 ? 1 : row_lo) - 1;
  const uint32_t x = (uint32_t)bit >> 5;
  return x + g.B > g.tw ? g.tw - g.B : x;
}

// Returns 0 and fills g when the candidate is traced; else the numOps code
// of its record (not traced / inconsistent), or 1 for an empty query.
__device__ __forceinline__ uint32_t tb_setup(const TbArgs& a, uint32_t id, uint2 res, TbGeom& g) {
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
  const uint32_t words = (g.m + 31u) >> 5;
  g.wl = tb_words_per_lane(words);
  g.L = (words + g.wl - 1u) / g.wl;
  g.tw = g.L * g.wl;
  g.p = 32u * g.tw - g.m;
  g.off = (int)g.c1 - (int)g.m;
  g.a0 = g.c1 > g.m + g.s ? g.c1 - g.m - g.s : 0u;
  const uint32_t b = (2u * g.s + 3u + 31u) / 32u + 1u;
  g.B = b < g.tw ? b : g.tw;
  g.start = a.exact ? cd.position : (cd.position & ~7ull);
  return 0u;
}

__device__ __forceinline__ unsigned long long tb_slot_bytes(const TbGeom& g) {
  return (unsigned long long)(g.c1 - g.a0 + 1u) * g.B * 16ull;
}

// Pick the candidates to trace; write the records of the others.
__global__ void k_tb_select(TbArgs a) {
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t base = blockIdx.x * blockDim.x; base < a.num_cands; base += gridDim.x * blockDim.x) {
    const uint32_t id = base + threadIdx.x;
    bool traced = false;
    TbGeom g;
    if (id < a.num_cands) {
      const uint2 res = a.results[id];
      const uint32_t why = tb_setup(a, id, res, g);
      uint4 rec = make_uint4(kTbNotTraced, why, res.y, res.x);
      if (why == 1u) rec = make_uint4(res.x + 1u, 0u, res.y, res.x);  // empty query: empty alignment
      if (why == 0u) {
        traced = true;
        rec.y = 0u;
        atomicMax(&a.st->max_wl, g.wl);
        atomicMax(&a.st->max_slot, tb_slot_bytes(g));
      }
      a.alns[id] = rec;
    }
    // warp-aggregated append of the traced ids
    const uint32_t mask = __ballot_sync(FULL_MASK, traced);
    uint32_t first = 0;
    if (lane == 0 && mask) first = atomicAdd(&a.st->count, (unsigned)__popc(mask));
    first = __shfl_sync(FULL_MASK, first, 0);
    if (traced) a.ids[first + __popc(mask & ((1u << lane) - 1u))] = id;
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
  for (int k = 0; k < W; ++k) e[k] = eq[k];
  const uint32_t e0 = e[0] | (hin < 0 ? 1u : 0u);
  t[0] = e0 & Pv[0];
#pragma unroll
  for (int k = 1; k < W; ++k) t[k] = e[k] & Pv[k];
  // multi-word add t + Pv
  uint32_t carry = 0;
#pragma unroll
  for (int k = 0; k < W; ++k) {
    const uint32_t x = t[k] + Pv[k];
    const uint32_t y = x + carry;
    carry = (x < t[k]) | (y < x);
    s[k] = y;
  }
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

template <int W>
__device__ void tb_forward_one(const TbArgs& a, const TbGeom& g, uint32_t id, uint32_t* __restrict__ sm,
                               uint4* __restrict__ slot) {
  const int l = (int)(threadIdx.x & 31u);
  const bool on = (uint32_t)l < g.L;
  // the lane's W words of the top-aligned query, all five bases: sm[(l*5 + c)*W + k]
  if (on) {
    const int nw = (int)((g.m + 31u) >> 5);
    const int pw = (int)(g.p >> 5), ps = (int)(g.p & 31u);
    for (int c = 0; c < 5; ++c)
#pragma unroll
      for (int k = 0; k < W; ++k) {
        const int x = l * W + k - pw;
        const uint32_t hi = qword(a.peq, g.pos_entry, nw, c, x);
        const uint32_t lo = qword(a.peq, g.pos_entry, nw, c, x - 1);
        sm[(l * 5 + c) * W + k] = ps ? __funnelshift_r(lo, hi, 32 - ps) : hi;
      }
  }
  __syncwarp();
  uint32_t Pv[W], Mv[W], ph[W], mh[W];
#pragma unroll
  for (int k = 0; k < W; ++k) {
    Pv[k] = FULL_MASK;
    Mv[k] = 0u;
  }
  int hout = 0;
  uint32_t top = 32u * g.tw;  // D at the top row, column 0 (lane L-1)
  const uint32_t steps = g.c1 + g.L - 1u;
  for (uint32_t t = 0; t < steps; ++t) {
    int hin = __shfl_up_sync(FULL_MASK, hout, 1);
    if (l == 0) hin = 0;
    const int j = (int)t - l;  // 0-based text base of this lane's column
    hout = 0;
    if (on && j >= 0 && (uint32_t)j < g.c1) {
      const uint32_t code = ref_code(a.ref, g.start + (unsigned long long)j, a.ref_words);
      hout = tb_column<W>(sm + (l * 5 + (int)code) * W, Pv, Mv, hin, ph, mh);
      const uint32_t j1 = (uint32_t)j + 1u;
      if (l == (int)g.L - 1) top += (uint32_t)hout;
      if (j1 >= g.a0) {
        const uint32_t xlo = tb_xlo(g, j1);
        uint4* col = slot + (size_t)(j1 - g.a0) * g.B;
#pragma unroll
        for (int k = 0; k < W; ++k) {
          const uint32_t x = (uint32_t)(l * W + k);
          if (x >= xlo && x < xlo + g.B) col[x - xlo] = make_uint4(Pv[k], Mv[k], ph[k], mh[k]);
        }
      }
    }
  }
  // the recomputed score at the end column must be the result's
  if (l == (int)g.L - 1 && top - g.p != g.s) a.alns[id].y = kTbInconsistent;
}

template <int WMAX>
__global__ void __launch_bounds__(128) k_tb_forward(TbArgs a, uint32_t first, uint32_t cnt) {
  extern __shared__ uint32_t tb_smem[];
  const uint32_t warp = threadIdx.x >> 5;
  uint32_t* sm = tb_smem + warp * (32u * 5u * WMAX);
  for (uint32_t k = blockIdx.x * 4u + warp; k < cnt; k += gridDim.x * 4u) {
    const uint32_t id = a.ids[first + k];
    TbGeom g;
    if (tb_setup(a, id, a.results[id], g) != 0u) continue;  // warp-uniform
    uint4* slot = reinterpret_cast<uint4*>(a.scratch + (size_t)k * a.slot_bytes);
    switch (g.wl) {
      case 1: tb_forward_one<1>(a, g, id, sm, slot); break;
      case 2: if (WMAX >= 2) tb_forward_one<(WMAX >= 2 ? 2 : 1)>(a, g, id, sm, slot); break;
      case 4: if (WMAX >= 4) tb_forward_one<(WMAX >= 4 ? 4 : 1)>(a, g, id, sm, slot); break;
      case 8: if (WMAX >= 8) tb_forward_one<(WMAX >= 8 ? 8 : 1)>(a, g, id, sm, slot); break;
      case 16: if (WMAX >= 16) tb_forward_one<(WMAX >= 16 ? 16 : 1)>(a, g, id, sm, slot); break;
      case 32: if (WMAX >= 32) tb_forward_one<(WMAX >= 32 ? 32 : 1)>(a, g, id, sm, slot); break;
      default: break;
    }
    __syncwarp();
  }
}

__device__ __forceinline__ int tb_delta(uint32_t p, uint32_t m, uint32_t sh) {
  return (int)((p >> sh) & 1u) - (int)((m >> sh) & 1u);
}

__global__ void __launch_bounds__(128) k_tb_walk(TbArgs a, uint32_t first, uint32_t cnt) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
    const uint32_t id = a.ids[first + k];
    TbGeom g;
    if (tb_setup(a, id, a.results[id], g) != 0u) continue;
    if (a.alns[id].y == kTbInconsistent) continue;
    const uint4* slot = reinterpret_cast<const uint4*>(a.scratch + (size_t)k * a.slot_bytes);
    uint32_t* out = a.ops + (size_t)id * a.max_ops;
    const int nw = (int)((g.m + 31u) >> 5);
    uint32_t i = g.m, j1 = g.c1;
    uint32_t nruns = 0, cur = 0, len = 0;
    bool bad = false;
    // every step lowers i or j1: at most m + c1 steps
    while (i > 0u) {
      uint32_t op;
      if (j1 <= g.a0) {
        op = kOpI;  // only the query base alone is left (column 0, or the first kept column)
        --i;
      } else {
        const uint32_t bit = g.p + i - 1u, x = bit >> 5, sh = bit & 31u;
        const uint32_t xa = tb_xlo(g, j1);
        if (x < xa || x >= xa + g.B) { bad = true; break; }
        const uint4 c = slot[(size_t)(j1 - g.a0) * g.B + (x - xa)];
        const int h = tb_delta(c.z, c.w, sh), v = tb_delta(c.x, c.y, sh);
        int vl = 1;  // column 0: D[i][0] = i
        if (j1 - 1u > 0u) {
          const uint32_t xb = tb_xlo(g, j1 - 1u);
          if (x < xb || x >= xb + g.B) { bad = true; break; }
          const uint4 cl = slot[(size_t)(j1 - 1u - g.a0) * g.B + (x - xb)];
          vl = tb_delta(cl.x, cl.y, sh);
        }
        const uint32_t code = ref_code(a.ref, g.start + j1 - 1u, a.ref_words);
        const uint32_t q = i - 1u;
        const uint32_t match = (qword(a.peq, g.pos_entry, nw, (int)code, (int)(q >> 5)) >> (q & 31u)) & 1u;
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
      continue;
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
  TbState* d_state;
  TbState* h_state;
  uint32_t last_count;
  uint32_t last_chunks;
};

extern "C" int myersTracebackCreate(myersTraceback_t** tb, uint64_t maxCandidates, uint64_t scratchBytes) {
  if (tb == nullptr || maxCandidates == 0 || maxCandidates > 0xFFFFFFFFull || scratchBytes < (1u << 20))
    return MYERS_E_INVALID_ARGUMENT;
  *tb = nullptr;
  myersTraceback_t* t = new myersTraceback_t();
  memset(t, 0, sizeof(*t));
  cudaError_t e = cudaGetDevice(&t->device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&t->num_sms, cudaDevAttrMultiProcessorCount, t->device);
  t->capacity = maxCandidates;
  t->scratch_bytes = scratchBytes;
  if (e == cudaSuccess) e = cudaMalloc((void**)&t->d_scratch, scratchBytes);
  if (e == cudaSuccess) e = cudaMalloc((void**)&t->d_ids, maxCandidates * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc((void**)&t->d_state, sizeof(TbState));
  if (e == cudaSuccess) e = cudaHostAlloc((void**)&t->h_state, sizeof(TbState), cudaHostAllocDefault);
  if (e != cudaSuccess) {
    cudaFree(t->d_scratch);
    cudaFree(t->d_ids);
    cudaFree(t->d_state);
    delete t;
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
  cudaFree(tb->d_scratch);
  cudaFree(tb->d_ids);
  cudaFree(tb->d_state);
  cudaFreeHost(tb->h_state);
  delete tb;
  return MYERS_SUCCESS;
}

extern "C" uint32_t myersTracebackLastCount(const myersTraceback_t* tb) { return tb ? tb->last_count : 0u; }
extern "C" uint32_t myersTracebackLastChunks(const myersTraceback_t* tb) { return tb ? tb->last_chunks : 0u; }

template <int WMAX>
static cudaError_t launch_tb_forward(const TbArgs& a, uint32_t first, uint32_t cnt, int num_sms, cudaStream_t s) {
  const size_t smem = 4u * 32u * 5u * WMAX * sizeof(uint32_t);
  if (smem > 48u * 1024u) {  // per function and device; cheap to repeat
    cudaError_t e = cudaFuncSetAttribute(k_tb_forward<WMAX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  uint32_t blocks = (cnt + 3u) / 4u;
  const uint32_t cap = (uint32_t)num_sms * 16u;
  if (blocks > cap) blocks = cap;
  k_tb_forward<WMAX><<<blocks, 128, smem, s>>>(a, first, cnt);
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
  if (numCandidates == 0) {
    tb->last_count = 0;
    tb->last_chunks = 0;
    return MYERS_SUCCESS;
  }
  if (d_peq == nullptr || d_qinfo == nullptr || d_cands == nullptr || d_results == nullptr || d_ops == nullptr ||
      d_alignments == nullptr)
    return MYERS_E_INVALID_ARGUMENT;
  if (numCandidates > tb->capacity) return MYERS_E_CAPACITY;
  if (ref->device != tb->device) return MYERS_E_INVALID_ARGUMENT;
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
  a.ids = tb->d_ids;
  a.st = tb->d_state;
  a.scratch = tb->d_scratch;
  if ((e = cudaMemsetAsync(tb->d_state, 0, sizeof(TbState), s)) != cudaSuccess) return cuda_fail(e, "memset");
  uint32_t blocks = (numCandidates + 255u) / 256u;
  if (blocks > (uint32_t)tb->num_sms * 8u) blocks = (uint32_t)tb->num_sms * 8u;
  k_tb_select<<<blocks, 256, 0, s>>>(a);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "k_tb_select");
  // the pass count depends on how many candidates are traced and their band sizes
  if ((e = cudaMemcpyAsync(tb->h_state, tb->d_state, sizeof(TbState), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return cuda_fail(e, "traceback count");
  const TbState st = *tb->h_state;
  tb->last_count = st.count;
  tb->last_chunks = 0;
  if (st.count == 0) return MYERS_SUCCESS;
  const unsigned long long slot = (st.max_slot + 255ull) & ~255ull;
  const unsigned long long per = tb->scratch_bytes / slot;
  if (per == 0) return MYERS_E_CAPACITY;  // one candidate's band does not fit the scratch
  a.slot_bytes = slot;
  for (uint32_t first = 0; first < st.count; first += (uint32_t)per) {
    const uint32_t cnt = (uint32_t)(st.count - first < per ? st.count - first : per);
    switch (st.max_wl) {
      case 1: e = launch_tb_forward<1>(a, first, cnt, tb->num_sms, s); break;
      case 2: e = launch_tb_forward<2>(a, first, cnt, tb->num_sms, s); break;
      case 4: e = launch_tb_forward<4>(a, first, cnt, tb->num_sms, s); break;
      case 8: e = launch_tb_forward<8>(a, first, cnt, tb->num_sms, s); break;
      case 16: e = launch_tb_forward<16>(a, first, cnt, tb->num_sms, s); break;
      default: e = launch_tb_forward<32>(a, first, cnt, tb->num_sms, s); break;
    }
    if (e != cudaSuccess) return cuda_fail(e, "k_tb_forward");
    uint32_t wb = (cnt + 127u) / 128u;
    if (wb > (uint32_t)tb->num_sms * 16u) wb = (uint32_t)tb->num_sms * 16u;
    k_tb_walk<<<wb, 128, 0, s>>>(a, first, cnt);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "k_tb_walk");
    ++tb->last_chunks;
  }
  return MYERS_SUCCESS;
}
