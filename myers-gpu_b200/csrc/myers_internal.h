// Internal types shared by the kernels (myers_kernels.cu) and the host
// runtime (myers_api.cu). Not part of the public ABI.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

namespace myers {

// An NVTX range over a scope: host stages show up by name on a profiler's
// timeline (nsys, ncu's NVTX filters); without a tool attached a push/pop is
// a check of a null callback.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Eight N codes: what the kernels read past the end of the packed reference.
constexpr uint32_t kPadWord = 0x44444444u;
// Words of N padding appended to the device copy of the reference, so the
// window reads past the last packed word stay inside the allocation.
constexpr uint64_t kRefPadWords = 64;
constexpr uint32_t kNoResult = 0xFFFFFFFFu;
// Column and score of a candidate whose minimum exceeds the cut-off bound.
constexpr uint32_t kNoMatch = 0xFFFFFFFFu;
constexpr uint32_t kMaxWords = 1024;          // 32768 bases
constexpr uint32_t kMaxColumns = 65535;       // the result key keeps 16 column bits

// Device error flags (BucketState::flags / DevInputs::flags).
constexpr uint32_t kFlagUnsupported = 1u;     // query too long or window too wide
constexpr uint32_t kFlagBadQuery = 2u;        // candidate query index >= numQueries
constexpr uint32_t kFlagBadEntry = 4u;        // query PEQ entries beyond numPEQEntries

// Candidate as laid out by the API (candInfo_t with its 4 padding bytes).
struct Cand {
  uint32_t query;
  uint32_t pad;
  unsigned long long position;
};

// Kernel variants. Single-lane variants (one candidate per lane, W words of
// 32 query rows each) cover W = 1..32; multi-lane variants spread one
// candidate over L lanes of W words and hand the horizontal delta from lane
// to lane once per column.
constexpr int kNumSingle = 32;
// Every width from 4 to 16 lets a long query's lanes fill the warp: with
// widths 4, 5, 6, 7, 8, 10, 12, 16 alone, lanes left idle where L does not
// divide 32 and padding rows capped long reads at about 0.89 of ALU time in
// the persistent kernel (0.94 with every width; measured +5%).
constexpr int kMultiW[] = {4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 32};
constexpr int kNumMulti = sizeof(kMultiW) / sizeof(kMultiW[0]);
constexpr int kNumVariants = kNumSingle + kNumMulti;
// The persistent kernel carries every single-lane shape and multi-lane
// shapes up to 16 words per lane.
constexpr int kBatchedMaxMultiW = 16;

// A length bucket's launch shape: variant (kernel template), lanes per
// candidate L and words per lane W. Buckets are indexed by the number of
// 32-bit query words, ceil(m/32).
struct Shape {
  uint8_t variant;  // 0..31 single W=variant+1; 32.. multi kMultiW[variant-32]
  uint8_t L;
  uint8_t W;
  uint8_t pad;
};

constexpr int kMaxCfg = 128;            // distinct shapes in one plan
// Batches of at least this many candidates take the batched path's shapes for
// large batches (every lane width; the autotuner cache's "batched_large").
constexpr uint64_t kLargeBatchCandidates = 150000;
// Batches below this many candidates take latency shapes on the batched path
// for reads of up to 1,024 bases: lanes of at most kSmallBatchLaneWords words.
constexpr uint64_t kSmallBatchCandidates = 280000;
constexpr uint32_t kSmallBatchLaneWords = 12;
// With fewer than two candidates per read, reads of 513..1,024 bases take
// lanes of at most this many words.
constexpr uint32_t kDistinctLaneWords = 16;
// Streams a context's plain launches of different shapes run on at once.
constexpr int kPlainStreams = 4;
constexpr uint8_t kNoCfg = 0xFF;

// Per-send plan, passed by value as a __grid_constant__ kernel parameter:
// word count -> shape index, and the shapes in launch order. The first
// num_batched shapes (most expensive first) go to the persistent kernel on
// the batched path; the rest always get plain launches.
struct PlanTable {
  uint8_t cfg_of_words[kMaxWords + 1];
  uint8_t pad[3];
  uint32_t num_cfg;
  uint32_t num_batched;
  Shape shape[kMaxCfg];
};

// Device-computed layout of the bucketed candidate list.
struct BucketState {
  uint32_t count[kMaxCfg];       // candidates per shape
  uint32_t first[kMaxCfg];       // first slot in the sorted id array
  uint32_t cursor[kMaxCfg];      // scatter cursors
  uint32_t tile_start[kMaxCfg + 1];
  uint32_t total_tiles;          // tiles of the first num_batched shapes
  uint32_t queue;                // persistent kernel work counter
  uint32_t pad[2];
  uint32_t next[kMaxCfg];        // plain launches: next warp tile per shape
};

struct DevInputs {
  const uint32_t* peq;           // qryEntry_t as 20 u32
  const uint2* qinfo;            // {posEntry, size}
  const Cand* cands;
  const uint32_t* ref;           // packed reference words
  unsigned long long ref_size;   // bases
  unsigned long long ref_words;  // readable words (packed + padding)
  uint2* results;                // {column, score}
  uint32_t* flags;               // device error flags (kFlag*)
  uint32_t num_cands;
  uint32_t num_queries;
  uint32_t num_entries;
  float distance;
  int exact;
  // Ukkonen cut-off: with `cut` set, a candidate whose minimum score exceeds
  // its bound k = (uint32_t)(m * cutoff) (float32) gets {kNoMatch, kNoMatch}.
  float cutoff;
  int cut;
  // The cut-off's first pass (prefix set): the DP runs on the first
  // prefix_rows(m) rows of each query only (prefix_rows in myers_device.cuh).
  // A candidate whose prefix minimum exceeds k cannot come within k and gets
  // {kNoMatch, kNoMatch}; the others are appended to esc_ids (shape
  // esc_cfg[id] of the second pass, or shape 0 without esc_cfg) for a second
  // pass over their full queries.
  int prefix;
  float prefix_mult;
  uint32_t* esc_ids;
  struct BucketState* esc_state;
  uint8_t* esc_cfg;
  // Multipliers the compiler cannot fold (set by set_multipliers): they keep
  // the per-column bookkeeping on the FMA pipe (see myers_kernels.cu).
  uint32_t one, two, k16, mk16, p28, kb33, kb17, mn16, mone;
};

inline void set_multipliers(DevInputs& in) {
  in.one = 1u;
  in.two = 2u;
  in.k16 = 1u << 16;
  in.mk16 = 0xFFFF0000u;
  in.p28 = 1u << 28;
  in.kb33 = 33u * 4u * 4u;  // bytes between the bases of a PEQ group, 33 columns
  in.kb17 = 17u * 4u * 4u;  // ... 17 columns
  in.mn16 = 0xFFFFFFF0u;    // -16
  in.mone = 0xFFFFFFFFu;    // -1
}

inline int variant_W(int v) { return v < kNumSingle ? v + 1 : kMultiW[v - kNumSingle]; }
inline bool variant_multi(int v) { return v >= kNumSingle; }
inline bool batched_supports(int v) { return !variant_multi(v) || variant_W(v) <= kBatchedMaxMultiW; }

// ---- host launchers (myers_kernels.cu) ----

// classify + plan + scatter; d_state must be zeroed first. Returns launches.
int launch_bucketing(const DevInputs& in, const PlanTable& plan, BucketState* d_state, uint8_t* d_cfg_of_cand,
                     uint32_t* d_ids, cudaStream_t s, int num_sms, cudaError_t* err);

// One plain launch of variant v. With d_state == nullptr the candidates are
// indices [first, first+count) (no bucketing); otherwise shape `cfg`'s range
// of the sorted id array, read from d_state on the device. d_next: the
// launch's warp-tile counter, zero when the launch starts.
cudaError_t launch_plain(int v, int L, const DevInputs& in, const uint32_t* d_ids, const BucketState* d_state,
                         int cfg, uint32_t first, uint32_t count, uint32_t* d_next, cudaStream_t s, int num_sms);

// The cut-off's bucketing: classify by the first pass's (prefix) shapes
// under `plan` and, for the candidates a prefix covers only in part, by their
// full-length shapes under `plan2` (into in.esc_cfg, counted in
// in.esc_state->cursor); then lay out both. d_state and in.esc_state must be
// zeroed first. Returns launches.
int launch_bucketing_cutoff(const DevInputs& in, const PlanTable& plan, const PlanTable& plan2,
                            BucketState* d_state, uint8_t* d_cfg_of_cand, uint32_t* d_ids, cudaStream_t s,
                            int num_sms, cudaError_t* err);

// The cut-off's second pass on the persistent path: tile layout of the lists
// the first pass filled (d_esc_state), after the first pass.
cudaError_t launch_plan_tiles(const PlanTable& plan2, BucketState* d_esc_state, cudaStream_t s);

// The persistent batched launch over the plan's first num_batched shapes;
// the grid is the device's resident capacity or, for small batches, one
// warp per tile of `max_tiles` (an upper bound of the tiles), whichever is
// smaller, so concurrent small batches share the device.
cudaError_t launch_batched(const DevInputs& in, const uint32_t* d_ids, const PlanTable& plan,
                           BucketState* d_state, cudaStream_t s, int num_sms, uint32_t max_tiles);

// Load every kernel the batched path can launch (bucketing, the persistent
// kernel, the plain launches of shapes it does not carry) on the current
// device. With lazy module loading a kernel is otherwise loaded, and its code
// allocated on the device, at its first launch.
cudaError_t load_batched_path_kernels();

// Bytes of shared memory one warp needs for a shape.
uint32_t warp_smem_bytes(int v, int L);

// Packers (ASCII -> PEQ entries; ASCII -> packed reference words).
cudaError_t launch_pack_peq(const uint8_t* ascii, unsigned long long ascii_bytes, const unsigned long long* offsets,
                            const uint2* qinfo, uint32_t num_reads, uint32_t* peq, uint32_t num_entries,
                            uint32_t* flags, cudaStream_t s, int num_sms);
cudaError_t launch_pack_reference(const uint8_t* ascii, unsigned long long n, uint32_t* words,
                                  unsigned long long nwords, cudaStream_t s, int num_sms);

// Integer-ALU peak probe: `iters` rounds of independent 3-input logic ops.
cudaError_t launch_lop3_probe(uint32_t* d_out, int blocks, int threads, int iters, cudaStream_t s);

// ---- host runtime internals (myers_api.cu) ----

// Shape plan for the word counts flagged in present[0..kMaxWords].
// n: the batch's candidates, which picks the batched path's table for large
// batches at kLargeBatchCandidates or more.
// reads: how many reads the n candidates come from (0: unknown).
int build_plan(PlanTable& t, const uint8_t* present, bool batched, uint32_t lane_words = 0, uint64_t n = 0,
               uint64_t reads = 0);
// Upper bound of the persistent kernel's tiles for n candidates under `plan`.
uint32_t batched_tile_bound(const PlanTable& plan, uint32_t n);
// Record a CUDA failure (message for myersGetErrorString) and return MYERS_E_CUDA.
int cuda_fail(cudaError_t e, const char* what);

}  // namespace myers

// Opaque handles of the C ABI (include/myers-interface.h).
struct myersReference {
  int device;
  uint32_t* d_words;
  uint64_t words;  // packed words (without padding)
  uint64_t size;   // bases
};

struct myersContext {
  int device;
  int num_sms;
  uint64_t capacity;
  uint32_t* d_ids;
  uint8_t* d_cfg;
  myers::BucketState* d_state;
  uint32_t* d_flags;
  uint32_t last_launches;
  // the cut-off's second pass (allocated at the first cut-off request)
  uint32_t* d_esc_ids;
  uint8_t* d_esc_cfg;
  myers::BucketState* d_esc_state;
  // streams the plain path spreads its per-shape launches over (forked from
  // and joined back to the caller's stream); null when they could not be made
  cudaStream_t aux[myers::kPlainStreams];
  cudaEvent_t fork;
  cudaEvent_t join[myers::kPlainStreams];
};

namespace myers {
// Enqueue the kernels of one batch on stream s (inputs already on the device).
// With in.cut and plan2 given, the cut-off runs in two passes: `plan` holds
// the first pass's (prefix) shapes and `plan2` the full-length shapes
// (cutoff_plans), on either path.
int verify_enqueue(myersContext* ctx, const myersReference* ref, const DevInputs& in, const PlanTable& plan, int path,
                   cudaStream_t s, const PlanTable* plan2 = nullptr);
// The cut-off's plans from the word counts of the full queries present: the
// first pass's prefix shapes into `plan`, the full-length shapes into
// `plan2`. `present_m[m]` flags each query length m (1..kMaxWords*32).
int cutoff_plans(PlanTable& plan, PlanTable& plan2, const uint8_t* present_m, float cutoff, float prefix_mult,
                 bool batched, uint64_t n);
// The first pass's rows of a query of m bases (as prefix_rows on the device).
uint32_t host_prefix_rows(uint32_t m, float cutoff, float prefix_mult);
// Device scratch of the cut-off's second pass for a context (once).
int ensure_cutoff_scratch(myersContext* ctx);
// The multiplier of the first pass's rows (MYERS_CUTOFF_PREFIX, default
// 2.25). A random decoy's prefix minimum sits close to 0.46-0.49 per row, so
// a prefix of 2.25 k rows (plus 8, rounded up to a word) settles almost every
// decoy while staying short.
float cutoff_prefix_mult();

// Capture what enqueue() puts on stream s and launch it as the graph *exec.
// Consecutive batches differ only in copy sizes and kernel arguments, so the
// executable graph is updated in place; when the topology changed (another
// set of length buckets on the plain path) it is instantiated anew. The
// capture is always ended, also when enqueue() fails.
template <class F>
int launch_as_graph(cudaStream_t s, cudaGraphExec_t* exec, F&& enqueue) {
  cudaError_t ce = cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed);
  if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamBeginCapture");
  const int st = enqueue();
  cudaGraph_t g = nullptr;
  ce = cudaStreamEndCapture(s, &g);
  if (st != 0 || ce != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return st != 0 ? st : cuda_fail(ce, "cudaStreamEndCapture");
  }
  if (*exec) {
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(*exec, g, &info) != cudaSuccess) {
      cudaGetLastError();
      cudaGraphExecDestroy(*exec);
      *exec = nullptr;
    }
  }
  if (*exec == nullptr && (ce = cudaGraphInstantiate(exec, g, 0)) != cudaSuccess) {
    *exec = nullptr;
    cudaGraphDestroy(g);
    return cuda_fail(ce, "cudaGraphInstantiate");
  }
  cudaGraphDestroy(g);
  ce = cudaGraphLaunch(*exec, s);
  return ce == cudaSuccess ? 0 : cuda_fail(ce, "cudaGraphLaunch");
}
}  // namespace myers
