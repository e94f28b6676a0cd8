// Host runtime and C ABI of libmyers_b200.so.
//
// Replaces the reference's host runtime (src-api/myersGPU.c): reference load,
// per-buffer pinned/device buffers and streams, send/receive, teardown. The
// differences that matter:
//  * all buffers live on one device, one stream each (the reference spreads
//    buffers over devices, myersGPU.c:303-341);
//  * buffers are sized from a memory budget, not 95% of free memory
//    (myersGPU.c:323-333);
//  * length bucketing runs on the device (the reference does three O(C)
//    passes on the host per send, myersGPU.c:351-422, and un-permutes the
//    results on the host, :500-513); results land in caller order directly;
//  * every input index is checked on the device, so malformed buffers give
//    flagged results instead of out-of-bounds reads;
//  * errors can be returned (myers*) as well as ending the process (the
//    reference's calls, which always exit).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <dlfcn.h>
#include <cuda.h>  // driver types only: entry points come through cudaGetDriverEntryPointByVersion
#include <cuda_runtime.h>

#include "../../include/myers-interface.h"
#include "myers_internal.h"

using namespace myers;

static_assert(sizeof(qryEntry_t) == 80, "qryEntry_t layout");
static_assert(sizeof(candInfo_t) == 16, "candInfo_t layout");
static_assert(sizeof(qryInfo_t) == 8, "qryInfo_t layout");
static_assert(sizeof(resEntry_t) == 8, "resEntry_t layout");
static_assert(sizeof(Cand) == 16, "Cand layout");

// ---------------------------------------------------------------------------
// errors

static thread_local char g_cuda_msg[256];

int myers::cuda_fail(cudaError_t e, const char* what) {
  snprintf(g_cuda_msg, sizeof(g_cuda_msg), "%s: %s", what, cudaGetErrorString(e));
  return MYERS_E_CUDA;
}

#define CU(call)                                   \
  do {                                             \
    cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

extern "C" const char* myersGetErrorString(int status) {
  switch (status) {
    case MYERS_SUCCESS: return "Myers - Success";
    case MYERS_E_OPENING_FILE: return "Myers - Error: opening file";
    case MYERS_E_READING_FILE: return "Myers - Error: reading file";
    case MYERS_E_INSUFFICIENT_MEM_GPU: return "Myers - Error: there aren't enough GPU memory space";
    case MYERS_E_ALLOCATE_MEM: return "Myers - Error: allocating data";
    case MYERS_E_INCOMPATIBLE_GPU: return "Myers - Error: incompatible GPU (needs compute capability 10.0)";
    case MYERS_E_INVALID_ARGUMENT: return "Myers - Error: invalid argument";
    case MYERS_E_CAPACITY: return "Myers - Error: more data than the buffer holds";
    case MYERS_E_QUERY_TOO_LONG: return "Myers - Error: query or window too long, or invalid query/PEQ indices";
    case MYERS_E_CUDA: return g_cuda_msg[0] ? g_cuda_msg : "Myers - Error: CUDA runtime call failed";
    case MYERS_E_TIMEOUT: return "Myers - Error: device wait timed out";
    case MYERS_E_NOT_READY: return "Myers - Error: not ready";
    case MYERS_E_BUSY: return "Myers - Error: busy";
    default: return "Myers - Unknown error";
  }
}

// The reference's convention: print and end the process (myersGPU.c:24-47).
static void fatal(int status, const char* where) {
  if (status != MYERS_SUCCESS) {
    fprintf(stderr, "%s in %s\n", myersGetErrorString(status), where);
    exit(EXIT_FAILURE);
  }
}

// ---------------------------------------------------------------------------
// reference


static int reference_upload(myersReference** out, const uint32_t* host, uint64_t words, uint64_t size) {
  if (out == nullptr || (words > 0 && host == nullptr)) return MYERS_E_INVALID_ARGUMENT;
  if (size > words * 8) return MYERS_E_INVALID_ARGUMENT;
  int dev = 0;
  CU(cudaGetDevice(&dev));
  int major = 0;
  CU(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  if (major < 10) return MYERS_E_INCOMPATIBLE_GPU;
  size_t freeb = 0, totalb = 0;
  CU(cudaMemGetInfo(&freeb, &totalb));
  const uint64_t bytes = (words + kRefPadWords) * 4;
  if (bytes > freeb) return MYERS_E_INSUFFICIENT_MEM_GPU;
  myersReference* r = new myersReference();
  r->device = dev;
  r->words = words;
  r->size = size;
  if (cudaMalloc((void**)&r->d_words, bytes) != cudaSuccess) {
    delete r;
    return MYERS_E_INSUFFICIENT_MEM_GPU;
  }
  cudaError_t e = cudaMemcpy(r->d_words, host, words * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    std::vector<uint32_t> pad(kRefPadWords, kPadWord);
    e = cudaMemcpy(r->d_words + words, pad.data(), kRefPadWords * 4, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    cudaFree(r->d_words);
    delete r;
    return cuda_fail(e, "reference upload");
  }
  *out = r;
  return MYERS_SUCCESS;
}

extern "C" int myersReferenceCreate(myersReference_t** ref, const uint32_t* hostWords, uint64_t numWords,
                                    uint64_t sizeBases) {
  return reference_upload(ref, hostWords, numWords, sizeBases);
}

// File format of src-api/genReference-4bits.c:121-140: u32 numEntries,
// u32 size, then numEntries packed words (read at src-api/myersGPU.c:106-128).
// The header is checked against the file's length before anything is
// allocated: a file that is shorter than its header says, or whose base count
// exceeds its words, is MYERS_E_READING_FILE (the reference reads whatever
// fread returns, myersGPU.c:117-122).
extern "C" int myersReferenceLoad(myersReference_t** ref, const char* fileName) {
  if (ref == nullptr || fileName == nullptr) return MYERS_E_INVALID_ARGUMENT;
  NvtxRange range("myers: reference load");
  FILE* fp = fopen(fileName, "rb");
  if (fp == nullptr) return MYERS_E_OPENING_FILE;
  uint32_t hdr[2];
  long long file_bytes = -1;
  if (fseek(fp, 0, SEEK_END) == 0) file_bytes = ftell(fp);
  if (file_bytes < 8 || fseek(fp, 0, SEEK_SET) != 0 || fread(hdr, sizeof(uint32_t), 2, fp) != 2 ||
      (unsigned long long)file_bytes < 8ull + 4ull * hdr[0] || (uint64_t)hdr[1] > (uint64_t)hdr[0] * 8) {
    fclose(fp);
    return MYERS_E_READING_FILE;
  }
  uint32_t* host = nullptr;
  if (cudaMallocHost((void**)&host, (size_t)hdr[0] * 4 + 4) != cudaSuccess) {
    fclose(fp);
    return MYERS_E_ALLOCATE_MEM;
  }
  size_t got = fread(host, sizeof(uint32_t), hdr[0], fp);
  fclose(fp);
  int st = MYERS_E_READING_FILE;
  if (got == hdr[0]) st = reference_upload(ref, host, hdr[0], hdr[1]);
  cudaFreeHost(host);
  return st;
}

extern "C" int myersReferenceDestroy(myersReference_t* ref) {
  if (ref == nullptr) return MYERS_E_INVALID_ARGUMENT;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(ref->device);
  cudaFree(ref->d_words);
  cudaSetDevice(cur);
  delete ref;
  return MYERS_SUCCESS;
}

extern "C" uint64_t myersReferenceSize(const myersReference_t* ref) { return ref ? ref->size : 0; }

// ---------------------------------------------------------------------------
// shapes and plans

// Lanes a candidate effectively occupies (a warp holds floor(32/L)
// candidates) times the instructions of one column step per lane.
static double shape_cost(int v, int L) {
  const int W = variant_W(v);
  if (!variant_multi(v)) return 10.0 * W + 8.0;
  const int nseg = 32 / L;
  return (32.0 / nseg) * (10.0 * W + 16.0);
}

// Optional per-word-count overrides (variant, L) set by the autotuner.
struct Override {
  bool set;
  uint8_t variant;
  uint8_t L;
};
static std::mutex g_override_mu;
static Override g_override[2][kMaxWords + 1];
// from the autotuner's cache file: plain, batched, and batched for large
// batches (see large_batch)
static Override g_tuned[3][kMaxWords + 1];

// Load the autotuner's cache: `autotune_b200.json` next to this library (or
// the file named by MYERS_AUTOTUNE; MYERS_AUTOTUNE=0 disables it). Format:
// {"plain": {"<words>": [W, L], ...}, "batched": {...}, "batched_large": {...}}
// with W words per lane and L lanes per candidate; entries naming a shape that
// is not compiled or that the path cannot run are ignored.
static void load_tuned_once() {
  static std::once_flag once;
  std::call_once(once, [] {
    std::string path;
    const char* env = getenv("MYERS_AUTOTUNE");
    if (env && strcmp(env, "0") == 0) return;
    if (env && *env) {
      path = env;
    } else {
      Dl_info info;
      if (dladdr((void*)&load_tuned_once, &info) == 0 || info.dli_fname == nullptr) return;
      path = info.dli_fname;
      const size_t slash = path.rfind('/');
      path = (slash == std::string::npos ? std::string(".") : path.substr(0, slash)) + "/autotune_b200.json";
    }
    FILE* fp = fopen(path.c_str(), "rb");
    if (fp == nullptr) return;
    std::string text;
    char buf[4096];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), fp)) > 0) text.append(buf, n);
    fclose(fp);
    std::lock_guard<std::mutex> lk(g_override_mu);
    for (int path_id = 0; path_id < 3; ++path_id) {
      const char* key = path_id == 0 ? "\"plain\"" : path_id == 1 ? "\"batched\"" : "\"batched_large\"";
      size_t at = text.find(key);
      if (at == std::string::npos) continue;
      at = text.find('{', at);
      const size_t end = text.find('}', at);
      if (at == std::string::npos || end == std::string::npos) continue;
      const char* p = text.c_str() + at;
      const char* e = text.c_str() + end;
      while (p < e) {
        unsigned w = 0;
        int W = 0, L = 0, used = 0;
        if (sscanf(p, " \"%u\" : [ %d , %d ]%n", &w, &W, &L, &used) == 3 && used > 0) {
          // [W, L]: L == 1 is one candidate per lane with W words, L >= 2 a
          // candidate over L lanes of W words
          int v = -1;
          if (L == 1 && W >= 1 && W <= kNumSingle) v = W - 1;
          for (int mi = 0; L >= 2 && mi < kNumMulti; ++mi)
            if (kMultiW[mi] == W) v = kNumSingle + mi;
          if (v >= 0 && w >= 1 && w <= kMaxWords && L <= 32 && (uint32_t)(W * L) >= w &&
              (path_id == 0 || batched_supports(v)))
            g_tuned[path_id][w] = Override{true, (uint8_t)v, (uint8_t)L};
          p += used;
        } else {
          ++p;
        }
      }
    }
  });
}

// Whether a batch of n candidates takes the batched path's shapes for large
// batches. Those use every lane width, which fills the lanes best; but the
// persistent kernel runs whatever tiles come next, and in a small batch of
// long reads the tiles of many different shapes run side by side and thrash
// the instruction cache (10K long-read candidates: 12.2 ms with them, 8.2 ms
// with the few-width table; 125K: 80.1 against 79.2 ms; 250K: 151.3 against
// 156.6 ms; 500K: 296 against 312 ms). MYERS_LARGE_BATCH sets the threshold
// in candidates.
static bool large_batch(uint64_t n) {
  static const uint64_t threshold = [] {
    const char* env = getenv("MYERS_LARGE_BATCH");
    return env ? strtoull(env, nullptr, 10) : (uint64_t)kLargeBatchCandidates;
  }();
  return n >= threshold;
}

// How many of a context's streams the plain path spreads its launches over
// (MYERS_PLAIN_STREAMS, 1..kPlainStreams; 1 keeps them on the caller's stream).
static int plain_streams() {
  static const int k = [] {
    const char* env = getenv("MYERS_PLAIN_STREAMS");
    const int v = env ? atoi(env) : kPlainStreams;
    return v < 1 ? 1 : (v > kPlainStreams ? kPlainStreams : v);
  }();
  return k;
}

// Whether a batch of n candidates on the batched path takes latency shapes
// (lanes of at most kSmallBatchLaneWords words) for reads of up to 1,024
// bases. A small batch runs about one wave of tiles and ends with its longest
// tile; lanes of 12 words make the tiles of 1,000-base reads a quarter as long
// for about 13% more instructions (mixed reads of 100..1,000 bases: 11K
// candidates 0.93 -> 0.45 ms, 110K 1.50 -> 0.90 ms, 220K 1.86 -> 1.70 ms;
// 330K 2.44 -> 2.53 ms, 1.1M 7.3 -> 8.4 ms).
// MYERS_SMALL_BATCH sets the threshold in candidates (0 turns it off).
static bool small_batch(uint64_t n) {
  static const uint64_t threshold = [] {
    const char* env = getenv("MYERS_SMALL_BATCH");
    return env ? strtoull(env, nullptr, 10) : (uint64_t)kSmallBatchCandidates;
  }();
  return n > 0 && n < threshold;
}

// lane_words > 0 asks for latency-oriented shapes: a query of more than
// lane_words words is spread over ceil(words / W) lanes of W <= lane_words
// words, the cheapest such shape by the cost model (shorter per-candidate
// time, some more instructions). `large`: the batch is large (large_batch).
static Shape pick_shape(uint32_t w, bool batched, uint32_t lane_words = 0, bool large = false) {
  load_tuned_once();
  {
    std::lock_guard<std::mutex> lk(g_override_mu);
    const Override& o = g_override[batched ? 1 : 0][w];
    if (o.set) return Shape{o.variant, o.L, (uint8_t)variant_W(o.variant), 0};
  }
  if (lane_words > 0 && w > lane_words) {
    // the cheapest multi-lane shape whose lanes hold at most lane_words words
    // (the smallest width if none does)
    double best = 1e300;
    Shape bs{0, 0, 0, 0};
    for (int mi = 0; mi < kNumMulti; ++mi) {
      const uint32_t W = (uint32_t)kMultiW[mi];
      if ((W > lane_words && mi > 0) || (batched && W > (uint32_t)kBatchedMaxMultiW)) continue;
      const uint32_t L = (w + W - 1) / W;
      if (L < 2 || L > 32) continue;
      const double c = shape_cost(kNumSingle + mi, (int)L);
      if (c < best) {
        best = c;
        bs = Shape{(uint8_t)(kNumSingle + mi), (uint8_t)L, (uint8_t)W, 0};
      }
    }
    if (bs.L) return bs;
  }
  {
    std::lock_guard<std::mutex> lk(g_override_mu);
    if (batched && large && g_tuned[2][w].set) {
      const Override& o = g_tuned[2][w];
      return Shape{o.variant, o.L, (uint8_t)variant_W(o.variant), 0};
    }
    const Override& o = g_tuned[batched ? 1 : 0][w];
    if (o.set) return Shape{o.variant, o.L, (uint8_t)variant_W(o.variant), 0};
  }
  if (w <= 32) return Shape{(uint8_t)(w - 1), 1, (uint8_t)w, 0};
  double best = 1e300;
  Shape bs{0, 0, 0, 0};
  for (int mi = 0; mi < kNumMulti; ++mi) {
    const int W = kMultiW[mi];
    const uint32_t L = (w + W - 1) / W;
    if (L < 2 || L > 32) continue;
    const double c = shape_cost(kNumSingle + mi, (int)L);
    // batched shapes that the persistent kernel cannot carry cost extra
    const double pen = (batched && W > kBatchedMaxMultiW) ? 4.0 : 1.0;
    if (c * pen < best) {
      best = c * pen;
      bs = Shape{(uint8_t)(kNumSingle + mi), (uint8_t)L, (uint8_t)W, 0};
    }
  }
  return bs;
}

// Build the plan for the word counts flagged in `present` (size kMaxWords+1).
// Uses fixed-size stack arrays only: no allocation on the send path.
int myers::build_plan(PlanTable& t, const uint8_t* present, bool batched, uint32_t lane_words, uint64_t n,
                      uint64_t reads) {
  memset(&t, 0, sizeof(t));
  memset(t.cfg_of_words, kNoCfg, sizeof(t.cfg_of_words));
  Shape shapes[kMaxCfg];
  uint32_t max_words[kMaxCfg];
  int16_t cfg_of[kMaxWords + 1];
  int nshapes = 0;
  for (uint32_t w = 0; w <= kMaxWords; ++w) cfg_of[w] = -1;
  const bool small = batched && lane_words == 0 && small_batch(n);
  // Fewer than two candidates per read: a warp of 32 one-lane candidates then
  // holds more distinct reads than the 16 PEQ slots of the single-lane shapes
  // of more than 16 words, and runs its lanes in two rounds. Lanes of at most
  // 16 words stage each lane's own words instead.
  const bool distinct = lane_words == 0 && reads > 0 && n < 2 * reads;
  for (uint32_t w = 1; w <= kMaxWords; ++w) {
    if (!present[w]) continue;
    uint32_t lw = lane_words;
    if (small && w <= 32) lw = kSmallBatchLaneWords;
    else if (distinct && w > kDistinctLaneWords && w <= 32) lw = kDistinctLaneWords;
    const Shape s = pick_shape(w, batched, lw, large_batch(n));
    if (s.L == 0) return MYERS_E_QUERY_TOO_LONG;
    int found = -1;
    for (int i = 0; i < nshapes; ++i)
      if (shapes[i].variant == s.variant && shapes[i].L == s.L) found = i;
    if (found < 0) {
      if (nshapes == kMaxCfg) return MYERS_E_QUERY_TOO_LONG;
      shapes[nshapes] = s;
      max_words[nshapes] = w;
      found = nshapes++;
    }
    if (w > max_words[found]) max_words[found] = w;
    cfg_of[w] = (int16_t)found;
  }
  // order: persistent-kernel shapes first, each group by decreasing cost
  int order[kMaxCfg];
  double cost[kMaxCfg];
  bool group[kMaxCfg];
  for (int i = 0; i < nshapes; ++i) {
    order[i] = i;
    group[i] = !batched_supports(shapes[i].variant);
    cost[i] = shape_cost(shapes[i].variant, shapes[i].L) * max_words[i];
  }
  auto before = [&](int a, int b) { return group[a] != group[b] ? group[a] < group[b] : cost[a] > cost[b]; };
  for (int i = 1; i < nshapes; ++i)
    for (int j = i; j > 0 && before(order[j], order[j - 1]); --j) {
      const int x = order[j];
      order[j] = order[j - 1];
      order[j - 1] = x;
    }
  int rank[kMaxCfg];
  t.num_cfg = (uint32_t)nshapes;
  t.num_batched = 0;
  for (int r = 0; r < nshapes; ++r) {
    rank[order[r]] = r;
    t.shape[r] = shapes[order[r]];
    if (batched_supports(t.shape[r].variant)) t.num_batched = (uint32_t)r + 1;
  }
  for (uint32_t w = 1; w <= kMaxWords; ++w)
    if (cfg_of[w] >= 0) t.cfg_of_words[w] = (uint8_t)rank[cfg_of[w]];
  return MYERS_SUCCESS;
}

// ---------------------------------------------------------------------------
// context: device scratch for bucketing


static void destroy_plain_streams(myersContext* c) {
  for (int i = 0; i < kPlainStreams; ++i) {
    if (c->aux[i]) cudaStreamDestroy(c->aux[i]);
    if (c->join[i]) cudaEventDestroy(c->join[i]);
    c->aux[i] = nullptr;
    c->join[i] = nullptr;
  }
  if (c->fork) cudaEventDestroy(c->fork);
  c->fork = nullptr;
}

extern "C" int myersContextCreate(myersContext_t** out, uint64_t maxCandidates) {
  if (out == nullptr || maxCandidates > 0xFFFFFFFFull) return MYERS_E_INVALID_ARGUMENT;
  myersContext* c = new myersContext();
  memset(c, 0, sizeof(*c));
  cudaError_t e = cudaGetDevice(&c->device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device);
  c->capacity = maxCandidates;
  const size_t n = maxCandidates ? maxCandidates : 1;
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_ids, n * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_cfg, n);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_state, sizeof(BucketState));
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_flags, 4);
  if (e == cudaSuccess) e = cudaMemset(c->d_flags, 0, 4);
  if (e != cudaSuccess) {
    cudaFree(c->d_ids);
    cudaFree(c->d_cfg);
    cudaFree(c->d_state);
    cudaFree(c->d_flags);
    delete c;
    return e == cudaErrorMemoryAllocation ? MYERS_E_INSUFFICIENT_MEM_GPU : cuda_fail(e, "context");
  }
  // The plain path's streams. Without them its launches stay on the caller's
  // stream, one after another.
  bool streams = cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming) == cudaSuccess;
  for (int i = 0; i < kPlainStreams && streams; ++i)
    streams = cudaStreamCreateWithFlags(&c->aux[i], cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&c->join[i], cudaEventDisableTiming) == cudaSuccess;
  if (!streams) {
    destroy_plain_streams(c);
    cudaGetLastError();
  }
  *out = c;
  return MYERS_SUCCESS;
}

extern "C" int myersContextDestroy(myersContext_t* c) {
  if (c == nullptr) return MYERS_E_INVALID_ARGUMENT;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(c->device);
  cudaFree(c->d_ids);
  cudaFree(c->d_cfg);
  cudaFree(c->d_state);
  cudaFree(c->d_flags);
  cudaFree(c->d_esc_ids);
  cudaFree(c->d_esc_cfg);
  cudaFree(c->d_esc_state);
  destroy_plain_streams(c);
  cudaSetDevice(cur);
  delete c;
  return MYERS_SUCCESS;
}

int myers::ensure_cutoff_scratch(myersContext* c) {
  if (c->d_esc_ids != nullptr) return MYERS_SUCCESS;
  const size_t n = c->capacity ? c->capacity : 1;
  cudaError_t e = cudaMalloc((void**)&c->d_esc_ids, n * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_esc_cfg, n);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_esc_state, sizeof(BucketState));
  if (e != cudaSuccess) {
    cudaFree(c->d_esc_ids);
    cudaFree(c->d_esc_cfg);
    cudaFree(c->d_esc_state);
    c->d_esc_ids = nullptr;
    c->d_esc_cfg = nullptr;
    c->d_esc_state = nullptr;
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? MYERS_E_INSUFFICIENT_MEM_GPU : cuda_fail(e, "cut-off scratch");
  }
  return MYERS_SUCCESS;
}

float myers::cutoff_prefix_mult() {
  static const float mult = [] {
    const char* env = getenv("MYERS_CUTOFF_PREFIX");
    const float v = env ? strtof(env, nullptr) : 0.0f;
    return v > 0.0f ? v : 2.25f;
  }();
  return mult;
}

uint32_t myers::host_prefix_rows(uint32_t m, float cutoff, float mult) {
  const uint32_t k = (uint32_t)((float)m * cutoff);
  const float r = mult * (float)k;
  const uint32_t rows = r >= 65536.0f ? 0xFFFFFFFFu : (((uint32_t)r + 8u + 31u) & ~31u);
  return rows < m ? rows : m;
}

int myers::cutoff_plans(PlanTable& plan, PlanTable& plan2, const uint8_t* present_m, float cutoff, float mult,
                        bool batched, uint64_t n) {
  uint8_t w1[kMaxWords + 1], w2[kMaxWords + 1];
  memset(w1, 0, sizeof(w1));
  memset(w2, 0, sizeof(w2));
  for (uint32_t m = 1; m <= kMaxWords * 32; ++m) {
    if (!present_m[m]) continue;
    const uint32_t r = host_prefix_rows(m, cutoff, mult);
    w1[(r + 31) / 32] = 1;
    if (r < m) w2[(m + 31) / 32] = 1;
  }
  const int st = build_plan(plan, w1, batched, 0, n);
  // the second pass holds the candidates that survived, mostly one per read
  return st != MYERS_SUCCESS ? st : build_plan(plan2, w2, batched, 0, n, n);
}

extern "C" uint32_t myersContextLastLaunches(const myersContext_t* c) { return c ? c->last_launches : 0; }

// Enqueue the kernels for one batch. `uniform`: every query maps to the same
// (single) shape of `plan`, so no bucketing is needed on the plain path.
// Most work tiles the persistent kernel can see for n candidates: every
// candidate in the shape with the fewest candidates per tile, plus one
// partial tile per shape.
uint32_t myers::batched_tile_bound(const PlanTable& plan, uint32_t n) {
  uint32_t nseg_min = 32;
  for (uint32_t c = 0; c < plan.num_batched; ++c) {
    const Shape sh = plan.shape[c];
    const uint32_t nseg = variant_multi(sh.variant) ? 32u / sh.L : 32u;
    if (nseg < nseg_min) nseg_min = nseg;
  }
  return (uint32_t)(((uint64_t)n + nseg_min - 1) / nseg_min + plan.num_batched);
}

int myers::verify_enqueue(myersContext* ctx, const myersReference* ref, const DevInputs& in0, const PlanTable& plan,
                          int path, cudaStream_t s, const PlanTable* plan2) {
  DevInputs in = in0;
  in.ref = ref->d_words;
  in.ref_size = ref->size;
  in.ref_words = ref->words + kRefPadWords;
  in.flags = ctx->d_flags;
  set_multipliers(in);
  ctx->last_launches = 0;
  if (in.num_cands == 0) return MYERS_SUCCESS;
  if (in.num_cands > ctx->capacity) return MYERS_E_CAPACITY;
  if (plan.num_cfg == 0) {
    // no query needs the DP (all empty or all too long): classify alone
    // writes every result
  }
  auto plain = [&](uint32_t c, const uint32_t* ids, const BucketState* st, uint32_t count, uint32_t* next) {
    const Shape sh = plan.shape[c];
    return launch_plain(sh.variant, sh.L, in, ids, st, (int)c, 0, count, next, s, ctx->num_sms);
  };
  // Plain launches of shapes c0..c1-1 of `pl` over the lists in `st`. With
  // more than one shape they are spread over the context's streams, forked
  // from s and joined back to it: each launch ends in a partial wave, which
  // the other shapes' launches fill.
  auto plain_range = [&](const PlanTable& pl, const DevInputs& din, uint32_t c0, uint32_t c1, const uint32_t* ids,
                         BucketState* st) -> cudaError_t {
    const uint32_t k = c1 - c0 < (uint32_t)plain_streams() ? c1 - c0 : (uint32_t)plain_streams();
    cudaError_t e = cudaSuccess;
    if (k <= 1 || ctx->aux[0] == nullptr) {
      for (uint32_t c = c0; c < c1 && e == cudaSuccess; ++c)
        e = launch_plain(pl.shape[c].variant, pl.shape[c].L, din, ids, st, (int)c, 0, 0, &st->next[c], s,
                         ctx->num_sms);
      return e;
    }
    e = cudaEventRecord(ctx->fork, s);
    for (uint32_t i = 0; i < k && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(ctx->aux[i], ctx->fork, 0);
    for (uint32_t c = c0; c < c1 && e == cudaSuccess; ++c)
      e = launch_plain(pl.shape[c].variant, pl.shape[c].L, din, ids, st, (int)c, 0, 0, &st->next[c],
                       ctx->aux[(c - c0) % k], ctx->num_sms);
    for (uint32_t i = 0; i < k && e == cudaSuccess; ++i) {
      e = cudaEventRecord(ctx->join[i], ctx->aux[i]);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ctx->join[i], 0);
    }
    return e;
  };
  if (in.cut && path == MYERS_PATH_BATCHED && plan2 != nullptr) {
    // The cut-off's two passes as two persistent launches: the first over
    // the prefixes' tiles (plan), then the tile layout of the lists it filled,
    // then the second over those lists' full queries (plan2). Shapes the
    // persistent kernel does not carry get plain launches after each.
    if (ctx->d_esc_ids == nullptr) return MYERS_E_INVALID_ARGUMENT;  // ensure_cutoff_scratch first
    in.prefix = 1;
    in.esc_ids = ctx->d_esc_ids;
    in.esc_state = ctx->d_esc_state;
    in.esc_cfg = ctx->d_esc_cfg;
    CU(cudaMemsetAsync(ctx->d_esc_state, 0, sizeof(BucketState), s));
    CU(cudaMemsetAsync(ctx->d_state, 0, sizeof(BucketState), s));
    cudaError_t e = cudaSuccess;
    uint32_t launches = (uint32_t)launch_bucketing_cutoff(in, plan, *plan2, ctx->d_state, ctx->d_cfg, ctx->d_ids, s,
                                                          ctx->num_sms, &e);
    if (e != cudaSuccess) return cuda_fail(e, "bucketing");
    if (plan.num_batched > 0) {
      CU(launch_batched(in, ctx->d_ids, plan, ctx->d_state, s, ctx->num_sms, batched_tile_bound(plan, in.num_cands)));
      ++launches;
    }
    for (uint32_t c = plan.num_batched; c < plan.num_cfg; ++c) {
      CU(plain(c, ctx->d_ids, ctx->d_state, 0, &ctx->d_state->next[c]));
      ++launches;
    }
    DevInputs in2 = in;
    in2.prefix = 0;
    CU(launch_plan_tiles(*plan2, ctx->d_esc_state, s));
    ++launches;
    if (plan2->num_batched > 0) {
      CU(launch_batched(in2, ctx->d_esc_ids, *plan2, ctx->d_esc_state, s, ctx->num_sms,
                        batched_tile_bound(*plan2, in.num_cands)));
      ++launches;
    }
    for (uint32_t c = plan2->num_batched; c < plan2->num_cfg; ++c) {
      const Shape sh = plan2->shape[c];
      CU(launch_plain(sh.variant, sh.L, in2, ctx->d_esc_ids, ctx->d_esc_state, (int)c, 0, 0,
                      &ctx->d_esc_state->next[c], s, ctx->num_sms));
      ++launches;
    }
    ctx->last_launches = launches;
    return MYERS_SUCCESS;
  }
  if (in.cut && path == MYERS_PATH_PLAIN && plan2 != nullptr) {
    // Ukkonen's cut-off in two passes. The first runs every candidate's DP
    // on a prefix of its query (plan: the prefixes' shapes) and settles the
    // candidates whose prefix minimum exceeds the bound; the others are
    // appended to lists by full-length shape (plan2), and the second pass
    // runs their full queries.
    if (ctx->d_esc_ids == nullptr) return MYERS_E_INVALID_ARGUMENT;  // ensure_cutoff_scratch first
    in.prefix = 1;
    in.esc_ids = ctx->d_esc_ids;
    in.esc_state = ctx->d_esc_state;
    CU(cudaMemsetAsync(ctx->d_esc_state, 0, sizeof(BucketState), s));
    uint32_t launches = 0;
    if (plan.num_cfg <= 1 && plan2->num_cfg <= 1) {
      in.esc_cfg = nullptr;  // one full-length shape: list 0
      if (plan.num_cfg == 1) {
        uint32_t* next = &ctx->d_state->next[0];
        CU(cudaMemsetAsync(next, 0, sizeof(uint32_t), s));
        CU(plain(0, nullptr, nullptr, in.num_cands, next));
        ++launches;
      }
    } else {
      in.esc_cfg = ctx->d_esc_cfg;
      CU(cudaMemsetAsync(ctx->d_state, 0, sizeof(BucketState), s));
      cudaError_t e = cudaSuccess;
      launches += (uint32_t)launch_bucketing_cutoff(in, plan, *plan2, ctx->d_state, ctx->d_cfg, ctx->d_ids, s,
                                                    ctx->num_sms, &e);
      if (e != cudaSuccess) return cuda_fail(e, "bucketing");
      CU(plain_range(plan, in, 0, plan.num_cfg, ctx->d_ids, ctx->d_state));
      launches += plan.num_cfg;
    }
    DevInputs in2 = in;
    in2.prefix = 0;
    CU(plain_range(*plan2, in2, 0, plan2->num_cfg, ctx->d_esc_ids, ctx->d_esc_state));
    launches += plan2->num_cfg;
    ctx->last_launches = launches;
    return MYERS_SUCCESS;
  }
  if (path == MYERS_PATH_PLAIN && plan.num_cfg == 1) {
    uint32_t* next = &ctx->d_state->next[0];  // the launch's tile counter
    CU(cudaMemsetAsync(next, 0, sizeof(uint32_t), s));
    CU(plain(0, nullptr, nullptr, in.num_cands, next));
    ctx->last_launches = 1;
    return MYERS_SUCCESS;
  }
  CU(cudaMemsetAsync(ctx->d_state, 0, sizeof(BucketState), s));
  cudaError_t e = cudaSuccess;
  uint32_t launches = (uint32_t)launch_bucketing(in, plan, ctx->d_state, ctx->d_cfg, ctx->d_ids, s, ctx->num_sms, &e);
  if (e != cudaSuccess) return cuda_fail(e, "bucketing");
  uint32_t first_plain = 0;
  if (path == MYERS_PATH_BATCHED && plan.num_batched > 0) {
    CU(launch_batched(in, ctx->d_ids, plan, ctx->d_state, s, ctx->num_sms, batched_tile_bound(plan, in.num_cands)));
    ++launches;
    first_plain = plan.num_batched;
  }
  CU(plain_range(plan, in, first_plain, plan.num_cfg, ctx->d_ids, ctx->d_state));
  launches += plan.num_cfg - first_plain;
  ctx->last_launches = launches;
  return MYERS_SUCCESS;
}

static int plan_for_range(PlanTable& plan, uint32_t minSize, uint32_t maxSize, int path, uint64_t n,
                          uint64_t reads) {
  uint8_t present[kMaxWords + 1];
  memset(present, 0, sizeof(present));
  if (maxSize == 0) maxSize = kMaxWords * 32;
  if (maxSize > kMaxWords * 32) maxSize = kMaxWords * 32;
  const uint32_t wlo = minSize ? (minSize + 31) / 32 : 1, whi = (maxSize + 31) / 32;
  for (uint32_t w = wlo; w <= whi; ++w) present[w] = 1;
  return build_plan(plan, present, path == MYERS_PATH_BATCHED, 0, n, reads);
}

extern "C" int myersVerifyAsync(myersContext_t* ctx, const myersReference_t* ref, const qryEntry_t* d_peq,
                                uint32_t numPEQEntries, const qryInfo_t* d_qinfo, uint32_t numQueries,
                                const candInfo_t* d_cands, uint32_t numCandidates, float distance,
                                int windowMode, int path, resEntry_t* d_results, void* stream) {
  return myersVerifyRangeAsync(ctx, ref, d_peq, numPEQEntries, d_qinfo, numQueries, d_cands, numCandidates,
                               distance, windowMode, path, 0, 0, d_results, stream);
}

static int verify_range(myersContext_t* ctx, const myersReference_t* ref, const qryEntry_t* d_peq,
                        uint32_t numPEQEntries, const qryInfo_t* d_qinfo, uint32_t numQueries,
                        const candInfo_t* d_cands, uint32_t numCandidates, float distance, int windowMode, int path,
                        float cutoff, uint32_t minQuerySize, uint32_t maxQuerySize, resEntry_t* d_results,
                        void* stream);

extern "C" int myersVerifyRangeAsync(myersContext_t* ctx, const myersReference_t* ref, const qryEntry_t* d_peq,
                                     uint32_t numPEQEntries, const qryInfo_t* d_qinfo, uint32_t numQueries,
                                     const candInfo_t* d_cands, uint32_t numCandidates, float distance,
                                     int windowMode, int path, uint32_t minQuerySize, uint32_t maxQuerySize,
                                     resEntry_t* d_results, void* stream) {
  return verify_range(ctx, ref, d_peq, numPEQEntries, d_qinfo, numQueries, d_cands, numCandidates, distance,
                      windowMode, path, -1.0f, minQuerySize, maxQuerySize, d_results, stream);
}

// Ukkonen's cut-off (GEMTools/src/gt_map_align_bpm.c:141-210,
// gt_map_block_bpm_get_distance__cutoff): the result is exact where the
// minimum is at most (uint32_t)(m * cutoff), else {MYERS_NO_MATCH,
// MYERS_NO_MATCH}. The plain path's single-lane shapes of 8..32 words (a
// multiple of 4) skip the rows above the band; other shapes and the batched
// path compute every row and apply the same contract.
extern "C" int myersVerifyCutoffAsync(myersContext_t* ctx, const myersReference_t* ref, const qryEntry_t* d_peq,
                                      uint32_t numPEQEntries, const qryInfo_t* d_qinfo, uint32_t numQueries,
                                      const candInfo_t* d_cands, uint32_t numCandidates, float distance,
                                      int windowMode, int path, float cutoff, uint32_t minQuerySize,
                                      uint32_t maxQuerySize, resEntry_t* d_results, void* stream) {
  if (!(cutoff >= 0.0f) || !std::isfinite(cutoff)) return MYERS_E_INVALID_ARGUMENT;
  return verify_range(ctx, ref, d_peq, numPEQEntries, d_qinfo, numQueries, d_cands, numCandidates, distance,
                      windowMode, path, cutoff, minQuerySize, maxQuerySize, d_results, stream);
}

static int verify_range(myersContext_t* ctx, const myersReference_t* ref, const qryEntry_t* d_peq,
                        uint32_t numPEQEntries, const qryInfo_t* d_qinfo, uint32_t numQueries,
                        const candInfo_t* d_cands, uint32_t numCandidates, float distance, int windowMode, int path,
                        float cutoff, uint32_t minQuerySize, uint32_t maxQuerySize, resEntry_t* d_results,
                        void* stream) {
  if (ctx == nullptr || ref == nullptr) return MYERS_E_INVALID_ARGUMENT;
  if (!(distance >= 0.0f) || !std::isfinite(distance)) return MYERS_E_INVALID_ARGUMENT;
  NvtxRange range("myers: verify (enqueue)");
  if (windowMode != MYERS_WINDOW_ALIGNED && windowMode != MYERS_WINDOW_EXACT) return MYERS_E_INVALID_ARGUMENT;
  if (path != MYERS_PATH_PLAIN && path != MYERS_PATH_BATCHED) return MYERS_E_INVALID_ARGUMENT;
  if (numCandidates > 0 && (d_peq == nullptr || d_qinfo == nullptr || d_cands == nullptr || d_results == nullptr))
    return MYERS_E_INVALID_ARGUMENT;
  PlanTable plan, plan2;
  const bool two_pass = cutoff >= 0.0f;
  const float mult = cutoff_prefix_mult();
  int st;
  if (two_pass) {
    std::vector<uint8_t> present_m(kMaxWords * 32 + 1, 0);
    const uint32_t hi = (maxQuerySize == 0 || maxQuerySize > kMaxWords * 32) ? kMaxWords * 32 : maxQuerySize;
    for (uint32_t m = minQuerySize ? minQuerySize : 1; m <= hi; ++m) present_m[m] = 1;
    st = cutoff_plans(plan, plan2, present_m.data(), cutoff, mult, path == MYERS_PATH_BATCHED, numCandidates);
    if (st == MYERS_SUCCESS) st = ensure_cutoff_scratch(ctx);
  } else {
    st = plan_for_range(plan, minQuerySize, maxQuerySize, path, numCandidates, numQueries);
  }
  if (st != MYERS_SUCCESS) return st;
  DevInputs in;
  memset(&in, 0, sizeof(in));
  in.prefix_mult = mult;
  in.peq = reinterpret_cast<const uint32_t*>(d_peq);
  in.qinfo = reinterpret_cast<const uint2*>(d_qinfo);
  in.cands = reinterpret_cast<const Cand*>(d_cands);
  in.results = reinterpret_cast<uint2*>(d_results);
  in.num_cands = numCandidates;
  in.num_queries = numQueries;
  in.num_entries = numPEQEntries;
  in.distance = distance;
  in.exact = windowMode == MYERS_WINDOW_EXACT;
  in.cut = cutoff >= 0.0f;
  in.cutoff = in.cut ? cutoff : 0.0f;
  return verify_enqueue(ctx, ref, in, plan, path, (cudaStream_t)stream, two_pass ? &plan2 : nullptr);
}

extern "C" int myersContextFlags(myersContext_t* ctx, uint32_t* flags, int clear) {
  if (ctx == nullptr || flags == nullptr) return MYERS_E_INVALID_ARGUMENT;
  CU(cudaMemcpy(flags, ctx->d_flags, 4, cudaMemcpyDeviceToHost));
  if (clear) CU(cudaMemset(ctx->d_flags, 0, 4));
  return MYERS_SUCCESS;
}

// PEQ entries from ASCII reads on the device (genCandidate-reorder.c:258-317
// as a kernel): read r is ascii[offsets[r] .. offsets[r] + qinfo[r].size),
// its entries go to d_peq + qinfo[r].posEntry. Reads whose entries or bytes
// fall outside the buffers are skipped and raise flag 4 on the context.
extern "C" int myersPackPEQAsync(myersContext_t* ctx, const uint8_t* d_ascii, uint64_t asciiBytes,
                                 const uint64_t* d_offsets, const qryInfo_t* d_qinfo, uint32_t numReads,
                                 qryEntry_t* d_peq, uint32_t numPEQEntries, void* stream) {
  if (ctx == nullptr || (numReads > 0 && (d_ascii == nullptr || d_offsets == nullptr || d_qinfo == nullptr ||
                                           d_peq == nullptr)))
    return MYERS_E_INVALID_ARGUMENT;
  CU(launch_pack_peq(d_ascii, asciiBytes, reinterpret_cast<const unsigned long long*>(d_offsets),
                     reinterpret_cast<const uint2*>(d_qinfo), numReads, reinterpret_cast<uint32_t*>(d_peq),
                     numPEQEntries, ctx->d_flags, (cudaStream_t)stream, ctx->num_sms));
  return MYERS_SUCCESS;
}

// Packed reference words from ASCII bases on the device
// (genReference-4bits.c:43-72 as a kernel): numWords words, bases at or past
// numBases are N.
extern "C" int myersPackReferenceAsync(const uint8_t* d_ascii, uint64_t numBases, uint32_t* d_words,
                                       uint64_t numWords, void* stream) {
  if (numWords > 0 && (d_ascii == nullptr || d_words == nullptr)) return MYERS_E_INVALID_ARGUMENT;
  int dev = 0, sms = 0;
  CU(cudaGetDevice(&dev));
  CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  CU(launch_pack_reference(d_ascii, numBases, d_words, numWords, (cudaStream_t)stream, sms));
  return MYERS_SUCCESS;
}

// Autotuner hook: force the shape of one word count (variant, L); variant
// -1 clears the override.
extern "C" int myersSetShapeOverride(int path, uint32_t words, int variant, int L) {
  if ((path != MYERS_PATH_PLAIN && path != MYERS_PATH_BATCHED) || words == 0 || words > kMaxWords)
    return MYERS_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(g_override_mu);
  Override& o = g_override[path][words];
  if (variant < 0) {
    o.set = false;
    return MYERS_SUCCESS;
  }
  if (variant >= kNumVariants) return MYERS_E_INVALID_ARGUMENT;
  if (!variant_multi(variant)) L = 1;
  if (L < 1 || L > 32 || (uint32_t)(variant_W(variant) * L) < words) return MYERS_E_INVALID_ARGUMENT;
  if (path == MYERS_PATH_BATCHED && variant_multi(variant) == false && !batched_supports(variant))
    return MYERS_E_INVALID_ARGUMENT;
  o.set = true;
  o.variant = (uint8_t)variant;
  o.L = (uint8_t)L;
  return MYERS_SUCCESS;
}

// Shape the plan would use for a query length (for tests and the autotuner).
extern "C" int myersShapeOf(int path, uint32_t querySize, int* variant, int* L, int* W) {
  if (querySize == 0 || querySize > kMaxWords * 32 || variant == nullptr || L == nullptr || W == nullptr)
    return MYERS_E_INVALID_ARGUMENT;
  const Shape s = pick_shape((querySize + 31) / 32, path == MYERS_PATH_BATCHED);
  *variant = s.variant;
  *L = s.L;
  *W = s.W;
  return MYERS_SUCCESS;
}

// Word counts with an autotuned shape for the path (0 if no cache was loaded).
extern "C" int myersTunedShapes(int path) {
  if (path != MYERS_PATH_PLAIN && path != MYERS_PATH_BATCHED) return -1;
  load_tuned_once();
  std::lock_guard<std::mutex> lk(g_override_mu);
  int n = 0;
  for (uint32_t w = 1; w <= kMaxWords; ++w) n += g_tuned[path][w].set;
  return n;
}

extern "C" int myersNumVariants(void) { return kNumVariants; }
extern "C" int myersVariantWords(int v) { return (v >= 0 && v < kNumVariants) ? variant_W(v) : -1; }
extern "C" int myersVariantIsMulti(int v) { return (v >= 0 && v < kNumVariants) ? (int)variant_multi(v) : -1; }

// Integer-ALU probe: returns 3-input logic ops executed per second by a
// device-filling launch (timed with CUDA events on the given stream).
extern "C" int myersProbeIntPeak(double* opsPerSecond, int iters) {
  if (opsPerSecond == nullptr || iters <= 0) return MYERS_E_INVALID_ARGUMENT;
  int dev = 0, sms = 0;
  CU(cudaGetDevice(&dev));
  CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int threads = 256, blocks = sms * 8;
  uint32_t* d_out = nullptr;
  CU(cudaMalloc((void**)&d_out, (size_t)blocks * threads * 4));
  cudaEvent_t a, b;
  CU(cudaEventCreate(&a));
  CU(cudaEventCreate(&b));
  CU(launch_lop3_probe(d_out, blocks, threads, 2, nullptr));  // warm-up
  CU(cudaEventRecord(a, nullptr));
  CU(launch_lop3_probe(d_out, blocks, threads, iters, nullptr));
  CU(cudaEventRecord(b, nullptr));
  CU(cudaEventSynchronize(b));
  float ms = 0.f;
  CU(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(d_out);
  const double ops = (double)blocks * threads * iters * 16.0 * 8.0;
  *opsPerSecond = ops / (ms * 1e-3);
  return MYERS_SUCCESS;
}

// ---------------------------------------------------------------------------
// drop-in buffers (the reference's buffer_t, src-api/myers-common.h:129-145)

static std::mutex g_budget_mu;
static uint64_t g_budget = 0;

extern "C" int myersSetMemoryBudget(uint64_t bytes) {
  std::lock_guard<std::mutex> lk(g_budget_mu);
  g_budget = bytes;
  return MYERS_SUCCESS;
}

static uint64_t budget_bytes(uint64_t freeb) {
  uint64_t b;
  {
    std::lock_guard<std::mutex> lk(g_budget_mu);
    b = g_budget;
  }
  if (b == 0) {
    const char* env = getenv("MYERS_MEMORY_BUDGET");
    b = env ? strtoull(env, nullptr, 10) : 0;
  }
  if (b == 0) b = 4ull << 30;
  const uint64_t cap = (uint64_t)(freeb * 0.8);
  return b < cap ? b : cap;
}

struct Shared {
  myersReference* ref;
  uint32_t refs;  // buffers still holding it
};

struct Buffer {
  uint32_t numBuffers;
  uint32_t idBuffer;
  uint32_t maxPEQEntries, maxCandidates, maxQueries;
  int device;
  cudaStream_t stream;
  Shared* shared;
  myersContext* ctx;
  qryEntry_t* h_peq;
  qryInfo_t* h_qinfo;
  candInfo_t* h_cands;
  resEntry_t* h_results;
  uint32_t* h_flags;
  qryEntry_t* d_peq;
  qryInfo_t* d_qinfo;
  candInfo_t* d_cands;
  resEntry_t* d_results;
  int window_mode;
  int path;
  float cutoff;  // < 0: off
  int use_graphs;
  cudaGraphExec_t exec;  // the last send, updated in place by the next
  int last_status;
  bool pending;
  std::vector<uint8_t> present;    // word counts of the last send
  std::vector<uint8_t> present_m;  // query lengths of the last send (cut-off only)
  PlanTable plan, plan2;
  bool plan_valid;
  int plan_path;
};

extern "C" qryEntry_t* getPEQBuffer(void* b) { return b ? static_cast<Buffer*>(b)->h_peq : nullptr; }
extern "C" candInfo_t* getCandidatesBuffer(void* b) { return b ? static_cast<Buffer*>(b)->h_cands : nullptr; }
extern "C" qryInfo_t* getPEQInfoBuffer(void* b) { return b ? static_cast<Buffer*>(b)->h_qinfo : nullptr; }
extern "C" resEntry_t* getResultsBuffer(void* b) { return b ? static_cast<Buffer*>(b)->h_results : nullptr; }
extern "C" uint32_t getMaxPEQEntries(void* b) { return b ? static_cast<Buffer*>(b)->maxPEQEntries : 0; }
extern "C" uint32_t getMaxCandidates(void* b) { return b ? static_cast<Buffer*>(b)->maxCandidates : 0; }
extern "C" uint32_t getMaxQueries(void* b) { return b ? static_cast<Buffer*>(b)->maxQueries : 0; }

static void buffer_free(Buffer* b) {
  if (b == nullptr) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  cudaFreeHost(b->h_peq);
  cudaFreeHost(b->h_qinfo);
  cudaFreeHost(b->h_cands);
  cudaFreeHost(b->h_results);
  cudaFreeHost(b->h_flags);
  cudaFree(b->d_peq);
  cudaFree(b->d_qinfo);
  cudaFree(b->d_cands);
  cudaFree(b->d_results);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->ctx) myersContextDestroy(b->ctx);
  if (b->stream) cudaStreamDestroy(b->stream);
  if (b->shared && --b->shared->refs == 0) {
    myersReferenceDestroy(b->shared->ref);
    delete b->shared;
  }
  delete b;
}

static int buffer_alloc(Buffer* b) {
#define ALLOC_H(p, n) \
  if (cudaHostAlloc((void**)&(p), (size_t)(n) ? (size_t)(n) : 1, cudaHostAllocDefault) != cudaSuccess) return MYERS_E_ALLOCATE_MEM
#define ALLOC_D(p, n) \
  if (cudaMalloc((void**)&(p), (size_t)(n) ? (size_t)(n) : 1) != cudaSuccess) return MYERS_E_INSUFFICIENT_MEM_GPU
  CU(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  ALLOC_H(b->h_peq, (size_t)b->maxPEQEntries * sizeof(qryEntry_t));
  ALLOC_H(b->h_qinfo, (size_t)b->maxQueries * sizeof(qryInfo_t));
  ALLOC_H(b->h_cands, (size_t)b->maxCandidates * sizeof(candInfo_t));
  ALLOC_H(b->h_results, (size_t)b->maxCandidates * sizeof(resEntry_t));
  ALLOC_H(b->h_flags, 4);
  ALLOC_D(b->d_peq, (size_t)b->maxPEQEntries * sizeof(qryEntry_t));
  ALLOC_D(b->d_qinfo, (size_t)b->maxQueries * sizeof(qryInfo_t));
  ALLOC_D(b->d_cands, (size_t)b->maxCandidates * sizeof(candInfo_t));
  ALLOC_D(b->d_results, (size_t)b->maxCandidates * sizeof(resEntry_t));
#undef ALLOC_H
#undef ALLOC_D
  return myersContextCreate(&b->ctx, b->maxCandidates);
}

extern "C" int myersInit(void*** myersBuffer, uint32_t numBuffers, const char* referenceFileName,
                         int32_t averageQuerySize, int32_t candidatesPerQuery) {
  if (myersBuffer == nullptr || numBuffers == 0 || referenceFileName == nullptr) return MYERS_E_INVALID_ARGUMENT;
  // defaults of src-api/myersGPU.c:300-301
  if (averageQuerySize <= 0) averageQuerySize = 1024;
  if (candidatesPerQuery <= 0) candidatesPerQuery = 1;
  myersReference* ref = nullptr;
  int st = myersReferenceLoad(&ref, referenceFileName);
  if (st != MYERS_SUCCESS) return st;
  Shared* shared = new Shared{ref, 0};
  size_t freeb = 0, totalb = 0;
  const cudaError_t me = cudaMemGetInfo(&freeb, &totalb);
  if (me != cudaSuccess) {
    myersReferenceDestroy(ref);
    delete shared;
    return cuda_fail(me, "cudaMemGetInfo");
  }
  // sizing as src-api/myersGPU.c:312-330, over the budget instead of free memory
  const uint32_t entries_per_query = (averageQuerySize + NUM_BASES_ENTRY - 1) / NUM_BASES_ENTRY;
  const double bytes_per_cand = (entries_per_query * sizeof(qryEntry_t) + sizeof(qryInfo_t)) / (double)candidatesPerQuery +
                                sizeof(candInfo_t) + sizeof(resEntry_t) + sizeof(uint32_t) + 1.0;
  const uint64_t per_buffer = budget_bytes(freeb) / numBuffers;
  uint64_t max_cands = (uint64_t)(per_buffer / bytes_per_cand);
  if (max_cands > 0x7FFFFFFFull) max_cands = 0x7FFFFFFFull;
  uint64_t max_queries = max_cands / (uint32_t)candidatesPerQuery;
  uint64_t max_entries = max_queries * entries_per_query;
  if (max_cands < 1 || max_queries < 1 || max_entries > 0xFFFFFFFFull) {
    myersReferenceDestroy(ref);
    delete shared;
    return MYERS_E_INSUFFICIENT_MEM_GPU;
  }
  Buffer** bufs = (Buffer**)calloc(numBuffers, sizeof(Buffer*));
  if (bufs == nullptr) {
    myersReferenceDestroy(ref);
    delete shared;
    return MYERS_E_ALLOCATE_MEM;
  }
  for (uint32_t i = 0; i < numBuffers; ++i) {
    Buffer* b = new Buffer();
    b->numBuffers = numBuffers;
    b->idBuffer = i;
    b->maxCandidates = (uint32_t)max_cands;
    b->maxQueries = (uint32_t)max_queries;
    b->maxPEQEntries = (uint32_t)max_entries;
    b->device = ref->device;
    b->shared = shared;
    shared->refs++;
    b->window_mode = MYERS_WINDOW_ALIGNED;
    b->path = MYERS_PATH_PLAIN;
    b->cutoff = -1.0f;
    const char* p = getenv("MYERS_PATH");
    if (p && strcmp(p, "batched") == 0) b->path = MYERS_PATH_BATCHED;
    const char* g = getenv("MYERS_GRAPHS");
    b->use_graphs = !(g && strcmp(g, "0") == 0);
    b->present.assign(kMaxWords + 1, 0);
    bufs[i] = b;
    st = buffer_alloc(b);
    if (st != MYERS_SUCCESS) {
      for (uint32_t j = 0; j <= i; ++j) buffer_free(bufs[j]);
      free(bufs);
      return st;
    }
  }
  *myersBuffer = (void**)bufs;
  return MYERS_SUCCESS;
}

extern "C" int initMyers(void*** myersBuffer, uint32_t numBuffers, const char* referenceFileName,
                         int32_t averageQuerySize, int32_t candidatesPerQuery) {
  fatal(myersInit(myersBuffer, numBuffers, referenceFileName, averageQuerySize, candidatesPerQuery), "initMyers");
  return 0;
}

extern "C" int myersSend(void* mb, float distance, uint32_t numPEQEntries, uint32_t numQueries,
                         uint32_t numCandidates) {
  Buffer* b = static_cast<Buffer*>(mb);
  if (b == nullptr) return MYERS_E_INVALID_ARGUMENT;
  b->last_status = MYERS_SUCCESS;
  if (!(distance >= 0.0f) || !std::isfinite(distance)) return b->last_status = MYERS_E_INVALID_ARGUMENT;
  if (numPEQEntries > b->maxPEQEntries || numQueries > b->maxQueries || numCandidates > b->maxCandidates)
    return b->last_status = MYERS_E_CAPACITY;
  NvtxRange range("myers: send");
  CU(cudaSetDevice(b->device));
  // O(queries) host pass: the word counts present pick the shapes
  std::vector<uint8_t>& present = b->present;
  std::fill(present.begin(), present.end(), 0);
  for (uint32_t q = 0; q < numQueries; ++q) {
    const uint32_t m = b->h_qinfo[q].size;
    if (m > 0 && m <= kMaxWords * 32) present[(m + 31) / 32] = 1;  // longer: flagged on the device
  }
  PlanTable& plan = b->plan;
  const bool two_pass = b->cutoff >= 0.0f;
  int st;
  {
    NvtxRange plan_range("myers: send: shape plan");
    if (two_pass) {
      std::vector<uint8_t>& pm = b->present_m;
      pm.assign(kMaxWords * 32 + 1, 0);
      for (uint32_t q = 0; q < numQueries; ++q) {
        const uint32_t m = b->h_qinfo[q].size;
        if (m > 0 && m <= kMaxWords * 32) pm[m] = 1;
      }
      st = cutoff_plans(plan, b->plan2, pm.data(), b->cutoff, cutoff_prefix_mult(), b->path == MYERS_PATH_BATCHED,
                        numCandidates);
    } else {
      st = build_plan(plan, present.data(), b->path == MYERS_PATH_BATCHED, 0, numCandidates, numQueries);
    }
  }
  if (st != MYERS_SUCCESS) return b->last_status = st;
  cudaStream_t s = b->stream;
  auto enqueue = [&]() -> int {
    CU(cudaMemsetAsync(b->ctx->d_flags, 0, 4, s));
    if (numCandidates == 0) {  // nothing to verify: only the flags travel back
      CU(cudaMemcpyAsync(b->h_flags, b->ctx->d_flags, 4, cudaMemcpyDeviceToHost, s));
      return MYERS_SUCCESS;
    }
    if (numPEQEntries)
      CU(cudaMemcpyAsync(b->d_peq, b->h_peq, (size_t)numPEQEntries * sizeof(qryEntry_t), cudaMemcpyHostToDevice, s));
    if (numQueries)
      CU(cudaMemcpyAsync(b->d_qinfo, b->h_qinfo, (size_t)numQueries * sizeof(qryInfo_t), cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(b->d_cands, b->h_cands, (size_t)numCandidates * sizeof(candInfo_t), cudaMemcpyHostToDevice,
                       s));
    DevInputs in;
    memset(&in, 0, sizeof(in));
    in.peq = reinterpret_cast<const uint32_t*>(b->d_peq);
    in.qinfo = reinterpret_cast<const uint2*>(b->d_qinfo);
    in.cands = reinterpret_cast<const Cand*>(b->d_cands);
    in.results = reinterpret_cast<uint2*>(b->d_results);
    in.num_cands = numCandidates;
    in.num_queries = numQueries;
    in.num_entries = numPEQEntries;
    in.distance = distance;
    in.exact = b->window_mode == MYERS_WINDOW_EXACT;
    in.cut = b->cutoff >= 0.0f;
    in.cutoff = in.cut ? b->cutoff : 0.0f;
    in.prefix_mult = cutoff_prefix_mult();
    const int est = verify_enqueue(b->ctx, b->shared->ref, in, plan, b->path, s, two_pass ? &b->plan2 : nullptr);
    if (est != MYERS_SUCCESS) return est;
    CU(cudaMemcpyAsync(b->h_results, b->d_results, (size_t)numCandidates * sizeof(resEntry_t),
                       cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(b->h_flags, b->ctx->d_flags, 4, cudaMemcpyDeviceToHost, s));
    return MYERS_SUCCESS;
  };
  st = b->use_graphs ? launch_as_graph(s, &b->exec, enqueue) : enqueue();
  if (st != MYERS_SUCCESS) return b->last_status = st;
  b->pending = true;
  return MYERS_SUCCESS;
}

extern "C" void sendMyersBuffer(void* mb, float distance, uint32_t numPEQEntries, uint32_t numQueries,
                                uint32_t numCandidates) {
  fatal(myersSend(mb, distance, numPEQEntries, numQueries, numCandidates), "sendMyersBuffer");
}

extern "C" int myersReceive(void* mb) {
  Buffer* b = static_cast<Buffer*>(mb);
  if (b == nullptr) return MYERS_E_INVALID_ARGUMENT;
  NvtxRange range("myers: receive (stream sync)");
  CU(cudaSetDevice(b->device));
  CU(cudaStreamSynchronize(b->stream));
  if (b->pending) {
    b->pending = false;
    if (*b->h_flags != 0) b->last_status = MYERS_E_QUERY_TOO_LONG;
  }
  return b->last_status;
}

extern "C" void receiveMyersBuffer(void* mb) { fatal(myersReceive(mb), "receiveMyersBuffer"); }

extern "C" int myersEnd(void*** myersBuffer) {
  if (myersBuffer == nullptr || *myersBuffer == nullptr) return MYERS_E_INVALID_ARGUMENT;
  Buffer** bufs = (Buffer**)(*myersBuffer);
  const uint32_t n = bufs[0]->numBuffers;
  for (uint32_t i = 0; i < n; ++i) buffer_free(bufs[i]);
  free(bufs);
  *myersBuffer = nullptr;
  return MYERS_SUCCESS;
}

extern "C" void endMyers(void*** myersBuffer) { fatal(myersEnd(myersBuffer), "endMyers"); }

extern "C" int myersSetWindowMode(void* mb, int mode) {
  Buffer* b = static_cast<Buffer*>(mb);
  if (b == nullptr || (mode != MYERS_WINDOW_ALIGNED && mode != MYERS_WINDOW_EXACT)) return MYERS_E_INVALID_ARGUMENT;
  b->window_mode = mode;
  return MYERS_SUCCESS;
}

extern "C" int myersSetKernelPath(void* mb, int path) {
  Buffer* b = static_cast<Buffer*>(mb);
  if (b == nullptr || (path != MYERS_PATH_PLAIN && path != MYERS_PATH_BATCHED)) return MYERS_E_INVALID_ARGUMENT;
  b->path = path;
  return MYERS_SUCCESS;
}

extern "C" int myersSetCutoff(void* mb, float cutoff) {
  Buffer* b = static_cast<Buffer*>(mb);
  if (b == nullptr || std::isnan(cutoff) || std::isinf(cutoff)) return MYERS_E_INVALID_ARGUMENT;
  if (cutoff >= 0.0f) {
    CU(cudaSetDevice(b->device));
    const int st = ensure_cutoff_scratch(b->ctx);
    if (st != MYERS_SUCCESS) return st;
  }
  b->cutoff = cutoff < 0.0f ? -1.0f : cutoff;
  return MYERS_SUCCESS;
}

extern "C" int myersSetGraphs(void* mb, int enable) {
  Buffer* b = static_cast<Buffer*>(mb);
  if (b == nullptr) return MYERS_E_INVALID_ARGUMENT;
  b->use_graphs = enable != 0;
  return MYERS_SUCCESS;
}

extern "C" int myersGetDevice(void* mb) { return mb ? static_cast<Buffer*>(mb)->device : -1; }
extern "C" int myersGetLastStatus(void* mb) { return mb ? static_cast<Buffer*>(mb)->last_status : MYERS_E_INVALID_ARGUMENT; }
extern "C" uint32_t myersBufferLastLaunches(void* mb) {
  return mb ? static_cast<Buffer*>(mb)->ctx->last_launches : 0;
}

// ---------------------------------------------------------------------------
// Verification that allocates nothing (no counterpart in the reference).
//
// Some callers cannot call cudaMalloc: programs whose own allocator owns all
// of device memory (a caching allocator, or a fixed arena handed out once,
// where an outside cudaMalloc fails or fragments it), and services whose
// memory budget is fixed after start-up. For them this entry point runs the
// batched path with its bucketing scratch (candidate ids sorted by shape, a
// shape byte per candidate, the bucket table and the error flags) in the
// file-scope device array below instead of a context's allocations. The
// array is sized for MYERS_NOALLOC_MAX_CANDIDATES candidates (about 1.3 MB)
// and every GPU that loads this library holds it until the process exits.

constexpr uint32_t kNoAllocMax = MYERS_NOALLOC_MAX_CANDIDATES;
constexpr size_t kNoAllocStateBytes = (sizeof(BucketState) + 255) & ~(size_t)255;
constexpr size_t kNoAllocIdsOffset = kNoAllocStateBytes;
constexpr size_t kNoAllocCfgOffset = kNoAllocIdsOffset + (size_t)kNoAllocMax * 4;
constexpr size_t kNoAllocFlagsOffset = kNoAllocCfgOffset + (((size_t)kNoAllocMax + 255) & ~(size_t)255);
constexpr size_t kNoAllocBytes = kNoAllocFlagsOffset + 256;

// Host code must not use this name as a device address: on the host it is a
// stand-in symbol. Its device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
struct NoAllocDevice {
  bool ready;
  unsigned long long context;  // id of the context the set-up ran in (0: unknown)
  unsigned char* scratch;      // device address of g_noalloc_scratch in that context
  int num_sms;
};
static std::mutex g_noalloc_mu;
static NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];

// Id of the current CUDA context, unique for the life of the process (0 if
// no context is current or the driver cannot tell). Driver entry points are
// looked up through the runtime, so the library needs no link to libcuda.
static unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", (void**)&get_current, 12000, cudaEnableDefault, &q) !=
            cudaSuccess || q != cudaDriverEntryPointSuccess)
      get_current = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", (void**)&get_id, 12000, cudaEnableDefault, &q) !=
            cudaSuccess || q != cudaDriverEntryPointSuccess)
      get_id = nullptr;
    cudaGetLastError();
  });
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (get_current == nullptr || get_id == nullptr || get_current(&c) != CUDA_SUCCESS || c == nullptr ||
      get_id(c, &id) != CUDA_SUCCESS)
    return 0;
  return id;
}

// Once per device, with that device current (and again when the device's
// context is not the one the set-up ran in, e.g. after cudaDeviceReset):
// resolve the array's device address and load every kernel this entry point
// can launch. Both may load code onto the device, so the first call should
// come before any stream capture.
static int noalloc_setup(NoAllocDevice* out) {
  int dev = 0;
  CU(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) return MYERS_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  NoAllocDevice& d = g_noalloc_dev[dev];
  const unsigned long long ctx = current_context_id();
  if (!d.ready || (ctx != 0 && ctx != d.context)) {
    d.ready = false;
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(noalloc scratch)");
    e = load_batched_path_kernels();
    if (e != cudaSuccess) return cuda_fail(e, "loading the batched path's kernels");
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute");
    d.scratch = static_cast<unsigned char*>(p);
    d.num_sms = sms;
    d.context = current_context_id();  // the set-up made the primary context current if none was
    d.ready = true;
  }
  *out = d;
  return MYERS_SUCCESS;
}

extern "C" int myersVerifyNoAllocAsync(const uint32_t* d_refWords, uint64_t refWords, uint64_t refSizeBases,
                                       const qryEntry_t* d_peq, uint32_t numPEQEntries,
                                       const qryInfo_t* d_qinfo, uint32_t numQueries,
                                       const candInfo_t* d_cands, uint32_t numCandidates, float distance,
                                       int windowMode, uint32_t minQuerySize, uint32_t maxQuerySize,
                                       resEntry_t* d_results, void* stream) {
  if (!(distance >= 0.0f) || !std::isfinite(distance)) return MYERS_E_INVALID_ARGUMENT;
  if (windowMode != MYERS_WINDOW_ALIGNED && windowMode != MYERS_WINDOW_EXACT) return MYERS_E_INVALID_ARGUMENT;
  if (refWords > UINT64_MAX / 8 || refSizeBases > refWords * 8) return MYERS_E_INVALID_ARGUMENT;
  if (numCandidates > kNoAllocMax) return MYERS_E_CAPACITY;  // beyond the static scratch
  if (numCandidates == 0) return MYERS_SUCCESS;
  if (d_refWords == nullptr || d_peq == nullptr || d_qinfo == nullptr || d_cands == nullptr || d_results == nullptr)
    return MYERS_E_INVALID_ARGUMENT;
  NoAllocDevice dev;
  int st = noalloc_setup(&dev);
  if (st != MYERS_SUCCESS) return st;
  PlanTable plan;
  st = plan_for_range(plan, minQuerySize, maxQuerySize, MYERS_PATH_BATCHED, numCandidates, numQueries);
  if (st != MYERS_SUCCESS) return st;
  BucketState* d_state = reinterpret_cast<BucketState*>(dev.scratch);
  uint32_t* d_ids = reinterpret_cast<uint32_t*>(dev.scratch + kNoAllocIdsOffset);
  uint8_t* d_cfg = dev.scratch + kNoAllocCfgOffset;
  uint32_t* d_flags = reinterpret_cast<uint32_t*>(dev.scratch + kNoAllocFlagsOffset);
  DevInputs in;
  memset(&in, 0, sizeof(in));
  in.peq = reinterpret_cast<const uint32_t*>(d_peq);
  in.qinfo = reinterpret_cast<const uint2*>(d_qinfo);
  in.cands = reinterpret_cast<const Cand*>(d_cands);
  in.ref = d_refWords;
  in.ref_size = refSizeBases;
  in.ref_words = refWords;
  in.results = reinterpret_cast<uint2*>(d_results);
  in.flags = d_flags;
  in.num_cands = numCandidates;
  in.num_queries = numQueries;
  in.num_entries = numPEQEntries;
  in.distance = distance;
  in.exact = windowMode == MYERS_WINDOW_EXACT;
  set_multipliers(in);
  cudaStream_t s = (cudaStream_t)stream;
  // the array keeps the previous call's contents: the bucket table (counts,
  // cursors, work queue) and the flags must start at zero
  CU(cudaMemsetAsync(d_state, 0, sizeof(BucketState), s));
  CU(cudaMemsetAsync(d_flags, 0, sizeof(uint32_t), s));
  cudaError_t e = cudaSuccess;
  launch_bucketing(in, plan, d_state, d_cfg, d_ids, s, dev.num_sms, &e);
  if (e != cudaSuccess) return cuda_fail(e, "bucketing");
  if (plan.num_batched > 0)
    CU(launch_batched(in, d_ids, plan, d_state, s, dev.num_sms, batched_tile_bound(plan, numCandidates)));
  for (uint32_t c = plan.num_batched; c < plan.num_cfg; ++c)
    CU(launch_plain(plan.shape[c].variant, plan.shape[c].L, in, d_ids, d_state, (int)c, 0, 0, &d_state->next[c], s,
                    dev.num_sms));
  return MYERS_SUCCESS;
}
