/*
 * myers-interface.h - C ABI of the B200 Myers candidate-verification library
 * (libmyers_b200.so).
 *
 * The first part is a drop-in for the reference's public header
 * (src-api/myers-interface.h:1-46 in achacond/myers-gpu): same types with the
 * same layouts, same buffer getters and the same four main calls, with the
 * same fatal error convention (print, then exit(EXIT_FAILURE)).
 *
 * The second part adds what the reference lacks: status-returning variants
 * of the main calls, options (window mode, kernel path, memory budget), a
 * stream-ordered entry point on device-resident inputs, and a serving loop.
 *
 * All entry points take plain pointers and sizes; there are no C++ or torch
 * types in any signature.
 */
#ifndef MYERS_INTERFACE_H
#define MYERS_INTERFACE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NUM_BITS         4
#define NUM_BASES        5
#define NUM_BASES_ENTRY  128
#define SIZE_GPU_HW_WORD 32
#define NUM_SUB_ENTRIES  (NUM_BASES_ENTRY / SIZE_GPU_HW_WORD)

/* PEQ entry: 128 query bases. Bit i of bitmap[c][w] is set iff query base
 * 32*w+i of this entry has code c (A0 C1 G2 T3 N4). Replaces the reference's
 * qryEntry_t, src-api/myers-interface.h:10-12 (80 bytes). */
typedef struct {
    uint32_t bitmap[NUM_BASES][NUM_SUB_ENTRIES];
} qryEntry_t;

/* Result of one candidate: end column of the first minimum and its edit
 * distance. Replaces resEntry_t, src-api/myers-interface.h:14-17. */
typedef struct {
    uint32_t column;
    uint32_t score;
} resEntry_t;

/* Candidate: query index and reference base position (16 bytes with the
 * compiler's padding). Replaces candInfo_t, src-api/myers-interface.h:19-22. */
typedef struct {
    uint32_t query;
    uint64_t position;
} candInfo_t;

/* Query: first PEQ entry and length in bases. Replaces qryInfo_t,
 * src-api/myers-interface.h:24-27. */
typedef struct {
    uint32_t posEntry;
    uint32_t size;
} qryInfo_t;

/* ---------------------------------------------------------------------------
 * Drop-in API (reference: src-api/myers-interface.h:30-46, src-api/myersGPU.c)
 * ------------------------------------------------------------------------- */

/* Library-owned pinned host buffers of one Myers buffer; the caller fills
 * them in place between calls. Replaces the getters at
 * src-api/myers-interface.h:31-34 (src-api/myersGPU.c:70-88). The reference
 * declares them `inline`; here they are ordinary exported functions so that
 * both C89-inline and C99 callers link. */
qryEntry_t *getPEQBuffer(void *myersBuffer);
candInfo_t *getCandidatesBuffer(void *myersBuffer);
qryInfo_t  *getPEQInfoBuffer(void *myersBuffer);
resEntry_t *getResultsBuffer(void *myersBuffer);

/* Capacities of one buffer. Replace src-api/myers-interface.h:37-39
 * (src-api/myersGPU.c:55-68). */
uint32_t getMaxPEQEntries(void *myersBuffer);
uint32_t getMaxCandidates(void *myersBuffer);
uint32_t getMaxQueries(void *myersBuffer);

/* Load the packed reference (`u32 numEntries, u32 size, u32 words[]`) once
 * into device memory and create `numBuffers` buffers, each with its own
 * stream on the current device, sized from the memory budget (see
 * myersSetMemoryBudget). Returns 0. Replaces src-api/myers-interface.h:42
 * (defined at src-api/myersGPU.c:284-344). */
int initMyers(void ***myersBuffer, uint32_t numBuffers, const char *referenceFileName,
              int32_t averageQuerySize, int32_t candidatesPerQuery);

/* Enqueue the verification of the buffer's first numCandidates candidates on
 * the buffer's stream and return; the buffer must not be touched until
 * receiveMyersBuffer. `distance` is the error fraction: the window of a
 * query of m bases spans (uint32_t)(m*(1+2*distance)) bases. Replaces
 * src-api/myers-interface.h:44 (src-api/myersGPU.c:466-494). */
void sendMyersBuffer(void *myersBuffer, float distance, uint32_t numPEQEntries,
                     uint32_t numQueries, uint32_t numCandidates);

/* Wait for the buffer; afterwards getResultsBuffer()[i] holds candidate i's
 * result in caller order. Replaces src-api/myers-interface.h:45
 * (src-api/myersGPU.c:515-524). */
void receiveMyersBuffer(void *myersBuffer);

/* Release every buffer, the streams and the device reference. Replaces
 * src-api/myers-interface.h:46 (src-api/myersGPU.c:651-676). */
void endMyers(void ***myersBuffer);

/* ---------------------------------------------------------------------------
 * Extensions (no counterpart in the reference unless stated)
 * ------------------------------------------------------------------------- */

/* Error codes. The first six keep the values of the reference's
 * myersError_t (src-api/myers-common.h:13-24). */
typedef enum {
    MYERS_SUCCESS = 0,
    MYERS_E_OPENING_FILE = 1,
    MYERS_E_READING_FILE = 2,
    MYERS_E_INSUFFICIENT_MEM_GPU = 3,
    MYERS_E_ALLOCATE_MEM = 4,
    MYERS_E_INCOMPATIBLE_GPU = 5,
    MYERS_E_INVALID_ARGUMENT = 6,
    MYERS_E_CAPACITY = 7,        /* more entries/queries/candidates than the buffer holds */
    MYERS_E_QUERY_TOO_LONG = 8,  /* a query longer than MYERS_MAX_QUERY_BASES */
    MYERS_E_CUDA = 9,            /* a CUDA runtime call failed */
    MYERS_E_TIMEOUT = 10,        /* a bounded device-side wait gave up */
    MYERS_E_NOT_READY = 11,      /* serving: request not finished yet */
    MYERS_E_BUSY = 12            /* serving: admission refused (queue or budget full) */
} myersStatus_t;

/* Longest query (bases) the kernels verify: 32 lanes x 32 words x 32 bits. */
#define MYERS_MAX_QUERY_BASES 32768u
/* Longest window (columns) a result column can address. */
#define MYERS_MAX_WINDOW_COLUMNS 65535u

const char *myersGetErrorString(int status);

/* Window semantics.
 *  ALIGNED (default, the API's): the text starts at the packed word holding
 *    the candidate position and spans 8*E columns, E = W/8 + (W%8 ? 2 : 1);
 *    columns are counted from that word (src-api/coreMyersGPU-CC50.cu:131-166).
 *  EXACT: the text starts at the position and spans W columns; columns are
 *    counted from the position (src/myers-4bits.c:75-153). */
enum { MYERS_WINDOW_ALIGNED = 0, MYERS_WINDOW_EXACT = 1 };

/* Kernel path.
 *  PLAIN: one launch per length bucket present (the fixed-length kernel;
 *    a single launch when all queries share one bucket).
 *  BATCHED: one persistent launch pulling length-bucketed work tiles from a
 *    device queue.
 * A buffer's send (copies in, kernels, copies out) is captured and replayed
 * as one CUDA graph, updated in place from send to send (myersSetGraphs). */
enum { MYERS_PATH_PLAIN = 0, MYERS_PATH_BATCHED = 1 };

/* Status-returning versions of the main calls: same behaviour, but errors
 * are returned instead of ending the process. */
int myersInit(void ***myersBuffer, uint32_t numBuffers, const char *referenceFileName,
              int32_t averageQuerySize, int32_t candidatesPerQuery);
int myersSend(void *myersBuffer, float distance, uint32_t numPEQEntries,
              uint32_t numQueries, uint32_t numCandidates);
int myersReceive(void *myersBuffer);
int myersEnd(void ***myersBuffer);

/* Per-buffer options; take effect at the next send. */
int myersSetWindowMode(void *myersBuffer, int mode);
int myersSetKernelPath(void *myersBuffer, int path);
/* Non-zero (default): replay each send as a CUDA graph; 0: plain stream
 * launches. The environment variable MYERS_GRAPHS=0 sets the default to 0. */
int myersSetGraphs(void *myersBuffer, int enable);
/* Ukkonen's cut-off for the buffer's sends (see myersVerifyCutoffAsync):
 * cutoff >= 0 reports a candidate whose minimum exceeds (uint32_t)(m *
 * cutoff) as {MYERS_NO_MATCH, MYERS_NO_MATCH}; cutoff < 0 (default) turns it
 * off. Replaces gt_map_block_bpm_get_distance__cutoff
 * (GEMTools/src/gt_map_align_bpm.c:141-210) for a verifier whose caller
 * drops candidates above an error bound anyway. */
int myersSetCutoff(void *myersBuffer, float cutoff);

/* Device memory budget (bytes) for all buffers created by the next
 * initMyers/myersInit, replacing the reference's "95% of free memory"
 * (src-api/myersGPU.c:323-333). 0 restores the default (the environment
 * variable MYERS_MEMORY_BUDGET if set, else 4 GiB, capped at 80% of free). */
int myersSetMemoryBudget(uint64_t bytes);

/* Device of the library's streams (default: the current device at init). */
int myersGetDevice(void *myersBuffer);

/* Status of the last send/receive of a buffer (sticky until the next send). */
int myersGetLastStatus(void *myersBuffer);

/* ---------------------------------------------------------------------------
 * Stream-ordered verification on device-resident inputs
 * ------------------------------------------------------------------------- */

/* Opaque handle of a packed reference resident in device memory. */
typedef struct myersReference myersReference_t;

/* Upload `numWords` packed words (the body of a .4bits.ref file) describing
 * `sizeBases` bases; the library appends N padding. */
int myersReferenceCreate(myersReference_t **ref, const uint32_t *hostWords, uint64_t numWords,
                         uint64_t sizeBases);
/* Load a .4bits.ref file (src-api/genReference-4bits.c:121-140 format). */
int myersReferenceLoad(myersReference_t **ref, const char *fileName);
int myersReferenceDestroy(myersReference_t *ref);
uint64_t myersReferenceSize(const myersReference_t *ref);

/* Opaque per-stream work context: device scratch for length bucketing and
 * the work queue, sized for up to maxCandidates candidates, and four streams
 * the plain path runs its per-shape launches on (forked from the caller's
 * stream and joined back to it; MYERS_PLAIN_STREAMS=1 keeps them on the
 * caller's stream). */
typedef struct myersContext myersContext_t;
int myersContextCreate(myersContext_t **ctx, uint64_t maxCandidates);
int myersContextDestroy(myersContext_t *ctx);

/* Verify numCandidates candidates on `stream` (a cudaStream_t; NULL is the
 * legacy default stream). All pointers are device pointers: d_peq
 * (numPEQEntries qryEntry_t), d_qinfo (numQueries qryInfo_t), d_cands
 * (numCandidates candInfo_t) and d_results (numCandidates resEntry_t).
 * Candidates whose window does not fit the reference get {0, 0xFFFFFFFF}.
 * Asynchronous: returns after enqueueing. */
int myersVerifyAsync(myersContext_t *ctx, const myersReference_t *ref,
                     const qryEntry_t *d_peq, uint32_t numPEQEntries,
                     const qryInfo_t *d_qinfo, uint32_t numQueries,
                     const candInfo_t *d_cands, uint32_t numCandidates,
                     float distance, int windowMode, int path,
                     resEntry_t *d_results, void *stream);

/* As myersVerifyAsync, with the range of query lengths the batch holds
 * (bases; 0,0 = any). The kernels' shapes are chosen per length bucket; a
 * narrow range lets the plain path launch only the buckets that can occur
 * (a single launch, without bucketing, when the range is one bucket).
 * Queries outside the range get {0, 0xFFFFFFFF} and raise a context flag. */
int myersVerifyRangeAsync(myersContext_t *ctx, const myersReference_t *ref,
                          const qryEntry_t *d_peq, uint32_t numPEQEntries,
                          const qryInfo_t *d_qinfo, uint32_t numQueries,
                          const candInfo_t *d_cands, uint32_t numCandidates,
                          float distance, int windowMode, int path,
                          uint32_t minQuerySize, uint32_t maxQuerySize,
                          resEntry_t *d_results, void *stream);

/* Column and score of a candidate whose minimum exceeds the cut-off bound. */
#define MYERS_NO_MATCH 0xFFFFFFFFu

/* As myersVerifyRangeAsync, under Ukkonen's cut-off with the bound
 * k = (uint32_t)(m * cutoff) (float32) for a query of m bases. The analogue of
 * GEMTools' gt_map_block_bpm_get_distance__cutoff
 * (GEMTools/src/gt_map_align_bpm.c:141-210), which returns the distance and
 * position only when the minimum is within its max_distance:
 *  - a candidate whose minimum score is <= k gets exactly the result of
 *    myersVerifyRangeAsync (score, first column of that score);
 *  - a candidate whose minimum exceeds k gets {MYERS_NO_MATCH, MYERS_NO_MATCH};
 *  - candidates that are not verified (window out of range, invalid indices,
 *    unsupported sizes) get {0, 0xFFFFFFFF} as without the cut-off.
 * The work is cut in two passes: the first runs every
 * candidate's DP over a prefix of its query of about 2.25k rows (the environment
 * variable MYERS_CUTOFF_PREFIX sets the multiplier), which settles every
 * candidate whose prefix minimum exceeds k (every path to the last row
 * crosses the prefix's last row); the second runs the full DP of the rest.
 * The first call on a context allocates the second pass's scratch (5 bytes
 * per candidate of its capacity). On the batched path the two passes are two
 * persistent launches. */
int myersVerifyCutoffAsync(myersContext_t *ctx, const myersReference_t *ref,
                           const qryEntry_t *d_peq, uint32_t numPEQEntries,
                           const qryInfo_t *d_qinfo, uint32_t numQueries,
                           const candInfo_t *d_cands, uint32_t numCandidates,
                           float distance, int windowMode, int path, float cutoff,
                           uint32_t minQuerySize, uint32_t maxQuerySize,
                           resEntry_t *d_results, void *stream);

/* Largest batch myersVerifyNoAllocAsync accepts (candidates). */
#define MYERS_NOALLOC_MAX_CANDIDATES 262144u

/* Verification that allocates nothing. No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: programs whose own allocator owns
 * all of device memory (a caching allocator, or an arena carved out at
 * start-up, where an outside cudaMalloc fails or fragments the pool), and
 * services whose memory budget is fixed once they are up. Inputs and outputs
 * are the caller's device memory, as for myersVerifyRangeAsync, and the
 * reference is passed as raw device words (refWords readable words holding
 * refSizeBases bases; reads past them act as N). It runs the batched path;
 * its scratch lives in a device array inside this library, about 1.3 MB,
 * that every GPU which loads the library holds until the process exits.
 *
 *  - at most MYERS_NOALLOC_MAX_CANDIDATES candidates per call; larger batches
 *    return MYERS_E_CAPACITY and enqueue nothing;
 *  - the first call on a device (and again after that device's context was
 *    reset) does the set-up, with that device current: it looks up the
 *    array's device address and loads every kernel this entry point can
 *    launch, so later calls load no code; make that first call before any
 *    stream capture;
 *  - every call on a device shares the one array and leaves its contents
 *    behind (each call clears what must start at zero): calls that overlap on
 *    the GPU (other streams, or other threads) race and give wrong results;
 *    serialise them, e.g. on one stream;
 *  - error flags are not reported: flagged candidates get {0, 0xFFFFFFFF}.
 * Asynchronous on `stream` (a cudaStream_t). */
int myersVerifyNoAllocAsync(const uint32_t *d_refWords, uint64_t refWords, uint64_t refSizeBases,
                            const qryEntry_t *d_peq, uint32_t numPEQEntries,
                            const qryInfo_t *d_qinfo, uint32_t numQueries,
                            const candInfo_t *d_cands, uint32_t numCandidates,
                            float distance, int windowMode,
                            uint32_t minQuerySize, uint32_t maxQuerySize,
                            resEntry_t *d_results, void *stream);

/* Build PEQ entries from ASCII reads on the device (the packing of
 * src-api/genCandidate-reorder.c:258-317): read r is
 * d_ascii[d_offsets[r] .. d_offsets[r] + d_qinfo[r].size) (A/C/G/T either
 * case, anything else N); its ceil(size/128) entries are written at
 * d_peq + d_qinfo[r].posEntry. d_ascii holds asciiBytes bytes, d_offsets
 * numReads + 1 entries; reads whose bytes or entries fall outside the
 * buffers are skipped and raise context flag 4. */
int myersPackPEQAsync(myersContext_t *ctx, const uint8_t *d_ascii, uint64_t asciiBytes,
                      const uint64_t *d_offsets, const qryInfo_t *d_qinfo, uint32_t numReads,
                      qryEntry_t *d_peq, uint32_t numPEQEntries, void *stream);

/* Pack ASCII bases into reference words on the device (the packing of
 * src-api/genReference-4bits.c:43-72): numWords words, 8 bases each, base i
 * in bits 4*(i%8) of word i/8; bases at or past numBases are N. */
int myersPackReferenceAsync(const uint8_t *d_ascii, uint64_t numBases, uint32_t *d_words,
                            uint64_t numWords, void *stream);

/* Kernel launches the last myersVerify*Async on this context enqueued. */
uint32_t myersContextLastLaunches(const myersContext_t *ctx);

/* Device error flags raised since the last clear (synchronous read):
 * 1 query too long / window too wide, 2 candidate query index out of range,
 * 4 query PEQ entries out of range. */
int myersContextFlags(myersContext_t *ctx, uint32_t *flags, int clear);

/* Kernel launches of a buffer's last send. */
uint32_t myersBufferLastLaunches(void *myersBuffer);

/* ---------------------------------------------------------------------------
 * Traceback of accepted candidates (no counterpart in the reference, which
 * returns only the end column and the distance).
 *
 * For a candidate whose result (column c, score s) has s <= maxScore, the
 * alignment is the path through the semi-global edit-distance matrix of its
 * window (D[0][j] = 0, D[i][0] = i, unit costs; a query base matches a text
 * base as in the verification, so N matches N) from (m, c+1) back to row 0
 * that takes, at each cell, the first consistent step of: the diagonal
 * ('=' or 'X'), the query base alone ('I'), the text base alone ('D').
 * ------------------------------------------------------------------------- */

/* Per candidate: the first window column the alignment consumes (c + 1 when
 * it consumes none), the number of run-length ops, and the result's score
 * and end column. numOps is MYERS_TB_NOT_TRACED for candidates above
 * maxScore or without a result, MYERS_TB_INCONSISTENT when the result does
 * not follow from the inputs (or a candidate's indices are out of range),
 * and a count above maxOpsPerCandidate when the ops did not fit (the ops
 * are then unspecified; trace again with more room). */
typedef struct {
    uint32_t startColumn;
    uint32_t numOps;
    uint32_t score;
    uint32_t endColumn;
} myersAlignment_t;

#define MYERS_TB_NOT_TRACED 0xFFFFFFFFu
#define MYERS_TB_INCONSISTENT 0xFFFFFFFEu
/* ops[k] = length << 4 | code, first op first; codes as SAM's BAM encoding */
#define MYERS_CIGAR_INS 1u
#define MYERS_CIGAR_DEL 2u
#define MYERS_CIGAR_EQ 7u
#define MYERS_CIGAR_X 8u

/* Work space of the traceback: ids of up to maxCandidates candidates and
 * scratchBytes (>= 1 MiB) of device memory for the stored bit-vectors of the
 * traced candidates. Passes alternate between the two halves of the scratch
 * (one pass's walk overlaps the next pass's recomputation), so half of it
 * must hold the band of the widest traced candidate, else myersTraceback
 * returns MYERS_E_CAPACITY: a read of 1000 bases needs about 90 KB at score
 * 60 and about 900 KB at score 600. Calls on one traceback object must be
 * ordered (one stream, or synchronised). */
typedef struct myersTraceback myersTraceback_t;
int myersTracebackCreate(myersTraceback_t **tb, uint64_t maxCandidates, uint64_t scratchBytes);
int myersTracebackDestroy(myersTraceback_t *tb);

/* Trace the candidates of a verified batch. Inputs as myersVerifyAsync plus
 * the batch's results (d_results, device) from the same distance and window
 * mode; outputs: d_ops (numCandidates * maxOpsPerCandidate u32; candidate
 * k's ops at k * maxOpsPerCandidate) and d_alignments (numCandidates).
 * Enqueued on `stream`; synchronises the stream once, after selecting the
 * candidates to trace, to size the passes over the scratch. Not for use
 * during stream capture. */
int myersTraceback(myersTraceback_t *tb, const myersReference_t *ref,
                   const qryEntry_t *d_peq, uint32_t numPEQEntries,
                   const qryInfo_t *d_qinfo, uint32_t numQueries,
                   const candInfo_t *d_cands, const resEntry_t *d_results, uint32_t numCandidates,
                   float distance, int windowMode, uint32_t maxScore,
                   uint32_t *d_ops, uint32_t maxOpsPerCandidate, myersAlignment_t *d_alignments,
                   void *stream);

/* Candidates traced by the last myersTraceback, and the passes it made. */
uint32_t myersTracebackLastCount(const myersTraceback_t *tb);
uint32_t myersTracebackLastChunks(const myersTraceback_t *tb);

/* ---------------------------------------------------------------------------
 * Serving loop (no counterpart in the reference): requests -- one read and
 * its candidate positions -- are admitted under a device-memory budget and
 * verified in batches that form continuously: while some batches are on the
 * GPU, requests that arrive are gathered into the next batch, which starts as
 * soon as a batch slot frees up. Each slot has its own stream, so copies and
 * kernels of consecutive batches overlap on the device. The reference stays
 * resident.
 * ------------------------------------------------------------------------- */

typedef struct myersServer myersServer_t;

typedef struct {
    uint64_t budgetBytes;        /* device memory of all batch slots (0: 16 GiB, capped at 80% of free) */
    uint32_t slots;              /* batches in flight (0: 4) */
    uint32_t maxBatchCandidates; /* per batch slot (0: 1<<20, lowered to fit the budget) */
    uint32_t maxQueued;          /* requests waiting for a slot before submit refuses (0: 1<<20) */
    float distance;              /* error fraction, as sendMyersBuffer */
    int windowMode;              /* MYERS_WINDOW_* */
    int path;                    /* MYERS_PATH_* (default batched) */
    uint32_t maxQuerySize;       /* longest read accepted (0: 1024 bases) */
    uint32_t laneWords;          /* 0: shapes by batch size, as myersVerifyAsync picks them on the
                                    batched path (batches under 280K candidates run reads of up to
                                    1,024 bases on lanes of at most 12 words); k > 0: spread a read
                                    of more than k 32-bit words over several lanes of at most k
                                    words each (the cheapest such shape), which cuts its time on
                                    the GPU (latency) for some more work */
    int useGraphs;               /* non-zero: capture each batch's copies and kernels and replay them
                                    as a CUDA graph (updated in place batch to batch) */
} myersServerConfig_t;

typedef struct {
    uint64_t submitted, refused, completed, batches;
    uint64_t batchCandidatesMax;  /* largest batch dispatched */
    uint64_t candidatesCompleted;
    uint32_t slots, maxBatchCandidates, maxBatchQueries, maxBatchEntries;
} myersServerStats_t;

int myersServerCreate(myersServer_t **srv, const myersReference_t *ref, const myersServerConfig_t *cfg);

/* Queue one request: `peq` holds the read's ceil(querySize/128) PEQ entries,
 * `positions` its numCandidates reference positions. Copies both. Returns
 * MYERS_E_BUSY when maxQueued requests already wait, MYERS_E_CAPACITY when
 * the request alone exceeds a batch slot. */
int myersServerSubmit(myersServer_t *srv, const qryEntry_t *peq, uint32_t querySize,
                      const uint64_t *positions, uint32_t numCandidates, uint64_t *ticket);

/* MYERS_E_NOT_READY until the request is done; then copies its numCandidates
 * results (candidate order) into `results` and forgets the ticket. */
int myersServerPoll(myersServer_t *srv, uint64_t ticket, resEntry_t *results);

/* Block until the request is done (or timeoutMs passes: MYERS_E_TIMEOUT). */
int myersServerWait(myersServer_t *srv, uint64_t ticket, resEntry_t *results, uint32_t timeoutMs);

int myersServerStats(myersServer_t *srv, myersServerStats_t *stats);

/* Stop accepting, finish what is in flight, free everything. */
int myersServerDestroy(myersServer_t *srv);

/* Open-loop load for measurement: request i (read qinfo[i], PEQ entries from
 * qinfo[i].posEntry, candidates positions[candOffset[i] .. candOffset[i+1]))
 * is submitted at arrivalNs[i] after the start by a driver thread, whatever
 * the server's state. latencyNs[i] = completion - scheduled arrival
 * (UINT64_MAX if refused); results receive every candidate's result in
 * request order. *wallNs = first arrival to last completion. */
int myersServerReplay(myersServer_t *srv, const qryEntry_t *peq, const qryInfo_t *qinfo,
                      const uint32_t *candOffset, const uint64_t *positions, uint32_t numRequests,
                      const uint64_t *arrivalNs, uint64_t *latencyNs, resEntry_t *results,
                      uint64_t *wallNs);

/* ---------------------------------------------------------------------------
 * Kernel shapes (autotuning)
 * ------------------------------------------------------------------------- */

/* Kernel variants: 0..31 one candidate per lane with W = variant+1 words;
 * 32.. a candidate spread over L lanes of W words. */
int myersNumVariants(void);
int myersVariantWords(int variant);
int myersVariantIsMulti(int variant);

/* Shape the given path uses for a query length. */
int myersShapeOf(int path, uint32_t querySize, int *variant, int *L, int *W);

/* Force the shape used for queries of `words` 32-bit words
 * (ceil(size/32)); variant -1 restores the built-in choice. */
int myersSetShapeOverride(int path, uint32_t words, int variant, int L);

/* Shapes come, in this order, from myersSetShapeOverride, the serving loop's
 * latency policy (laneWords), the autotuner's cache -- autotune_b200.json next
 * to the library, written by myers-gpu_b200/autotune.py (MYERS_AUTOTUNE names
 * another file, MYERS_AUTOTUNE=0 ignores it) -- and a built-in cost model.
 * Returns how many word counts the loaded cache covers for the path. */
int myersTunedShapes(int path);

/* Integer-ALU throughput probe on the current device: 3-input logic ops per
 * second of a device-filling launch (the roofline denominator). */
int myersProbeIntPeak(double *opsPerSecond, int iters);

#ifdef __cplusplus
}
#endif

#endif /* MYERS_INTERFACE_H */
