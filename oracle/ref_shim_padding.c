/*
 * Test infrastructure only. Wraps the reference's own CPU Myers
 * (src-integration/myers-reorderBuffer-padding.c, the aligned-window API
 * semantics) into a shared library so the tests and the CPU-baseline leg of
 * the benchmark can call it on in-memory inputs.
 *
 * The reference source is compiled from where it lies: the Makefile passes
 * its path as REF_SOURCE and writes the library into oracle/_ref/ only.
 * Nothing of the reference is copied into this repository.
 */
#define main ref_padding_main
#include REF_SOURCE
#undef main

#include <omp.h>

/*
 * Runs the reference's computeAllQueriesCPU (myers-reorderBuffer-padding.c
 * :178-208) inside an OpenMP parallel region, exactly as its main() does
 * (:490-493), on caller-provided buffers.
 *
 *   peq      API PEQ entries (qryEntry_t, 80 B each)
 *   qinfo    qryInfo_t per query
 *   cands16  API candInfo_t (16 B: u32 query, 4 B padding, u64 position);
 *            converted here to the oracle's 8-byte layout (u32 position)
 *   ref      packed reference words; the caller pads the array so the window
 *            reads past the last word stay inside it
 *   res      receives {column, score}; pre-filled with {0, 0xFFFFFFFF}
 *            like the reference's initResults (:290-294)
 *   uncapped if non-zero, candidates whose query exceeds the driver's
 *            4096-base cap (:200) are computed by calling computeMyers
 *            directly with the same per-candidate sizing (:192-198)
 *   seconds  wall time of the computeAllQueriesCPU region plus, with
 *            `uncapped`, the direct computeMyers calls after it
 *
 * Returns 0, or -1 if a position does not fit the oracle's 32-bit field.
 */
int refshim_verify_aligned(qryEntry_t *peq, uint32_t num_entries,
                           qryInfo_t *qinfo, uint32_t num_queries,
                           const void *cands16, uint32_t num_cands,
                           uint32_t *ref, uint32_t ref_words, uint32_t ref_size,
                           float distance, resEntry_t *res, int nthreads,
                           int uncapped, double *seconds)
{
    const uint8_t *src = (const uint8_t *)cands16;
    candInfo_t *c8 = (candInfo_t *)malloc(sizeof(candInfo_t) * (num_cands ? num_cands : 1));
    if (c8 == NULL) return -2;
    for (uint32_t i = 0; i < num_cands; ++i) {
        uint32_t q;
        uint64_t pos;
        memcpy(&q, src + 16 * (size_t)i, 4);
        memcpy(&pos, src + 16 * (size_t)i + 8, 8);
        if (pos > 0xFFFFFFFFull) { free(c8); return -1; }
        c8[i].query = q;
        c8[i].position = (uint32_t)pos;
    }
    for (uint32_t i = 0; i < num_cands; ++i) { res[i].column = 0; res[i].score = MAX_VALUE; }

    ref_t r;
    memset(&r, 0, sizeof(r));
    r.size = ref_size;
    r.numEntries = ref_words;
    r.h_reference = ref;

    qry_t q;
    memset(&q, 0, sizeof(q));
    q.totalQueriesEntries = num_entries;
    q.numQueries = num_queries;
    q.numCandidates = num_cands;
    q.distance = distance;
    q.h_queries = peq;
    q.h_candidates = c8;
    q.h_qinfo = qinfo;

    res_t rs;
    memset(&rs, 0, sizeof(rs));
    rs.numResults = num_cands;
    rs.h_results = res;

    if (nthreads <= 0) nthreads = omp_get_max_threads();
    double t0 = omp_get_wtime();
#pragma omp parallel num_threads(nthreads)
    {
        computeAllQueriesCPU(&r, &q, &rs);
    }
    if (uncapped) {
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
        for (int64_t i = 0; i < (int64_t)num_cands; ++i) {
            uint32_t initEntry = qinfo[c8[i].query].posEntry;
            uint32_t sizeQuery = qinfo[c8[i].query].size;
            if (sizeQuery <= 4096) continue;
            uint32_t positionRef = c8[i].position;
            uint32_t sizeCandidate = sizeQuery * (1 + 2 * distance);
            uint32_t numEntriesPerQuery = (sizeQuery / SIZE_HW_WORD) + ((sizeQuery % SIZE_HW_WORD) ? 1 : 0);
            uint32_t numLargeEntriesPerQuery = (sizeQuery / NUM_BASES_ENTRY) + ((sizeQuery % NUM_BASES_ENTRY) ? 1 : 0);
            uint32_t numEntriesPerCandidate = (sizeCandidate / BASES_PER_ENTRY) + ((sizeCandidate % BASES_PER_ENTRY) ? 2 : 1);
            computeMyers(peq, ref, res, (uint32_t)i, sizeCandidate, sizeQuery, ref_size,
                         numEntriesPerQuery, numLargeEntriesPerQuery, positionRef, initEntry,
                         numEntriesPerCandidate);
        }
    }
    double t1 = omp_get_wtime();
    if (seconds) *seconds = t1 - t0;
    free(c8);
    return 0;
}
