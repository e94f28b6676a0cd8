/*
 * Test infrastructure only. Wraps the reference's exact-window CPU Myers
 * (src/myers-4bits.c) into a shared library. The reference source is
 * compiled from where it lies (REF_SOURCE, set by the Makefile); the output
 * goes to oracle/_ref/ only.
 */
#define main ref_exact_main
#include REF_SOURCE
#undef main

#include <omp.h>

/*
 * Runs the reference's computeAllQueriesCPU (src/myers-4bits.c:155-175) in
 * an OpenMP parallel region, as its main() does. That oracle handles one
 * fixed query length with 32-base PEQ entries laid out query-major
 * (initEntry = query * numEntriesPerQuery, :94); the API's 128-base entries
 * are re-laid into that form here. All queries must share one length.
 *
 *   peq128   API PEQ entries, 20 u32 each: bitmap[5][4]
 *   qinfo    {posEntry, size} per query
 *   cands16  API candInfo_t (16 B); positions must fit 32 bits
 *   res      receives {column, score}, pre-filled {0, 0xFFFFFFFF} (:251-255)
 *
 * Returns 0, -1 for a position beyond 32 bits, -3 for mixed query lengths.
 */
int refshim_verify_exact(const uint32_t *peq128, const uint32_t *qinfo, uint32_t num_queries,
                         const void *cands16, uint32_t num_cands,
                         uint32_t *ref, uint32_t ref_words, uint32_t ref_size,
                         float distance, resEntry_t *res, int nthreads, double *seconds)
{
    if (num_queries == 0) return 0;
    uint32_t m = qinfo[1];
    for (uint32_t qi = 0; qi < num_queries; ++qi)
        if (qinfo[2 * qi + 1] != m) return -3;
    uint32_t nepq = (m / SIZE_HW_WORD) + ((m % SIZE_HW_WORD) ? 1 : 0);

    qryEntry_t *q32 = (qryEntry_t *)calloc((size_t)num_queries * (nepq ? nepq : 1), sizeof(qryEntry_t));
    candInfo_t *c8 = (candInfo_t *)malloc(sizeof(candInfo_t) * (num_cands ? num_cands : 1));
    if (q32 == NULL || c8 == NULL) { free(q32); free(c8); return -2; }
    for (uint32_t qi = 0; qi < num_queries; ++qi) {
        uint32_t pe = qinfo[2 * qi];
        for (uint32_t b = 0; b < nepq; ++b)
            for (uint32_t c = 0; c < NUM_BASES; ++c)
                q32[(size_t)qi * nepq + b].bitmap[c] = peq128[(size_t)(pe + b / 4) * 20 + c * 4 + b % 4];
    }
    const uint8_t *src = (const uint8_t *)cands16;
    for (uint32_t i = 0; i < num_cands; ++i) {
        uint32_t q;
        uint64_t pos;
        memcpy(&q, src + 16 * (size_t)i, 4);
        memcpy(&pos, src + 16 * (size_t)i + 8, 8);
        if (pos > 0xFFFFFFFFull) { free(q32); free(c8); return -1; }
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
    q.totalQueriesEntries = num_queries * nepq;
    q.sizeQueries = m;
    q.numQueries = num_queries;
    q.numCandidates = num_cands;
    q.distance = distance;
    q.h_queries = q32;
    q.h_candidates = c8;

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
    double t1 = omp_get_wtime();
    if (seconds) *seconds = t1 - t0;
    free(q32);
    free(c8);
    return 0;
}
