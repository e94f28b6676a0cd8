/*
 * CPU oracle for Myers candidate verification.
 *
 * TEST INFRASTRUCTURE ONLY. This file restates, in plain C, the reference
 * algorithm that the CUDA path must reproduce bit for bit. Only the tests,
 * the smoke check and the CPU-baseline leg of the benchmark load it, and only
 * as the checker. The product library never links or calls it.
 *
 * Every function cites the reference lines it follows (paths are relative to
 * the achacond/myers-gpu source tree).
 *
 * Parity pin: the restatement is checked against fixtures produced by the
 * reference's own CPU Myers (src-integration/myers-reorderBuffer-padding.c
 * and src/myers-4bits.c) and by its own packers (src-api/genReference-4bits.c,
 * src-api/genCandidate-reorder.c); see tests/golden/make_golden.py.
 *
 * Defined behaviour where the reference is undefined:
 *   - text words past the end of the packed reference read as ORC_PAD_WORD
 *     (eight N codes). The reference reads past its array there.
 *   - reference codes 5..7 behave as A (code 0), as in the reference GPU
 *     kernel (coreMyersGPU-CC50.cu:82-95); the reference CPU code indexes past
 *     the PEQ entry for them. The packers never produce them.
 *   - a candidate whose window does not fit gets {column 0, score 0xFFFFFFFF},
 *     the value the reference CPU oracle pre-fills
 *     (myers-reorderBuffer-padding.c:290-294).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PAD_WORD 0x44444444u
#define ORC_NO_RESULT 0xFFFFFFFFu

typedef struct { uint32_t bitmap[5][4]; } orc_peq_t;          /* myers-interface.h:10-12 */
typedef struct { uint32_t query; uint32_t _pad; uint64_t position; } orc_cand_t; /* :19-22 */
typedef struct { uint32_t posEntry; uint32_t size; } orc_qinfo_t;               /* :24-27 */
typedef struct { uint32_t column; uint32_t score; } orc_res_t;                 /* :14-17 */

/* Window length W in bases: float32 product truncated to an integer.
 * myers-reorderBuffer-padding.c:195, coreMyersGPU-CC50.cu:131. */
uint32_t orc_window_bases(uint32_t m, float distance)
{
    float factor = 1.0f + 2.0f * distance;
    return (uint32_t)((float)m * factor);
}

/* Number of packed 8-base words the aligned window reads (8 columns each).
 * myers-reorderBuffer-padding.c:198, coreMyersGPU-CC50.cu:132. */
uint32_t orc_window_words(uint32_t W)
{
    return W / 8 + ((W % 8) ? 2 : 1);
}

static inline uint32_t ref_word(const uint32_t *ref, uint64_t ref_words, uint64_t idx)
{
    return idx < ref_words ? ref[idx] : ORC_PAD_WORD;
}

static inline uint32_t code_of(uint32_t nibble)
{
    uint32_t c = nibble & 7u;      /* coreMyersGPU-CC50.cu:170 */
    return c > 4u ? 0u : c;
}

/* One column of the block-wise bit-parallel recurrence over nblk 32-bit
 * blocks, with the horizontal delta handed from block to block (Myers 1999
 * block form). Returns the horizontal delta out of the last query row.
 * myers-reorderBuffer-padding.c:131-161 and src/myers-4bits.c:111-135. */
static int column_step(const orc_peq_t *peq, uint32_t pos_entry, uint32_t nblk,
                       uint32_t last_mask, uint32_t code, uint32_t *Pv, uint32_t *Mv)
{
    int hin = 0;
    for (uint32_t b = 0; b < nblk; ++b) {
        uint32_t eq = peq[pos_entry + b / 4].bitmap[code][b % 4];
        uint32_t mask = (b + 1 == nblk) ? last_mask : 0x80000000u;
        uint32_t pv = Pv[b], mv = Mv[b];
        uint32_t xv = eq | mv;
        if (hin < 0) eq |= 1u;
        uint32_t xh = (((eq & pv) + pv) ^ pv) | eq;
        uint32_t ph = mv | ~(xh | pv);
        uint32_t mh = pv & xh;
        int hout = ((ph & mask) != 0) - ((mh & mask) != 0);
        ph <<= 1;
        mh <<= 1;
        if (hin < 0) mh |= 1u;
        else if (hin > 0) ph |= 1u;
        Pv[b] = mh | ~(xv | ph);
        Mv[b] = ph & xv;
        hin = hout;
    }
    return hin;
}

static uint32_t last_row_mask(uint32_t m)
{
    /* myers-reorderBuffer-padding.c:113 */
    return (m % 32 == 0) ? 0x80000000u : (1u << (m % 32 - 1));
}

/* Aligned-window mode, the API semantics: the text starts at the packed word
 * holding `pos` and spans 8*E columns; the column is relative to that word.
 * myers-reorderBuffer-padding.c:97-176 (computeMyers), sizing :192-198,
 * validity :118. */
void orc_myers_aligned_one(const orc_peq_t *peq, const uint32_t *ref, uint64_t ref_words,
                           uint64_t ref_size, uint32_t pos_entry, uint32_t m, uint64_t pos,
                           float distance, orc_res_t *out)
{
    uint32_t W = orc_window_bases(m, distance);
    out->column = 0;
    out->score = ORC_NO_RESULT;
    if (!(pos < ref_size && ref_size - pos > W)) return;

    uint32_t E = orc_window_words(W);
    uint32_t nblk = (m + 31) / 32;
    uint32_t *Pv = (uint32_t *)malloc(sizeof(uint32_t) * (nblk ? nblk : 1) * 2);
    uint32_t *Mv = Pv + (nblk ? nblk : 1);
    for (uint32_t b = 0; b < nblk; ++b) { Pv[b] = 0xFFFFFFFFu; Mv[b] = 0u; }
    uint32_t last_mask = last_row_mask(m);

    int32_t score = (int32_t)m, best = (int32_t)m;
    uint32_t best_col = 0, col = 0;
    uint64_t w0 = pos / 8;
    for (uint32_t e = 0; e < E; ++e) {
        uint32_t word = ref_word(ref, ref_words, w0 + e);
        for (uint32_t k = 0; k < 8; ++k, ++col) {
            uint32_t code = code_of(word >> (4 * k));
            score += column_step(peq, pos_entry, nblk, last_mask, code, Pv, Mv);
            if (score < best) { best = score; best_col = col; }
        }
    }
    free(Pv);
    out->column = best_col;
    out->score = (uint32_t)best;
}

/* Exact-window mode: the text starts exactly at `pos` and spans W columns;
 * the column is relative to `pos`. src/myers-4bits.c:75-153 (which reads one
 * fixed query length with 32-base PEQ entries; this form takes the API's
 * 128-base entries and a per-query length). */
void orc_myers_exact_one(const orc_peq_t *peq, const uint32_t *ref, uint64_t ref_words,
                         uint64_t ref_size, uint32_t pos_entry, uint32_t m, uint64_t pos,
                         float distance, orc_res_t *out)
{
    uint32_t W = orc_window_bases(m, distance);
    out->column = 0;
    out->score = ORC_NO_RESULT;
    if (!(pos < ref_size && ref_size - pos > W)) return;

    uint32_t nblk = (m + 31) / 32;
    uint32_t *Pv = (uint32_t *)malloc(sizeof(uint32_t) * (nblk ? nblk : 1) * 2);
    uint32_t *Mv = Pv + (nblk ? nblk : 1);
    for (uint32_t b = 0; b < nblk; ++b) { Pv[b] = 0xFFFFFFFFu; Mv[b] = 0u; }
    uint32_t last_mask = last_row_mask(m);

    int32_t score = (int32_t)m, best = (int32_t)m;
    uint32_t best_col = 0;
    for (uint32_t col = 0; col < W; ++col) {
        uint64_t p = pos + col;
        uint32_t code = code_of(ref_word(ref, ref_words, p / 8) >> (4 * (p % 8)));
        score += column_step(peq, pos_entry, nblk, last_mask, code, Pv, Mv);
        if (score < best) { best = score; best_col = col; }
    }
    free(Pv);
    out->column = best_col;
    out->score = (uint32_t)best;
}

/* Batch drivers (OpenMP over candidates, as the reference's
 * computeAllQueriesCPU, myers-reorderBuffer-padding.c:178-208, minus its
 * 4096-base cap). exact != 0 selects the exact-window mode. */
void orc_verify(const orc_peq_t *peq, const orc_qinfo_t *qinfo, const orc_cand_t *cands,
                uint64_t num_cands, const uint32_t *ref, uint64_t ref_words, uint64_t ref_size,
                float distance, int exact, orc_res_t *res, int nthreads)
{
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
#endif
    for (int64_t i = 0; i < (int64_t)num_cands; ++i) {
        const orc_qinfo_t q = qinfo[cands[i].query];
        if (exact)
            orc_myers_exact_one(peq, ref, ref_words, ref_size, q.posEntry, q.size,
                                cands[i].position, distance, &res[i]);
        else
            orc_myers_aligned_one(peq, ref, ref_words, ref_size, q.posEntry, q.size,
                                  cands[i].position, distance, &res[i]);
    }
}

/* Base code of an ASCII base: A0 C1 G2 T3, anything else 4.
 * src-api/genReference-4bits.c:21-40 (codes), genCandidate-reorder.c:237-256
 * (the same five classes as one-hot bits). */
static inline uint32_t ascii_code(uint8_t b)
{
    switch (b) {
    case 'A': case 'a': return 0;
    case 'C': case 'c': return 1;
    case 'G': case 'g': return 2;
    case 'T': case 't': return 3;
    default: return 4;
    }
}

/* Pack n ASCII bases, 8 per 32-bit word, base i in bits 4*(i%8)..+3 of word
 * i/8. Nibbles past n in the last word are N (4).
 * src-api/genReference-4bits.c:43-72. */
void orc_pack_reference(const uint8_t *ascii, uint64_t n, uint32_t *words)
{
    uint64_t nw = (n + 7) / 8;
    for (uint64_t w = 0; w < nw; ++w) {
        uint32_t v = 0;
        for (uint32_t k = 0; k < 8; ++k) {
            uint64_t i = w * 8 + k;
            uint32_t c = i < n ? ascii_code(ascii[i]) : 4u;
            v |= c << (4 * k);
        }
        words[w] = v;
    }
}

/* Build the PEQ entries of one read: ceil(m/128) entries; bit i%32 of
 * bitmap[c][(i%128)/32] of entry i/128 is set iff base i has code c.
 * src-api/genCandidate-reorder.c:258-317. */
void orc_pack_peq(const uint8_t *read, uint32_t m, orc_peq_t *entries)
{
    uint32_t ne = (m + 127) / 128;
    memset(entries, 0, sizeof(orc_peq_t) * ne);
    for (uint32_t i = 0; i < m; ++i) {
        uint32_t c = ascii_code(read[i]);
        entries[i / 128].bitmap[c][(i % 128) / 32] |= 1u << (i % 32);
    }
}

/* ---------------------------------------------------------------------------
 * Traceback of an accepted candidate. Not in the reference: the reference
 * returns only (column, score). This is the checker of the GPU traceback and
 * defines its result:
 *
 *   For a candidate whose result (column c, score s) has s <= max_score, the
 *   alignment is the path through the semi-global edit-distance matrix
 *   (D[0][j] = 0, D[i][0] = i, unit costs; query row i matches text column j
 *   iff PEQ[code of text j] has bit i-1, so N matches N) from (m, c+1) back
 *   to row 0, choosing at each cell, in this order: the diagonal
 *   (D[i-1][j-1] + mismatch == D[i][j]; '=' or 'X'), the query base alone
 *   (D[i-1][j] + 1 == D[i][j]; 'I'), the text base alone ('D'). Columns are
 *   window columns as in the verification (aligned or exact window).
 *
 * Record: start column (first text column consumed; c+1 when none), number
 * of run-length ops, score, end column. ops[k] = length << 4 | code with the
 * SAM codes '=' 7, 'X' 8, 'I' 1, 'D' 2, first op first. numOps is
 * ORC_TB_NOT_TRACED when s > max_score or the candidate has no result,
 * ORC_TB_INCONSISTENT when (c, s) is not the inputs' result at c, and a
 * count above max_ops when the ops did not fit (ops then unspecified).
 * ------------------------------------------------------------------------- */
#define ORC_TB_NOT_TRACED 0xFFFFFFFFu
#define ORC_TB_INCONSISTENT 0xFFFFFFFEu

typedef struct { uint32_t start_column; uint32_t num_ops; uint32_t score; uint32_t end_column; } orc_aln_t;

static inline uint32_t text_code(const uint32_t *ref, uint64_t ref_words, uint64_t base)
{
    return code_of(ref_word(ref, ref_words, base / 8) >> (4 * (base % 8)));
}

static inline int peq_bit(const orc_peq_t *peq, uint32_t pos_entry, uint32_t code, uint32_t row0)
{
    return (peq[pos_entry + row0 / 128].bitmap[code][(row0 % 128) / 32] >> (row0 % 32)) & 1u;
}

static void push_op(uint32_t *ops, uint32_t max_ops, uint32_t *n, uint32_t *cur, uint32_t *len, uint32_t op)
{
    if (*len && *cur == op) { ++*len; return; }
    if (*len) {
        if (*n < max_ops) ops[*n] = (*len << 4) | *cur;
        ++*n;
    }
    *cur = op;
    *len = 1;
}

void orc_traceback_one(const orc_peq_t *peq, const uint32_t *ref, uint64_t ref_words, uint64_t ref_size,
                       uint32_t pos_entry, uint32_t m, uint64_t pos, float distance, int exact,
                       orc_res_t res, uint32_t max_score, uint32_t *ops, uint32_t max_ops, orc_aln_t *aln)
{
    aln->score = res.score;
    aln->end_column = res.column;
    aln->start_column = ORC_TB_NOT_TRACED;
    aln->num_ops = ORC_TB_NOT_TRACED;
    if (res.score == ORC_NO_RESULT || res.score > max_score) return;
    aln->num_ops = ORC_TB_INCONSISTENT;
    const uint32_t W = orc_window_bases(m, distance);
    if (!(pos < ref_size && ref_size - pos > W)) return;
    const uint64_t ncols = exact ? W : 8ull * orc_window_words(W);
    const uint64_t start = exact ? pos : (pos / 8) * 8;
    const uint64_t c1 = (uint64_t)res.column + 1;  /* 1-based end column */
    if (c1 > ncols) return;
    /* The path consumes at most m + s text bases, so it stays in columns
     * >= a0; earlier columns are computed but not kept. */
    const uint64_t a0 = c1 > (uint64_t)m + res.score ? c1 - m - res.score : 0;
    const uint64_t kept = c1 - a0 + 1;
    uint16_t *D = (uint16_t *)malloc(sizeof(uint16_t) * (m + 1) * kept);
    uint16_t *col = (uint16_t *)malloc(sizeof(uint16_t) * (m + 1) * 2);
    if (!D || !col) { free(D); free(col); return; }
    uint16_t *prev = col, *cur = col + (m + 1);
    for (uint32_t i = 0; i <= m; ++i) prev[i] = (uint16_t)i;
    if (a0 == 0) memcpy(D, prev, sizeof(uint16_t) * (m + 1));
    for (uint64_t j = 1; j <= c1; ++j) {
        const uint32_t t = text_code(ref, ref_words, start + j - 1);
        cur[0] = 0;
        for (uint32_t i = 1; i <= m; ++i) {
            uint32_t d = prev[i - 1] + (peq_bit(peq, pos_entry, t, i - 1) ? 0u : 1u);
            uint32_t u = cur[i - 1] + 1u, l = prev[i] + 1u;
            if (u < d) d = u;
            if (l < d) d = l;
            cur[i] = (uint16_t)d;
        }
        if (j >= a0) memcpy(D + (j - a0) * (m + 1), cur, sizeof(uint16_t) * (m + 1));
        uint16_t *x = prev; prev = cur; cur = x;
    }
    if (D[(c1 - a0) * (m + 1) + m] != res.score) { free(D); free(col); return; }
#define DV(i, j) ((uint32_t)D[((j) - a0) * (m + 1) + (i)])
    uint32_t n = 0, cur_op = 0, len = 0;
    /* ops are produced last first; reversed below */
    uint32_t *rev = (uint32_t *)malloc(sizeof(uint32_t) * (m + c1 + 1));
    uint32_t i = m;
    uint64_t j = c1;
    while (i > 0) {
        uint32_t op;
        if (j == 0 || j <= a0) {
            /* j <= a0 only when a0 == 0 (the path never leaves columns >= a0) */
            op = 1; --i;
        } else {
            const uint32_t t = text_code(ref, ref_words, start + j - 1);
            const int match = peq_bit(peq, pos_entry, t, i - 1);
            if (DV(i - 1, j - 1) + (match ? 0u : 1u) == DV(i, j)) { op = match ? 7u : 8u; --i; --j; }
            else if (DV(i - 1, j) + 1u == DV(i, j)) { op = 1; --i; }
            else { op = 2; --j; }
        }
        push_op(rev, m + (uint32_t)c1 + 1, &n, &cur_op, &len, op);
    }
#undef DV
    if (len) rev[n++] = (len << 4) | cur_op;
    aln->start_column = (uint32_t)j;
    aln->num_ops = n;
    if (n <= max_ops)
        for (uint32_t k = 0; k < n; ++k) ops[k] = rev[n - 1 - k];
    free(rev);
    free(D);
    free(col);
}

void orc_traceback(const orc_peq_t *peq, const orc_qinfo_t *qinfo, const orc_cand_t *cands,
                   const orc_res_t *res, uint64_t num_cands, const uint32_t *ref, uint64_t ref_words,
                   uint64_t ref_size, float distance, int exact, uint32_t max_score, uint32_t *ops,
                   uint32_t max_ops, orc_aln_t *aln, int nthreads)
{
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
#endif
    for (int64_t k = 0; k < (int64_t)num_cands; ++k) {
        const orc_qinfo_t q = qinfo[cands[k].query];
        orc_traceback_one(peq, ref, ref_words, ref_size, q.posEntry, q.size, cands[k].position, distance, exact,
                          res[k], max_score, ops + (uint64_t)k * max_ops, max_ops, &aln[k]);
    }
}
