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
