/*
 * Seeded synthetic workloads for Myers candidate verification.
 *
 * The reference's datasets (a human reference and GEM candidate profiles) are
 * not available, so the benchmark and the tests generate inputs with the same
 * shapes: a 4-bit packed reference of i.i.d. A/C/G/T with runs of N, reads
 * copied from it and mutated, and per read one true candidate window plus
 * uniform decoys. Outputs use the API layouts of myers-interface.h (PEQ
 * entries of 128 bases, 16-byte candidates, {posEntry,size} query info).
 *
 * Every random draw comes from a counter-based stream keyed by (seed, object
 * index), so the output does not depend on the number of threads.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { uint32_t bitmap[5][4]; } syn_peq_t;
typedef struct { uint32_t query; uint32_t pad; uint64_t position; } syn_cand_t;
typedef struct { uint32_t posEntry; uint32_t size; } syn_qinfo_t;

typedef struct {
    uint64_t ref_size;       /* bases in the reference */
    uint32_t num_reads;
    /* read lengths: 0 fixed, 1 weighted set, 2 log-uniform [lo,hi], 3 uniform over set */
    uint32_t len_kind;
    uint32_t len_fixed;
    uint32_t len_lo, len_hi;
    uint32_t len_set_n;
    uint32_t len_set[16];
    double len_weights[16];
    /* mutations: 0 fixed per-base rates, 1 per-read total rate uniform in
     * [rate_lo, rate_hi] split sub:ins:del = 0.8:0.1:0.1 */
    uint32_t mut_kind;
    double sub, ins, del;
    double rate_lo, rate_hi;
    double indel_mean;       /* mean indel length (geometric); <= 1 gives single bases */
    /* candidates per read: 0 fixed, 1 1+Poisson(lambda) capped, 2 uniform [lo,hi] */
    uint32_t cand_kind;
    uint32_t cand_fixed;
    double cand_lambda;
    uint32_t cand_cap;
    uint32_t cand_lo, cand_hi;
    uint32_t jitter;         /* true window start jitter, +-bases */
    float distance;          /* error bound: window = read length * (1 + 2*distance) */
    uint64_t seed;
} synth_spec_t;

/* ---- counter-based random streams (splitmix64 seeding, xoshiro256**) ---- */

typedef struct { uint64_t s[4]; } rng_t;

static inline uint64_t splitmix64(uint64_t *x)
{
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline void rng_init(rng_t *r, uint64_t seed, uint64_t stream, uint64_t index)
{
    uint64_t x = seed ^ (stream * 0xD1B54A32D192ED03ull) ^ (index * 0x8CB92BA72F3D8DD7ull);
    for (int i = 0; i < 4; ++i) r->s[i] = splitmix64(&x);
}

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static inline uint64_t rng_next(rng_t *r)
{
    uint64_t *s = r->s;
    uint64_t result = rotl(s[1] * 5, 7) * 9;
    uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl(s[3], 45);
    return result;
}

static inline double rng_unit(rng_t *r) { return (rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }

static inline uint64_t rng_below(rng_t *r, uint64_t n)
{
    return n ? (uint64_t)(((unsigned __int128)rng_next(r) * n) >> 64) : 0;
}

static uint32_t rng_poisson(rng_t *r, double lambda)
{
    double l = exp(-lambda), p = 1.0;
    uint32_t k = 0;
    do { ++k; p *= rng_unit(r); } while (p > l && k < 10000);
    return k - 1;
}

/* geometric on {1,2,...} with the given mean */
static uint32_t rng_geometric(rng_t *r, double mean)
{
    if (mean <= 1.0) return 1;
    double p = 1.0 / mean, u = rng_unit(r);
    uint32_t k = 1 + (uint32_t)floor(log1p(-u) / log1p(-p));
    return k > 1000 ? 1000 : k;
}

enum { STREAM_REF = 1, STREAM_NRUN = 2, STREAM_PLAN = 3, STREAM_FILL = 4 };

/* ---- reference ---- */

#define SYN_PAD_WORD 0x44444444u

/*
 * Packed reference of `size` bases: i.i.d. uniform A/C/G/T, then runs of N
 * (code 4) of length uniform in [run_min, run_max] covering about n_frac of
 * the bases. words must hold nwords >= ceil(size/8) entries; nibbles past
 * `size` and words past ceil(size/8) are N.
 */
int synth_reference(uint64_t size, double n_frac, uint32_t run_min, uint32_t run_max,
                    uint64_t seed, uint32_t *words, uint64_t nwords)
{
    uint64_t used = (size + 7) / 8;
    if (nwords < used) return -1;
    const uint64_t chunk = 1u << 16; /* words per random stream */
    uint64_t nchunks = (used + chunk - 1) / chunk;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < (int64_t)nchunks; ++c) {
        rng_t r;
        rng_init(&r, seed, STREAM_REF, (uint64_t)c);
        uint64_t w0 = (uint64_t)c * chunk, w1 = w0 + chunk < used ? w0 + chunk : used;
        for (uint64_t w = w0; w < w1; w += 4) {
            uint64_t bits = rng_next(&r); /* 2 bits per base, 32 bases */
            for (uint64_t k = 0; k < 4 && w + k < w1; ++k) {
                uint32_t b16 = (uint32_t)(bits >> (16 * k)) & 0xFFFFu;
                uint32_t v = 0;
                for (int i = 0; i < 8; ++i) v |= ((b16 >> (2 * i)) & 3u) << (4 * i);
                words[w + k] = v;
            }
        }
    }
    /* N runs */
    rng_t r;
    rng_init(&r, seed, STREAM_NRUN, 0);
    double mean_run = 0.5 * (run_min + run_max);
    uint64_t nruns = (n_frac > 0 && mean_run > 0) ? (uint64_t)llround(size * n_frac / mean_run) : 0;
    for (uint64_t i = 0; i < nruns; ++i) {
        uint64_t len = run_min + rng_below(&r, (uint64_t)(run_max - run_min + 1));
        uint64_t start = rng_below(&r, size);
        for (uint64_t p = start; p < start + len && p < size; ++p)
            words[p / 8] |= 4u << (4 * (p % 8)), words[p / 8] &= ~(3u << (4 * (p % 8)));
    }
    /* tail nibbles and padding words */
    for (uint64_t p = size; p < used * 8; ++p) {
        words[p / 8] &= ~(0xFu << (4 * (p % 8)));
        words[p / 8] |= 4u << (4 * (p % 8));
    }
    for (uint64_t w = used; w < nwords; ++w) words[w] = SYN_PAD_WORD;
    return 0;
}

/* ---- reads and candidates ---- */

static uint32_t draw_length(const synth_spec_t *s, rng_t *r)
{
    switch (s->len_kind) {
    case 1: {
        double tot = 0, u;
        for (uint32_t i = 0; i < s->len_set_n; ++i) tot += s->len_weights[i];
        u = rng_unit(r) * tot;
        for (uint32_t i = 0; i < s->len_set_n; ++i) {
            if (u < s->len_weights[i]) return s->len_set[i];
            u -= s->len_weights[i];
        }
        return s->len_set[s->len_set_n - 1];
    }
    case 2: {
        double lo = log((double)s->len_lo), hi = log((double)s->len_hi);
        uint32_t m = (uint32_t)llround(exp(lo + (hi - lo) * rng_unit(r)));
        return m < s->len_lo ? s->len_lo : (m > s->len_hi ? s->len_hi : m);
    }
    case 3:
        return s->len_set[rng_below(r, s->len_set_n)];
    default:
        return s->len_fixed;
    }
}

static uint32_t draw_cands(const synth_spec_t *s, rng_t *r)
{
    switch (s->cand_kind) {
    case 1: {
        uint32_t k = 1 + rng_poisson(r, s->cand_lambda);
        return (s->cand_cap && k > s->cand_cap) ? s->cand_cap : k;
    }
    case 2:
        return s->cand_lo + (uint32_t)rng_below(r, (uint64_t)(s->cand_hi - s->cand_lo + 1));
    default:
        return s->cand_fixed;
    }
}

static inline uint32_t window_bases(uint32_t m, float distance)
{
    float factor = 1.0f + 2.0f * distance;
    return (uint32_t)((float)m * factor);
}

/*
 * Per-read lengths and candidate counts, and the totals the caller needs to
 * size its arrays.
 */
int synth_plan(const synth_spec_t *s, uint32_t *lengths, uint32_t *ncands,
               uint64_t *tot_entries, uint64_t *tot_cands, uint64_t *tot_bases)
{
    uint64_t te = 0, tc = 0, tb = 0;
#pragma omp parallel for schedule(static) reduction(+ : te, tc, tb)
    for (int64_t i = 0; i < (int64_t)s->num_reads; ++i) {
        rng_t r;
        rng_init(&r, s->seed, STREAM_PLAN, (uint64_t)i);
        uint32_t m = draw_length(s, &r);
        uint32_t k = draw_cands(s, &r);
        lengths[i] = m;
        ncands[i] = k;
        te += (m + 127) / 128;
        tc += k;
        tb += m;
    }
    *tot_entries = te;
    *tot_cands = tc;
    *tot_bases = tb;
    return 0;
}

static inline uint32_t ref_code(const uint32_t *words, uint64_t p)
{
    return (words[p / 8] >> (4 * (p % 8))) & 0xFu;
}

static const char ASCII_OF[5] = {'A', 'C', 'G', 'T', 'N'};

/*
 * Fill queries and candidates. For read i: copy from a uniform reference
 * position (away from the last W+16 bases), mutate, pack its PEQ entries,
 * then emit one true window (read start - floor(distance*m) +- jitter) at a
 * uniform slot among its candidates, the others uniform decoys.
 *
 * ascii (optional) receives the read bases back to back; true_pos (optional)
 * the reference start of each read.
 */
int synth_fill(const synth_spec_t *s, const uint32_t *ref_words, const uint32_t *lengths,
               const uint32_t *ncands, syn_qinfo_t *qinfo, syn_peq_t *peq, syn_cand_t *cands,
               uint8_t *ascii, uint64_t *true_pos)
{
    uint32_t n = s->num_reads;
    uint64_t *entry_off = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)n + 1));
    uint64_t *cand_off = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)n + 1));
    uint64_t *base_off = (uint64_t *)malloc(sizeof(uint64_t) * ((size_t)n + 1));
    if (!entry_off || !cand_off || !base_off) { free(entry_off); free(cand_off); free(base_off); return -2; }
    entry_off[0] = cand_off[0] = base_off[0] = 0;
    for (uint32_t i = 0; i < n; ++i) {
        entry_off[i + 1] = entry_off[i] + (lengths[i] + 127) / 128;
        cand_off[i + 1] = cand_off[i] + ncands[i];
        base_off[i + 1] = base_off[i] + lengths[i];
    }
    if (entry_off[n] > 0xFFFFFFFFull) { free(entry_off); free(cand_off); free(base_off); return -3; }
    int err = 0;

#pragma omp parallel
    {
        uint32_t cap = 0;
        uint8_t *codes = NULL;
#pragma omp for schedule(dynamic, 64)
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            uint32_t i = (uint32_t)ii;
            uint32_t m = lengths[i];
            if (m + 1 > cap) {
                cap = m + 1;
                uint8_t *nc = (uint8_t *)realloc(codes, cap);
                if (!nc) { err = -2; continue; }
                codes = nc;
            }
            rng_t r;
            rng_init(&r, s->seed, STREAM_FILL, i);
            double sub = s->sub, ins = s->ins, del = s->del;
            if (s->mut_kind == 1) {
                double rate = s->rate_lo + (s->rate_hi - s->rate_lo) * rng_unit(&r);
                sub = 0.8 * rate; ins = 0.1 * rate; del = 0.1 * rate;
            }
            uint32_t W = window_bases(m, s->distance);
            uint64_t span_max = (uint64_t)W + 2 * (uint64_t)m + 64; /* read walk can exceed m with deletions */
            uint64_t lim = s->ref_size > span_max + 16 ? s->ref_size - span_max - 16 : 1;
            uint64_t p0 = rng_below(&r, lim);
            uint64_t p = p0;
            uint32_t emitted = 0;
            while (emitted < m) {
                double u = rng_unit(&r);
                uint32_t base = p < s->ref_size ? ref_code(ref_words, p) : 4u;
                if (u < sub) {
                    uint32_t nb = (uint32_t)rng_below(&r, 3);
                    if (base < 4 && nb >= base) ++nb;
                    codes[emitted++] = (uint8_t)(base < 4 ? nb : nb);
                    ++p;
                } else if (u < sub + ins) {
                    uint32_t len = rng_geometric(&r, s->indel_mean);
                    for (uint32_t k = 0; k < len && emitted < m; ++k)
                        codes[emitted++] = (uint8_t)rng_below(&r, 4);
                } else if (u < sub + ins + del) {
                    p += rng_geometric(&r, s->indel_mean);
                } else {
                    codes[emitted++] = (uint8_t)base;
                    ++p;
                }
            }
            /* PEQ entries */
            uint64_t e0 = entry_off[i];
            uint32_t ne = (m + 127) / 128;
            memset(&peq[e0], 0, sizeof(syn_peq_t) * ne);
            for (uint32_t k = 0; k < m; ++k)
                peq[e0 + k / 128].bitmap[codes[k]][(k % 128) / 32] |= 1u << (k % 32);
            qinfo[i].posEntry = (uint32_t)e0;
            qinfo[i].size = m;
            if (ascii)
                for (uint32_t k = 0; k < m; ++k) ascii[base_off[i] + k] = (uint8_t)ASCII_OF[codes[k]];
            if (true_pos) true_pos[i] = p0;
            /* candidates */
            uint32_t nc = ncands[i];
            uint64_t c0 = cand_off[i];
            uint64_t dec_lim = s->ref_size > (uint64_t)W + 17 ? s->ref_size - W - 17 : 1;
            uint32_t true_slot = nc ? (uint32_t)rng_below(&r, nc) : 0;
            for (uint32_t k = 0; k < nc; ++k) {
                uint64_t pos;
                if (k == true_slot) {
                    int64_t t = (int64_t)p0 - (int64_t)floor((double)s->distance * m)
                              + (int64_t)rng_below(&r, 2 * (uint64_t)s->jitter + 1) - (int64_t)s->jitter;
                    if (t < 0) t = 0;
                    if ((uint64_t)t >= dec_lim) t = (int64_t)dec_lim - 1;
                    pos = (uint64_t)t;
                } else {
                    pos = rng_below(&r, dec_lim);
                }
                cands[c0 + k].query = i;
                cands[c0 + k].pad = 0;
                cands[c0 + k].position = pos;
            }
        }
        free(codes);
    }
    free(entry_off);
    free(cand_off);
    free(base_off);
    return err;
}
