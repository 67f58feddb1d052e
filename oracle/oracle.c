/*
 * CPU oracle for the all-vs-all scoring path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C, the reference seqtree arithmetic for the four dense
 * matrix calls that the CUDA library replaces.  It exists to CHECK the CUDA path: only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark may load it, and never
 * as the thing being measured or shipped.  The product path has no CPU fallback.
 *
 * Parity is pinned two ways (see tests/test_oracle_golden.py):
 *   - against golden vectors produced by the reference's own C++ compiled from its sources
 *     (oracle/Makefile -> oracle/_ref/libseqtree_ref.so, fixtures under tests/golden/);
 *   - against the known answers the reference's own tests hold for this path.
 *
 * Citations are file:line inside the seqtree 0.6.0 project.
 */
#include <limits.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- codec ------------ */
/* Symbol orders and case folding follow src/codec.cpp:9-35. */
static const char *const kSymbols[3] = {"ARNDCQEGHILKMFPSTWYVBZX*", "ACGT", "ACGTRYSWKMBDHVN"};

int or_alphabet_size(int alphabet) {
    if (alphabet < 0 || alphabet > 2) return -1;
    return (int)strlen(kSymbols[alphabet]);
}

/* Fills lut[256] with codes; 0xFF marks a symbol outside the alphabet. */
void or_codec_lut(int alphabet, uint8_t *lut) {
    memset(lut, 0xFF, 256);
    const char *s = kSymbols[alphabet];
    for (int i = 0; s[i]; ++i) {
        unsigned char up = (unsigned char)s[i];
        unsigned char lo = (up >= 'A' && up <= 'Z') ? (unsigned char)(up - 'A' + 'a') : up;
        lut[up] = (uint8_t)i;
        lut[lo] = (uint8_t)i;
    }
}

/* Encodes bytes[0..n) in place order; returns -1 on success or the index of the first byte
 * that is not in the alphabet (src/gapblock.cpp:12-22, src/pairwise.cpp:51-60). */
int64_t or_encode(int alphabet, const uint8_t *bytes, int64_t n, uint8_t *codes) {
    uint8_t lut[256];
    or_codec_lut(alphabet, lut);
    for (int64_t i = 0; i < n; ++i) {
        uint8_t v = lut[bytes[i]];
        if (v == 0xFF) return i;
        codes[i] = v;
    }
    return -1;
}

/* ----------------------------------------------------------- substitution ---------- */
/* Gram transform pen = s_aa + s_bb - 2 s_ab clamped at 0
 * (src/substitution_matrix.cpp:29-50); unit cost when sim is NULL (:15-27). */
void or_penalty_from_similarity(int A, const int32_t *sim, int32_t *pen) {
    for (int a = 0; a < A; ++a)
        for (int b = 0; b < A; ++b) {
            if (!sim) {
                pen[a * A + b] = (a != b);
                continue;
            }
            int32_t p = sim[a * A + a] + sim[b * A + b] - 2 * sim[a * A + b];
            pen[a * A + b] = p < 0 ? 0 : p;
        }
}

/* ----------------------------------------------------------- gap block ------------- */
/* One (query, ref) gap-block penalty, restating src/gapblock.cpp:39-62:
 *   suffix on diagonal d (offset on the longer sequence), prefix on diagonal 0,
 *   min over the L+1 block positions of prefix + suffix + prior, plus the affine gap cost;
 *   d == 0 returns the plain substitution sum (no gap cost, no prior). */
int32_t or_gapblock_cell(const uint8_t *q, uint32_t m, const uint8_t *r, uint32_t n,
                         const int32_t *pen, int A, int32_t gap_open, int32_t gap_extend,
                         const int32_t *prior_row, int32_t *suf) {
    const uint32_t L = m < n ? m : n;
    const uint32_t d = m > n ? m - n : n - m;
    const int q_longer = m >= n;
    suf[L] = 0;
    for (uint32_t j = L; j-- > 0;) {
        uint8_t a = q_longer ? q[j + d] : q[j];
        uint8_t b = q_longer ? r[j] : r[j + d];
        suf[j] = suf[j + 1] + pen[a * A + b];
    }
    if (d == 0) return suf[0];
    int32_t pre = 0, best = INT32_MAX;
    for (uint32_t i = 0; i <= L; ++i) {
        int32_t cand = pre + suf[i] + (prior_row ? prior_row[i] : 0);
        if (cand < best) best = cand;
        if (i < L) pre += pen[q[i] * A + r[i]];
    }
    return best + gap_open + (int32_t)(d - 1) * gap_extend;
}

/* ----------------------------------------------------------- Gotoh NW/SW ----------- */
#define OR_NEG_INF (INT64_MIN / 4) /* src/pairwise.cpp:36-37 */

static int64_t gap_run(int64_t L, int32_t open, int32_t extend) { /* pairwise.cpp:71-73 */
    return L <= 0 ? 0 : (int64_t)open + (L - 1) * (int64_t)extend;
}

static int64_t max64(int64_t a, int64_t b) { return a > b ? a : b; }

/* Three-state Gotoh score, two rows per state, int64 cells: src/pairwise.cpp:76-125.
 * `scratch` holds 6*(n+1) int64. */
int64_t or_gotoh_score(const uint8_t *q, int64_t m, const uint8_t *r, int64_t n,
                       const int32_t *sim, int A, int local, int32_t go, int32_t ge,
                       int64_t *scratch) {
    if (m == 0 || n == 0) {
        if (local) return 0;
        return -gap_run(m ? m : n, go, ge);
    }
    int64_t *Mp = scratch, *Xp = Mp + (n + 1), *Yp = Xp + (n + 1);
    int64_t *Mc = Yp + (n + 1), *Xc = Mc + (n + 1), *Yc = Xc + (n + 1);
    Mp[0] = 0;
    Xp[0] = OR_NEG_INF;
    Yp[0] = OR_NEG_INF;
    for (int64_t j = 1; j <= n; ++j) {
        Mp[j] = local ? 0 : OR_NEG_INF;
        Xp[j] = OR_NEG_INF;
        Yp[j] = local ? OR_NEG_INF : -gap_run(j, go, ge);
    }
    int64_t best = local ? 0 : OR_NEG_INF;
    for (int64_t i = 1; i <= m; ++i) {
        Mc[0] = local ? 0 : OR_NEG_INF;
        Xc[0] = local ? OR_NEG_INF : -gap_run(i, go, ge);
        Yc[0] = OR_NEG_INF;
        for (int64_t j = 1; j <= n; ++j) {
            int64_t s = sim[q[i - 1] * A + r[j - 1]];
            int64_t diag = max64(Mp[j - 1], max64(Xp[j - 1], Yp[j - 1]));
            int64_t mv = diag + s;
            if (local && mv < 0) mv = 0;
            Mc[j] = mv;
            Xc[j] = max64(Mp[j] - go, max64(Xp[j] - ge, Yp[j] - go));
            Yc[j] = max64(Mc[j - 1] - go, max64(Yc[j - 1] - ge, Xc[j - 1] - go));
            if (local && mv > best) best = mv;
        }
        int64_t *t;
        t = Mp; Mp = Mc; Mc = t;
        t = Xp; Xp = Xc; Xc = t;
        t = Yp; Yp = Yc; Yc = t;
    }
    if (local) return best;
    return max64(Mp[n], max64(Xp[n], Yp[n]));
}

/* ----------------------------------------------------------- edit distances -------- */
/* Byte-wise, case-sensitive: src/distance.cpp:68-76 (caller checks equal lengths). */
int32_t or_hamming(const uint8_t *a, const uint8_t *b, int64_t L) {
    int32_t d = 0;
    for (int64_t i = 0; i < L; ++i) d += (a[i] != b[i]);
    return d;
}

/* Two-row unit-cost DP over the shorter string: src/distance.cpp:78-95.
 * `row` holds 2*(min(m,n)+1) ints. */
int32_t or_levenshtein(const uint8_t *a, int64_t m, const uint8_t *b, int64_t n, int32_t *row) {
    if (n > m) {
        const uint8_t *t = a; a = b; b = t;
        int64_t u = m; m = n; n = u;
    }
    if (n == 0) return (int32_t)m;
    int32_t *prev = row, *cur = row + (n + 1);
    for (int64_t j = 0; j <= n; ++j) prev[j] = (int32_t)j;
    for (int64_t i = 1; i <= m; ++i) {
        cur[0] = (int32_t)i;
        for (int64_t j = 1; j <= n; ++j) {
            int32_t cost = (a[i - 1] == b[j - 1]) ? 0 : 1;
            int32_t v = prev[j] + 1;
            if (cur[j - 1] + 1 < v) v = cur[j - 1] + 1;
            if (prev[j - 1] + cost < v) v = prev[j - 1] + cost;
            cur[j] = v;
        }
        int32_t *t = prev; prev = cur; cur = t;
    }
    return prev[n];
}

/* ----------------------------------------------------------- dense matrices -------- */
/* Row-parallel drivers.  The reference hands rows to std::thread workers from an atomic
 * counter (gapblock.cpp:105-131, pairwise.cpp:298-332, distance.cpp:36-62); here rows are
 * split into contiguous blocks per pthread -- the result does not depend on the split. */

typedef struct {
    int kind; /* 0 gapblock, 1 gotoh, 2 hamming, 3 levenshtein */
    const uint8_t *qd; const int64_t *qo; int64_t N;
    const uint8_t *rd; const int64_t *ro; int64_t K;
    const int32_t *table; int A;
    int32_t go, ge; int local; int dist;
    const int32_t *prior; uint32_t prior_width;
    const int64_t *q_self; const int64_t *r_self;
    int32_t *out;
    int64_t row0, row1;
    int status; /* 0 ok, 2 overflow */
    int64_t max_len;
} job_t;

static void *run_rows(void *arg) {
    job_t *j = (job_t *)arg;
    size_t scratch_n = (size_t)(j->max_len + 2) * 6;
    int64_t *scratch = (int64_t *)malloc(scratch_n * sizeof(int64_t));
    int32_t *iscratch = (int32_t *)scratch;
    const size_t W1 = (size_t)j->prior_width + 1;
    for (int64_t i = j->row0; i < j->row1; ++i) {
        const uint8_t *q = j->qd + j->qo[i];
        int64_t m = j->qo[i + 1] - j->qo[i];
        for (int64_t k = 0; k < j->K; ++k) {
            const uint8_t *r = j->rd + j->ro[k];
            int64_t n = j->ro[k + 1] - j->ro[k];
            int32_t v = 0;
            if (j->kind == 0) {
                uint32_t M = (uint32_t)(m > n ? m : n), d = (uint32_t)(m > n ? m - n : n - m);
                const int32_t *prow = j->prior ? j->prior + ((size_t)M * W1 + d) * W1 : NULL;
                v = or_gapblock_cell(q, (uint32_t)m, r, (uint32_t)n, j->table, j->A, j->go,
                                     j->ge, prow, iscratch);
            } else if (j->kind == 1) {
                int64_t s = or_gotoh_score(q, m, r, n, j->table, j->A, j->local, j->go, j->ge,
                                           scratch);
                int64_t x = j->dist ? (j->q_self[i] + j->r_self[k] - 2 * s) : s;
                if (x < INT32_MIN || x > INT32_MAX) {
                    j->status = 2;
                    free(scratch);
                    return NULL;
                }
                v = (int32_t)x;
            } else if (j->kind == 2) {
                v = or_hamming(q, r, m);
            } else {
                v = or_levenshtein(q, m, r, n, iscratch);
            }
            j->out[i * j->K + k] = v;
        }
    }
    free(scratch);
    return NULL;
}

static int run_matrix(job_t *proto, int threads) {
    if (proto->N == 0 || proto->K == 0) return 0;
    int64_t mx = 0;
    for (int64_t i = 0; i < proto->N; ++i) {
        int64_t l = proto->qo[i + 1] - proto->qo[i];
        if (l > mx) mx = l;
    }
    for (int64_t k = 0; k < proto->K; ++k) {
        int64_t l = proto->ro[k + 1] - proto->ro[k];
        if (l > mx) mx = l;
    }
    proto->max_len = mx;
    if (threads < 1) threads = 1;
    if (threads > proto->N) threads = (int)proto->N;
    job_t *jobs = (job_t *)calloc((size_t)threads, sizeof(job_t));
    pthread_t *tids = (pthread_t *)calloc((size_t)threads, sizeof(pthread_t));
    int64_t per = (proto->N + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        jobs[t] = *proto;
        jobs[t].row0 = t * per;
        jobs[t].row1 = (t + 1) * per < proto->N ? (t + 1) * per : proto->N;
        pthread_create(&tids[t], NULL, run_rows, &jobs[t]);
    }
    int status = 0;
    for (int t = 0; t < threads; ++t) {
        pthread_join(tids[t], NULL);
        if (jobs[t].status && !status) status = jobs[t].status;
    }
    free(jobs);
    free(tids);
    return status;
}

/* Dense gap-block matrix over ENCODED sequences (src/gapblock.cpp:66-133).  `pen` is the
 * A*A penalty table; `prior` is the [m][d][i] cube of (prior_width+1)^3 entries or NULL. */
int or_gapblock_matrix(const uint8_t *qd, const int64_t *qo, int64_t N, const uint8_t *rd,
                       const int64_t *ro, int64_t K, const int32_t *pen, int A, int32_t go,
                       int32_t ge, const int32_t *prior, uint32_t prior_width, int32_t *out,
                       int threads) {
    job_t j;
    memset(&j, 0, sizeof j);
    j.kind = 0; j.qd = qd; j.qo = qo; j.N = N; j.rd = rd; j.ro = ro; j.K = K;
    j.table = pen; j.A = A; j.go = go; j.ge = ge; j.prior = prior;
    j.prior_width = prior_width; j.out = out;
    return run_matrix(&j, threads);
}

/* Dense Gotoh score / Gram-distance matrix over ENCODED sequences
 * (src/pairwise.cpp:273-334).  Returns 0, or 2 when a value does not fit int32
 * (the reference's std::overflow_error from narrow(), :42-49). */
int or_align_matrix(const uint8_t *qd, const int64_t *qo, int64_t N, const uint8_t *rd,
                    const int64_t *ro, int64_t K, const int32_t *sim, int A, int local,
                    int32_t go, int32_t ge, int dist, int32_t *out, int threads) {
    if (N == 0 || K == 0) return 0;
    int64_t *q_self = NULL, *r_self = NULL;
    if (dist) {
        int64_t mx = 0;
        for (int64_t i = 0; i < N; ++i) if (qo[i + 1] - qo[i] > mx) mx = qo[i + 1] - qo[i];
        for (int64_t k = 0; k < K; ++k) if (ro[k + 1] - ro[k] > mx) mx = ro[k + 1] - ro[k];
        int64_t *scratch = (int64_t *)malloc((size_t)(mx + 2) * 6 * sizeof(int64_t));
        q_self = (int64_t *)malloc((size_t)N * sizeof(int64_t));
        r_self = (int64_t *)malloc((size_t)K * sizeof(int64_t));
        for (int64_t i = 0; i < N; ++i) {
            int64_t m = qo[i + 1] - qo[i];
            q_self[i] = or_gotoh_score(qd + qo[i], m, qd + qo[i], m, sim, A, local, go, ge, scratch);
        }
        for (int64_t k = 0; k < K; ++k) {
            int64_t n = ro[k + 1] - ro[k];
            r_self[k] = or_gotoh_score(rd + ro[k], n, rd + ro[k], n, sim, A, local, go, ge, scratch);
        }
        free(scratch);
    }
    job_t j;
    memset(&j, 0, sizeof j);
    j.kind = 1; j.qd = qd; j.qo = qo; j.N = N; j.rd = rd; j.ro = ro; j.K = K;
    j.table = sim; j.A = A; j.go = go; j.ge = ge; j.local = local; j.dist = dist;
    j.q_self = q_self; j.r_self = r_self; j.out = out;
    int st = run_matrix(&j, threads);
    free(q_self);
    free(r_self);
    return st;
}

/* Dense Hamming matrix over RAW bytes (src/distance.cpp:97-102); the caller has already
 * checked that every pair has equal length. */
int or_hamming_matrix(const uint8_t *ad, const int64_t *ao, int64_t N, const uint8_t *bd,
                      const int64_t *bo, int64_t K, int32_t *out, int threads) {
    job_t j;
    memset(&j, 0, sizeof j);
    j.kind = 2; j.qd = ad; j.qo = ao; j.N = N; j.rd = bd; j.ro = bo; j.K = K; j.out = out;
    return run_matrix(&j, threads);
}

/* Dense Levenshtein matrix over RAW bytes (src/distance.cpp:104-109). */
int or_levenshtein_matrix(const uint8_t *ad, const int64_t *ao, int64_t N, const uint8_t *bd,
                          const int64_t *bo, int64_t K, int32_t *out, int threads) {
    job_t j;
    memset(&j, 0, sizeof j);
    j.kind = 3; j.qd = ad; j.qo = ao; j.N = N; j.rd = bd; j.ro = bo; j.K = K; j.out = out;
    return run_matrix(&j, threads);
}
