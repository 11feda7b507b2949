/*
 * tbo.c -- CPU oracle for the TEEbench equi-join hot path (TEST INFRASTRUCTURE).
 *
 * Restates, in plain C, the reference's generators and its RHO/RHT radix join
 * so that tests can check the CUDA path against the reference algorithm on the
 * same seeded inputs.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg use this file; the product never links it.
 *
 * Citations are to the reference project (agora-ecosystem/tee-bench).
 */
#define _GNU_SOURCE
#include "tbo.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* generators                                                                */
/* ------------------------------------------------------------------------ */

/* App/Lib/generator.cpp:22  RAND_RANGE(N) = rand() / (RAND_MAX + 1) * N */
static double rand_range(double n) {
    return (double)rand() / ((double)RAND_MAX + 1) * n;
}

/* App/Lib/generator.cpp:76-82 seed_generator -> srand(seed) (glibc rand) */
void tbo_seed(unsigned int seed) { srand(seed); }

/* App/Lib/generator.cpp:101-111 knuth_shuffle: for i = n-1 .. 1, swap the KEY
 * of i with the key of j = (int64)RAND_RANGE(i), j in [0, i). Payloads stay. */
static void knuth_shuffle(tbo_row *rows, uint64_t n) {
    if (n < 2) return;
    for (uint64_t i = n - 1; i > 0; i--) {
        int64_t j = (int64_t)rand_range((double)i);
        uint32_t tmp = rows[i].key;
        rows[i].key = rows[j].key;
        rows[j].key = tmp;
    }
}

/* App/Lib/generator.cpp:144-155 random_unique_gen: keys 1..n, shuffled. */
static void random_unique_gen(tbo_row *rows, uint64_t n) {
    for (uint64_t i = 0; i < n; i++) rows[i].key = (uint32_t)(i + 1);
    knuth_shuffle(rows, n);
}

/* App/Lib/generator.cpp:157-171 random_unique_gen_maxid: jump is the INTEGER
 * quotient maxid / n (uint32 / uint64), ids start at 1 (0 if maxid == 0). */
static void random_unique_gen_maxid(tbo_row *rows, uint64_t n, uint32_t maxid) {
    double jump = (double)((uint64_t)maxid / n);
    double id = maxid == 0 ? 0 : 1;
    for (uint32_t i = 0; i < n; i++) {
        rows[i].key = (uint32_t)id;
        id += jump;
    }
    knuth_shuffle(rows, n);
}

/* App/Lib/generator.cpp:353-379 create_relation_pk */
void tbo_gen_pk(tbo_row *rows, uint64_t n) { random_unique_gen(rows, n); }

/* App/Lib/generator.cpp:475-514 create_relation_fk: n / maxid shuffled copies
 * of 1..maxid, then a shuffled block of keys 1..(n % maxid). */
void tbo_gen_fk(tbo_row *rows, uint64_t n, int64_t maxid) {
    int64_t iters = (int64_t)n / maxid;
    for (int64_t i = 0; i < iters; i++) random_unique_gen(rows + maxid * i, (uint64_t)maxid);
    int64_t rem = (int64_t)n % maxid;
    if (rem > 0) random_unique_gen(rows + maxid * iters, (uint64_t)rem);
}

/* App/Lib/generator.cpp:516-555 create_relation_fk_sel */
void tbo_gen_fk_sel(tbo_row *rows, uint64_t n, int64_t maxid) {
    int64_t iters = maxid != 0 ? (int64_t)n / maxid : 0;
    for (int64_t i = 0; i < iters; i++)
        random_unique_gen_maxid(rows + maxid * i, (uint64_t)maxid, (uint32_t)maxid);
    int64_t rem = maxid != 0 ? (int64_t)n % maxid : (int64_t)n;
    if (rem > 0) random_unique_gen_maxid(rows + maxid * iters, (uint64_t)rem, (uint32_t)maxid);
}

/* App/Lib/genzipf.c:28-53 gen_alphabet.  The swap index is computed in 32-bit
 * unsigned arithmetic, (unsigned)i * rand() / RAND_MAX, whose product wraps;
 * k therefore lands in {0, 1, 2} and the alphabet stays nearly 1..size. */
static uint32_t *gen_alphabet(uint32_t size) {
    uint32_t *a = (uint32_t *)malloc((size_t)size * sizeof(uint32_t));
    for (uint32_t i = 0; i < size; i++) a[i] = i + 1;
    for (uint32_t i = size - 1; i > 0; i--) {
        uint32_t k = (uint32_t)i * (uint32_t)rand() / (uint32_t)RAND_MAX;
        uint32_t t = a[i];
        a[i] = a[k];
        a[k] = t;
    }
    return a;
}

/* App/Lib/genzipf.c:60-92 gen_zipf_lut: normalised running sum of i^-z. */
static double *gen_zipf_lut(double z, uint32_t size) {
    double *lut = (double *)malloc((size_t)size * sizeof(double));
    double scale = 0.0;
    for (uint32_t i = 1; i <= size; i++) scale += 1.0 / pow((double)i, z);
    double sum = 0.0;
    for (uint32_t i = 1; i <= size; i++) {
        sum += 1.0 / pow((double)i, z);
        lut[i - 1] = sum / scale;
    }
    return lut;
}

/* App/Lib/genzipf.c:97-158 gen_zipf (via generator.cpp:639-662): r = rand() /
 * RAND_MAX, binary search for the first lut entry >= r, key = alphabet[pos]. */
void tbo_gen_zipf(tbo_row *rows, uint64_t n, uint32_t alphabet, double zipf) {
    if (alphabet == 0) return;
    uint32_t *a = gen_alphabet(alphabet);
    double *lut = gen_zipf_lut(zipf, alphabet);
    for (uint32_t i = 0; i < (uint32_t)n; i++) {
        double r = ((double)rand()) / RAND_MAX;
        uint32_t pos;
        if (lut[0] >= r) {
            pos = 0;
        } else {
            uint32_t left = 0, right = alphabet - 1;
            while (right - left > 1) {
                uint32_t m = (left + right) / 2;
                if (lut[m] < r) left = m;
                else right = m;
            }
            pos = right;
        }
        rows[i].key = a[pos];
    }
    free(lut);
    free(a);
}

/* The reference never writes payloads (generator.cpp:144-155 sets keys only);
 * the harness writes them so materialised rows are checkable. */
void tbo_fill_payloads(tbo_row *rows, uint64_t n, int kind) {
    for (uint64_t i = 0; i < n; i++)
        rows[i].payload = kind == 0 ? (uint32_t)(i * 2654435761u) : (uint32_t)i;
}

/* ------------------------------------------------------------------------ */
/* radix join                                                                */
/* ------------------------------------------------------------------------ */

/* Joins/radix_join.c:34-43 NEXT_POW_2 on a 32-bit value */
static uint32_t next_pow2_u32(uint32_t v) {
    v--;
    v |= v >> 1; v |= v >> 2; v |= v >> 4; v |= v >> 8; v |= v >> 16;
    v++;
    return v;
}

typedef struct emit_t {
    uint32_t *out;
    uint64_t cap;
    uint64_t n;
} emit_t;

static void emit(emit_t *e, uint32_t k, uint32_t rp, uint32_t sp) {
    if (e->out && e->n < e->cap) {
        e->out[3 * e->n + 0] = k;
        e->out[3 * e->n + 1] = rp;
        e->out[3 * e->n + 2] = sp;
    }
    e->n++;
}

/* Joins/radix_join.c:187-244 bucket_chaining_join.  N = next_pow2(|R_p|),
 * bucket index = (key & ((N-1) << bits)) >> bits (HASH_BIT_MODULO, :21),
 * 1-based chains built in input order, probe walks the chain. */
static int64_t bucket_chaining_join(const tbo_row *R, uint64_t nR, const tbo_row *S,
                                    uint64_t nS, int bits, emit_t *e) {
    uint32_t N = next_pow2_u32((uint32_t)nR);
    const uint32_t MASK = (N - 1) << bits;
    int *next = (int *)malloc(sizeof(int) * nR);
    int *bucket = (int *)calloc(N, sizeof(int));
    for (uint32_t i = 0; i < nR;) {
        uint32_t idx = (R[i].key & MASK) >> bits;
        next[i] = bucket[idx];
        bucket[idx] = (int)++i;
    }
    int64_t matches = 0;
    for (uint64_t i = 0; i < nS; i++) {
        uint32_t idx = (S[i].key & MASK) >> bits;
        for (int hit = bucket[idx]; hit > 0; hit = next[hit - 1]) {
            if (S[i].key == R[hit - 1].key) {
                matches++;
                emit(e, S[i].key, R[hit - 1].payload, S[i].payload);
            }
        }
    }
    free(bucket);
    free(next);
    return matches;
}

/* Joins/radix_join.c:355-365 get_hist_size */
static uint32_t get_hist_size(uint32_t n) {
    n = next_pow2_u32(n);
    n >>= 2;
    if (n < 4) n = 4;
    return n;
}

/* Joins/radix_join.c:374-440 histogram_join: bucket counts, prefix sum,
 * reorder R_p by bucket, probe scans the bucket's contiguous range. */
static int64_t histogram_join(const tbo_row *R, uint64_t nR, const tbo_row *S,
                              uint64_t nS, int bits, emit_t *e) {
    uint32_t Nhist = get_hist_size((uint32_t)nR);
    const uint32_t MASK = (Nhist - 1) << bits;
    int32_t *hist = (int32_t *)calloc(Nhist + 2, sizeof(int32_t));
    tbo_row *tmp = (tbo_row *)malloc(sizeof(tbo_row) * (nR ? nR : 1));
    for (uint32_t i = 0; i < nR; i++) hist[((R[i].key & MASK) >> bits) + 2]++;
    for (uint32_t i = 2, sum = 0; i <= Nhist + 1; i++) {
        sum += hist[i];
        hist[i] = (int32_t)sum;
    }
    for (uint32_t i = 0; i < nR; i++) {
        uint32_t idx = ((R[i].key & MASK) >> bits) + 1;
        tmp[hist[idx]] = R[i];
        hist[idx]++;
    }
    int64_t match = 0;
    for (uint64_t i = 0; i < nS; i++) {
        uint32_t idx = (S[i].key & MASK) >> bits;
        for (int j = hist[idx], end = hist[idx + 1]; j < end; j++) {
            if (S[i].key == tmp[j].key) {
                match++;
                emit(e, S[i].key, tmp[j].payload, S[i].payload);
            }
        }
    }
    free(tmp);
    free(hist);
    return match;
}

typedef int64_t (*join_fn)(const tbo_row *, uint64_t, const tbo_row *, uint64_t, int,
                           emit_t *);

/* One stable radix scatter of rows[0..n) by digit (key >> shift) & (F-1):
 * histogram, exclusive prefix, scatter (radix_join.c:525-562 radix_cluster,
 * and :630-703 parallel_radix_partition with one thread, no padding). */
static void radix_scatter(const tbo_row *in, tbo_row *out, uint64_t n, int shift, int D,
                          uint64_t *hist /* F entries, zeroed by caller */) {
    const uint32_t F = 1u << D, M = F - 1;
    for (uint64_t i = 0; i < n; i++) hist[(in[i].key >> shift) & M]++;
    uint64_t *dst = (uint64_t *)malloc(sizeof(uint64_t) * F);
    uint64_t off = 0;
    for (uint32_t d = 0; d < F; d++) {
        dst[d] = off;
        off += hist[d];
    }
    for (uint64_t i = 0; i < n; i++) out[dst[(in[i].key >> shift) & M]++] = in[i];
    free(dst);
}

/* Joins/radix_join.c:840-1223 prj_thread with one thread: pass 1 over bits
 * [0, b1), pass 2 over bits [b1, bits) inside each pass-1 partition pair with
 * both sides non-empty (:951-997, serial_radix_partition :573-619), then the
 * join function on every final pair with both sides non-empty. */
static int64_t radix_join(const tbo_row *R, uint64_t nR, const tbo_row *S, uint64_t nS,
                          int bits, int passes, join_fn jf, uint32_t *out, uint64_t cap) {
    emit_t e = {out, cap, 0};
    if (nR == 0 || nS == 0) return 0;
    const int b1 = bits / passes, b2 = bits - b1;
    const uint32_t F1 = 1u << b1;
    tbo_row *tR = (tbo_row *)malloc(sizeof(tbo_row) * nR);
    tbo_row *tS = (tbo_row *)malloc(sizeof(tbo_row) * nS);
    uint64_t *hR = (uint64_t *)calloc(F1, sizeof(uint64_t));
    uint64_t *hS = (uint64_t *)calloc(F1, sizeof(uint64_t));
    radix_scatter(R, tR, nR, 0, b1, hR);
    radix_scatter(S, tS, nS, 0, b1, hS);
    int64_t matches = 0;
    uint64_t oR = 0, oS = 0;
    if (passes == 1) {
        for (uint32_t p = 0; p < F1; p++) {
            if (hR[p] > 0 && hS[p] > 0) matches += jf(tR + oR, hR[p], tS + oS, hS[p], bits, &e);
            oR += hR[p];
            oS += hS[p];
        }
    } else {
        const uint32_t F2 = 1u << b2;
        tbo_row *uR = (tbo_row *)malloc(sizeof(tbo_row) * nR);
        tbo_row *uS = (tbo_row *)malloc(sizeof(tbo_row) * nS);
        uint64_t *gR = (uint64_t *)malloc(sizeof(uint64_t) * F2);
        uint64_t *gS = (uint64_t *)malloc(sizeof(uint64_t) * F2);
        for (uint32_t p = 0; p < F1; p++) {
            if (hR[p] > 0 && hS[p] > 0) {
                memset(gR, 0, sizeof(uint64_t) * F2);
                memset(gS, 0, sizeof(uint64_t) * F2);
                radix_scatter(tR + oR, uR + oR, hR[p], b1, b2, gR);
                radix_scatter(tS + oS, uS + oS, hS[p], b1, b2, gS);
                uint64_t qR = oR, qS = oS;
                for (uint32_t q = 0; q < F2; q++) {
                    if (gR[q] > 0 && gS[q] > 0)
                        matches += jf(uR + qR, gR[q], uS + qS, gS[q], bits, &e);
                    qR += gR[q];
                    qS += gS[q];
                }
            }
            oR += hR[p];
            oS += hS[p];
        }
        free(uR); free(uS); free(gR); free(gS);
    }
    free(tR); free(tS); free(hR); free(hS);
    return matches;
}

int64_t tbo_rho(const tbo_row *R, uint64_t nR, const tbo_row *S, uint64_t nS, int radix_bits,
                int passes, uint32_t *rows_out, uint64_t cap) {
    return radix_join(R, nR, S, nS, radix_bits, passes, bucket_chaining_join, rows_out, cap);
}

int64_t tbo_rht(const tbo_row *R, uint64_t nR, const tbo_row *S, uint64_t nS, int radix_bits,
                int passes, uint32_t *rows_out, uint64_t cap) {
    return radix_join(R, nR, S, nS, radix_bits, passes, histogram_join, rows_out, cap);
}

void tbo_radix_hist(const tbo_row *rows, uint64_t n, int radix_bits, int passes,
                    uint64_t *hist) {
    const int b1 = radix_bits / passes, b2 = radix_bits - b1;
    const uint32_t m1 = (1u << b1) - 1, m2 = (1u << b2) - 1;
    memset(hist, 0, sizeof(uint64_t) << radix_bits);
    for (uint64_t i = 0; i < n; i++) {
        uint32_t k = rows[i].key;
        uint32_t f = passes == 1 ? (k & ((1u << radix_bits) - 1))
                                 : (((k & m1) << b2) | ((k >> b1) & m2));
        hist[f]++;
    }
}

/* ------------------------------------------------------------------------ */
/* digests and the large-size checker                                       */
/* ------------------------------------------------------------------------ */

/* splitmix64 finaliser (Steele, Lea, Flood 2014), used as a row mixer. */
static uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

uint64_t tbo_row_hash(uint32_t key, uint32_t rp, uint32_t sp) {
    return mix64((((uint64_t)key << 32) | rp) ^ mix64((uint64_t)sp));
}

uint64_t tbo_rows_checksum(const uint32_t *rows3, uint64_t n) {
    uint64_t s = 0;
    for (uint64_t i = 0; i < n; i++) s += tbo_row_hash(rows3[3 * i], rows3[3 * i + 1], rows3[3 * i + 2]);
    return s;
}

/* Direct addressing: R grouped by key with a counting sort over [0, maxkey]
 * (CSR), then every S row looks up its key's group.  This is the definition
 * of the equi-join {(s.key, r.payload, s.payload) : r.key == s.key}. */
typedef struct direct_ctx {
    const tbo_row *S;
    uint64_t lo, hi;
    const uint64_t *start; /* maxkey + 2 */
    const uint32_t *pay;
    uint32_t maxkey;
    int64_t count;
    uint64_t checksum;
} direct_ctx;

static void *direct_worker(void *arg) {
    direct_ctx *c = (direct_ctx *)arg;
    int64_t cnt = 0;
    uint64_t sum = 0;
    for (uint64_t i = c->lo; i < c->hi; i++) {
        uint32_t k = c->S[i].key;
        if (k > c->maxkey) continue;
        for (uint64_t j = c->start[k]; j < c->start[k + 1]; j++) {
            cnt++;
            sum += tbo_row_hash(k, c->pay[j], c->S[i].payload);
        }
    }
    c->count = cnt;
    c->checksum = sum;
    return NULL;
}

int tbo_join_direct(const tbo_row *R, uint64_t nR, const tbo_row *S, uint64_t nS,
                    int nthreads, int64_t *count, uint64_t *checksum) {
    uint32_t maxkey = 0;
    for (uint64_t i = 0; i < nR; i++)
        if (R[i].key > maxkey) maxkey = R[i].key;
    uint64_t *start = (uint64_t *)calloc((uint64_t)maxkey + 2, sizeof(uint64_t));
    uint32_t *pay = (uint32_t *)malloc(sizeof(uint32_t) * (nR ? nR : 1));
    if (!start || !pay) {
        free(start); free(pay);
        return -1;
    }
    for (uint64_t i = 0; i < nR; i++) start[R[i].key + 1]++;
    for (uint64_t k = 1; k <= (uint64_t)maxkey + 1; k++) start[k] += start[k - 1];
    uint64_t *fill = (uint64_t *)malloc(sizeof(uint64_t) * ((uint64_t)maxkey + 1));
    memcpy(fill, start, sizeof(uint64_t) * ((uint64_t)maxkey + 1));
    for (uint64_t i = 0; i < nR; i++) pay[fill[R[i].key]++] = R[i].payload;
    free(fill);
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    direct_ctx ctx[256];
    for (int t = 0; t < nthreads; t++) {
        ctx[t].S = S;
        ctx[t].lo = nS * (uint64_t)t / (uint64_t)nthreads;
        ctx[t].hi = nS * (uint64_t)(t + 1) / (uint64_t)nthreads;
        ctx[t].start = start;
        ctx[t].pay = pay;
        ctx[t].maxkey = maxkey;
        pthread_create(&th[t], NULL, direct_worker, &ctx[t]);
    }
    int64_t c = 0;
    uint64_t s = 0;
    for (int t = 0; t < nthreads; t++) {
        pthread_join(th[t], NULL);
        c += ctx[t].count;
        s += ctx[t].checksum;
    }
    free(start);
    free(pay);
    *count = c;
    *checksum = s;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* learned-partitioner model reference (float64 forward / backward)          */
/* ------------------------------------------------------------------------ */

void tbo_mlp_forward(int H, const float *p, const float *x, uint64_t n, double *out) {
    const float *W1 = p, *b1 = p + H, *W2 = p + 2 * H, *b2 = W2 + H * H, *W3 = b2 + H,
                *b3 = W3 + H;
    double h1[256], h2[256];
    for (uint64_t s = 0; s < n; s++) {
        for (int i = 0; i < H; i++) h1[i] = tanh((double)W1[i] * x[s] + (double)b1[i]);
        double y = (double)b3[0];
        for (int o = 0; o < H; o++) {
            double z = (double)b2[o];
            for (int i = 0; i < H; i++) z += (double)W2[o * H + i] * h1[i];
            h2[o] = tanh(z);
            y += (double)W3[o] * h2[o];
        }
        out[s] = y;
    }
}

double tbo_mlp_loss_grad(int H, const float *p, const float *x, const float *y, uint64_t n,
                         double *g) {
    const float *W1 = p, *b1 = p + H, *W2 = p + 2 * H, *b2 = W2 + H * H, *W3 = b2 + H,
                *b3 = W3 + H;
    const int P = 3 * H + H * H + H + 1;
    memset(g, 0, sizeof(double) * P);
    double *gW1 = g, *gb1 = g + H, *gW2 = g + 2 * H, *gb2 = gW2 + H * H, *gW3 = gb2 + H,
           *gb3 = gW3 + H;
    double h1[256], h2[256], dz2[256];
    double loss = 0.0;
    for (uint64_t s = 0; s < n; s++) {
        for (int i = 0; i < H; i++) h1[i] = tanh((double)W1[i] * x[s] + (double)b1[i]);
        double out = (double)b3[0];
        for (int o = 0; o < H; o++) {
            double z = (double)b2[o];
            for (int i = 0; i < H; i++) z += (double)W2[o * H + i] * h1[i];
            h2[o] = tanh(z);
            out += (double)W3[o] * h2[o];
        }
        double r = out - (double)y[s];
        loss += r * r;
        double dy = 2.0 * r / (double)n;
        gb3[0] += dy;
        for (int o = 0; o < H; o++) {
            gW3[o] += dy * h2[o];
            dz2[o] = dy * (double)W3[o] * (1.0 - h2[o] * h2[o]);
            gb2[o] += dz2[o];
        }
        for (int i = 0; i < H; i++) {
            double dh1 = 0.0;
            for (int o = 0; o < H; o++) {
                gW2[o * H + i] += dz2[o] * h1[i];
                dh1 += (double)W2[o * H + i] * dz2[o];
            }
            double dz1 = dh1 * (1.0 - h1[i] * h1[i]);
            gW1[i] += dz1 * (double)x[s];
            gb1[i] += dz1;
        }
    }
    return loss / (double)n;
}
