/*
 * tbo.h -- CPU oracle for the TEEbench equi-join hot path (TEST INFRASTRUCTURE).
 *
 * This is a plain-C restatement of the reference's algorithms, used ONLY by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the
 * checker.  Nothing in the product (tee-bench_b200/, include/) links or calls
 * it.  Every function cites the reference file:line it restates.
 *
 * Parity pin: tests/golden/ holds vectors produced by the reference's own
 * sources (compiled by oracle/Makefile into oracle/_ref/), and the tests check
 * this restatement against them bit for bit (generators and join results).
 */
#ifndef TBO_H
#define TBO_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as `struct row_t` (Include/data-types.h:44-47). */
typedef struct tbo_row { uint32_t key; uint32_t payload; } tbo_row;

/* ---- generators (App/Lib/generator.cpp, App/Lib/genzipf.c) ---- */
void tbo_seed(unsigned int seed);
void tbo_gen_pk(tbo_row *rows, uint64_t n);
void tbo_gen_fk(tbo_row *rows, uint64_t n, int64_t maxid);
void tbo_gen_fk_sel(tbo_row *rows, uint64_t n, int64_t maxid);
void tbo_gen_zipf(tbo_row *rows, uint64_t n, uint32_t alphabet, double zipf);
/* harness payload policy: kind 0 = R (i * 2654435761), kind 1 = S (row index) */
void tbo_fill_payloads(tbo_row *rows, uint64_t n, int kind);

/* ---- the join (Joins/radix_join.c RHO, single-threaded restatement) ---- */
int64_t tbo_rho(const tbo_row *R, uint64_t nR, const tbo_row *S, uint64_t nS,
                int radix_bits, int passes, uint32_t *rows_out, uint64_t cap);
/* histogram join variant (Joins/radix_join.c:374-440, RHT) */
int64_t tbo_rht(const tbo_row *R, uint64_t nR, const tbo_row *S, uint64_t nS,
                int radix_bits, int passes, uint32_t *rows_out, uint64_t cap);
/* final radix partition sizes: hist[f], f = (p1 << b2) | p2 with
 * p1 = key & (2^b1 - 1), p2 = (key >> b1) & (2^b2 - 1), b1 = bits / passes. */
void tbo_radix_hist(const tbo_row *rows, uint64_t n, int radix_bits, int passes,
                    uint64_t *hist);

/* ---- size-independent digests ---- */
uint64_t tbo_row_hash(uint32_t key, uint32_t rp, uint32_t sp);
uint64_t tbo_rows_checksum(const uint32_t *rows3, uint64_t n);
/* Multi-threaded equi-join count + row checksum by direct key addressing
 * (definition of the equi-join; used at sizes where tbo_rho is too slow). */
int tbo_join_direct(const tbo_row *R, uint64_t nR, const tbo_row *S, uint64_t nS,
                    int nthreads, int64_t *count, uint64_t *checksum);

/* ---- learned partitioner model: MLP 1->H->H->1, tanh, f64 reference ---- */
/* params layout (float): W1[H], b1[H], W2[H*H] (row-major out x in), b2[H],
 * W3[H], b3[1].  Returns mean squared error; grads (same layout) are the
 * gradient of the MSE over the n samples. */
double tbo_mlp_loss_grad(int H, const float *params, const float *x,
                         const float *y, uint64_t n, double *grads);
void tbo_mlp_forward(int H, const float *params, const float *x, uint64_t n,
                     double *out);

#ifdef __cplusplus
}
#endif
#endif
