// Host pipeline of LRN, the learned skew-aware join, and the C-ABI entry
// points of its model.
//
//   1. sample 1% of S's keys (seeded blocks of 64 rows) and count them: a
//      shared-memory aggregation per CTA, then a global hash table;
//   2. the sample's frequency curve: count-of-counts bins, one training point
//      per bin (rank feature -> log2(count), normalised over the points), and
//      the MLP trained on them on the GPU;
//   3. the decision kernel predicts the S rows of ranks 1 .. HEAVY_MAX from
//      the trained curve: the heavy keys are the sampled keys at the ranks
//      predicted to hold at least tau_min rows, and LRN bypasses when the
//      model predicts those keys to hold at least 5% of S (below that, the
//      bypass would not pay for its set-up and plain radix runs);
//   4. with the bypass: build the heavy table, count (and, materialising,
//      collect) R's heavy rows, radix partition R and the non-heavy rows of S
//      and join the partitions.  The S histogram takes the heavy rows out of
//      S: counting, it counts them per key (matches = S rows x R rows per
//      key); materialising, it sets them aside per chunk and totals their
//      output rows, and k_heavy_emit writes their pairs on the main stream
//      while S's kept rows are partitioned.
// Steps 1-3 run on a second stream while R is partitioned, and the host reads
// the decision back once.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "tbg_internal.h"
#include "tbg_learned.h"
#include "tbg_runtime.h"

namespace tbg {

static constexpr double kMinHeavyFraction = 0.05;

// 0 (default): R's partitioning is queued before the learning stage's
// kernels; 1: after them.  Measured at |R| = 2^26, |S| = 2^29, z = 1: 5.41 -
// 5.49 ms against 5.65 ms.  Queued first, the learning stage ends sooner
// (0.68 against 0.79 - 0.88 ms) but pushes R's partitioning into S's
// bandwidth-bound phase; queued after, R's passes use the bandwidth the
// latency-bound learning kernels leave idle.  A build option for A/B timing.
#ifndef TBG_LRN_LEARN_FIRST
#define TBG_LRN_LEARN_FIRST 0
#endif
static constexpr unsigned kCandCap = 1u << 20;

int run_learned_join(const tbg_config &cfg, const Row *dR, uint64_t nR, const Row *dS, uint64_t nS,
                     tbg_row_out *d_rows, uint64_t cap, Workspace &w, cudaStream_t st, JoinRun *run) {
    const bool timing = cfg.timing != 0;
    const bool mat = cfg.materialize != 0;
    const bool dbg = getenv("TBG_DEBUG") != nullptr;
    if (nS < 65536 || cfg.model == TBG_MODEL_UNIFORM) {  // too small to learn from, or no model
        run->used_fallback = 1;
        return run_radix_join(cfg, dR, nR, dS, nS, d_rows, cap, w, st, run);
    }
    cudaError_t e;
    if (!w.side) {
        // the learning stream gets the highest priority: its small kernels
        // are on the critical path and would otherwise queue behind R's
        // partitioning grids, which fill every SM
        int least = 0, greatest = 0;
        if ((e = cudaDeviceGetStreamPriorityRange(&least, &greatest)) != cudaSuccess ||
            (e = cudaStreamCreateWithPriority(&w.side, cudaStreamNonBlocking, greatest)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&w.fork, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&w.joined, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&w.table, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&w.emit, cudaEventDisableTiming)) != cudaSuccess)
            return cuda_error(e, "stream");
    }
    cudaStream_t s2 = w.side;
    // the sample: nb whole blocks of SAMPLE_BLOCK rows, one per stride of S
    const double rate = cfg.sample_rate > 0 ? cfg.sample_rate : 0.01;
    const uint64_t nfull = nS / SAMPLE_BLOCK;
    uint64_t nb = (uint64_t)((double)nS * rate / SAMPLE_BLOCK);
    nb = std::min<uint64_t>(std::max<uint64_t>(nb, 65536 / SAMPLE_BLOCK), nfull);
    const uint64_t stride = nfull / nb;
    const uint64_t m = nb * SAMPLE_BLOCK;
    uint32_t tslots = 1u << 16;
    while (tslots < m + m / 2 && tslots < (1u << 24)) tslots <<= 1;
    const int capR = join_capacity(nR, !cfg.materialize);
    const RadixGeom g = radix_geometry(cfg, nR, nS, capR, w);
    run->B = g.B;
    run->passes = g.passes;
    run->P = g.P;
    int rc = ensure_radix_buffers(g, true, w);
    if (rc) return rc;
#define ENSURE(buf, bytes)                                        \
    do {                                                          \
        e = (buf).ensure(bytes);                                  \
        if (e != cudaSuccess) return cuda_error(e, "cudaMalloc"); \
    } while (0)
    ENSURE(w.aux[0], m * 4);                                         // sample keys
    ENSURE(w.aux[1], (size_t)tslots * 8);                            // count table: keys, counts
    ENSURE(w.aux[2], (size_t)CC_BINS * (4 + 8 + 4 + 4 + 4) + (HEAVY_MAX + 2) * 4);  // bins, points, weights, predictions
    ENSURE(w.aux[3], (size_t)MLP_PARAMS_PAD * 4 + sizeof(LrnDecision));
    ENSURE(w.aux[6], (size_t)kCandCap * sizeof(HeavyCand));
    // heavy table: keys, R counts, starts, cursors, inserted count, S counts
    ENSURE(w.aux[7], (size_t)HEAVY_CAP * 4 * 5 + 16);
    ENSURE(w.aux[5], (size_t)g.G[1] * (8 + 8 + 4) + 16);  // materialising: per chunk heavy pairs, bases, rows
#undef ENSURE
    Ctrl *ctrl = w.ctrl.as<Ctrl>();
    // main stream: R's partitioning needs nothing from the model
    auto partition_r = [&]() -> int {
        int r;
        if ((r = part_histogram(0, g, dR, cfg, w, st, nullptr))) return r;
        if ((r = part_pass(0, 1, g, dR, w, st, false))) return r;
        return part_pass(0, 2, g, dR, w, st, false);
    };
    LearnBufs lb;
    lb.keys = w.aux[0].as<uint32_t>();
    lb.table = w.aux[1].as<unsigned long long>();
    lb.tmask = tslots - 1;
    lb.bin_rows = w.aux[2].as<unsigned long long>();
    lb.bin_keys = reinterpret_cast<unsigned *>(lb.bin_rows + CC_BINS);
    lb.xs = reinterpret_cast<float *>(lb.bin_keys + CC_BINS);
    lb.ys = lb.xs + CC_BINS;
    lb.cw = lb.ys + CC_BINS;
    lb.lpred = lb.cw + CC_BINS;
    lb.params = w.aux[3].as<float>();
    lb.dec = reinterpret_cast<LrnDecision *>(lb.params + MLP_PARAMS_PAD);
    lb.cand = w.aux[6].as<HeavyCand>();
    lb.cand_cap = kCandCap;
    lb.err = &ctrl->error;
    uint32_t *hkeys = w.aux[7].as<uint32_t>();
    unsigned *hcnt = hkeys + HEAVY_CAP, *hstart = hcnt + HEAVY_CAP, *hcur = hstart + HEAVY_CAP;
    unsigned *hinserted = hcur + HEAVY_CAP;
    unsigned *hscnt = hinserted + 4;  // S rows per heavy slot (counting joins)
    unsigned long long *hpairs = w.aux[5].as<unsigned long long>();  // materialising, per S chunk
    unsigned long long *hbase = hpairs + g.G[1];
    uint32_t *hkeptc = reinterpret_cast<uint32_t *>(hbase + g.G[1]);

    if (timing) cudaEventRecord(w.ev[0], st);
    if ((e = cudaMemsetAsync(ctrl, 0, sizeof(Ctrl), st)) != cudaSuccess) return cuda_error(e, "memset");
    if ((e = cudaEventRecord(w.fork, st)) != cudaSuccess) return cuda_error(e, "event");
    if (!TBG_LRN_LEARN_FIRST && (rc = partition_r()))
        return rc;

    // side stream: learn the heavy keys (on the high-priority stream, while
    // R is partitioned)
    if ((e = cudaStreamWaitEvent(s2, w.fork, 0)) != cudaSuccess) return cuda_error(e, "event");
    if ((e = cudaMemsetAsync(lb.table, 0xFF, (size_t)tslots * 8, s2)) != cudaSuccess ||
        (e = cudaMemsetAsync(lb.bin_rows, 0, (size_t)CC_BINS * 12, s2)) != cudaSuccess ||
        (e = cudaMemsetAsync(lb.dec, 0, sizeof(LrnDecision), s2)) != cudaSuccess ||
        (e = cudaMemsetAsync(hkeys, 0xFF, HEAVY_CAP * 4, s2)) != cudaSuccess ||
        (e = cudaMemsetAsync(hcnt, 0, HEAVY_CAP * 4 * 4 + 16, s2)) != cudaSuccess)
        return cuda_error(e, "memset");
    const int steps = cfg.model == TBG_MODEL_MLP ? std::min(std::max(cfg.train_steps, 1), 500) : 0;
    const int use_model = cfg.model == TBG_MODEL_SAMPLE ? 0 : 1;
    // a key must be predicted to hold at least tau_min S rows to be heavy
    const double tau_min = std::max(64.0, (double)nS / (double)(1 << 20));
    if ((e = launch_sample_blocks(dS, nS, lb.keys, nb, stride, cfg.seed, s2)) != cudaSuccess ||
        (e = launch_count_keys(lb, m, s2)) != cudaSuccess || (e = launch_count_stats(lb, s2)) != cudaSuccess ||
        (e = launch_rank_points(lb, s2)) != cudaSuccess || (e = launch_mlp_init(lb.params, cfg.seed, s2)) != cudaSuccess ||
        (steps && (e = launch_mlp_train(lb.xs, lb.ys, lb.cw, &lb.dec->npoints, 0, lb.params, steps, 0.03f, cfg.seed, s2)) !=
                      cudaSuccess) ||
        (e = launch_decide(lb, use_model, (double)nS, (double)m, tau_min, kMinHeavyFraction, s2)) != cudaSuccess)
        return cuda_error(e, "learning stage");
    LrnDecision *hd = static_cast<LrnDecision *>(w.host_small);
    if ((e = cudaMemcpyAsync(hd, lb.dec, sizeof(LrnDecision), cudaMemcpyDeviceToHost, s2)) != cudaSuccess)
        return cuda_error(e, "learning stage");
    if (TBG_LRN_LEARN_FIRST && (rc = partition_r())) return rc;
    if ((e = cudaStreamSynchronize(s2)) != cudaSuccess) return cuda_error(e, "learning stage");
    const LrnDecision dec = *hd;
    run->train_steps = steps;
    run->train_loss = dec.loss;
    run->predicted_imbalance = dec.next_rows / ((double)nS / (double)g.P);
    run->heavy_pred = dec.pred_mass;
    run->heavy_sampled = dec.sample_mass;
    const bool bypass = dec.bypass != 0;
    if (dbg)
        fprintf(stderr,
                "[lrn] m=%llu slots=%u points=%u cand=%u k*=%u count_min=%u heavy=%u pred_mass=%.0f "
                "sample_mass=%.0f loss=%.3e bypass=%d\n",
                (unsigned long long)m, tslots, dec.npoints, dec.ncand, dec.k_star, dec.count_min, dec.heavy_sample,
                dec.pred_mass, dec.sample_mass, (double)dec.loss, (int)bypass);
    if (timing) cudaEventRecord(w.ev[5], s2);
    SBypass bp;
    memset(&bp, 0, sizeof bp);
    if (bypass) {
        if ((e = launch_heavy_build(lb, hkeys, hinserted, s2)) != cudaSuccess)
            return cuda_error(e, "heavy build");
        if (mat) {
            // the S histogram totals each chunk's heavy output rows: R's rows
            // per heavy key are counted first; their payload lists are built
            // on the main stream meanwhile (after R's passes)
            if ((e = launch_heavy_r(dR, nR, hkeys, hcnt, nullptr, nullptr, nullptr, 0, w.nsm, s2)) !=
                    cudaSuccess ||
                (e = w.misc.ensure(std::max<uint64_t>(nR, 1) * 4 + 64)) != cudaSuccess)
                return cuda_error(e, "heavy R");
            if ((e = cudaEventRecord(w.table, s2)) != cudaSuccess ||
                (e = cudaStreamWaitEvent(st, w.table, 0)) != cudaSuccess)
                return cuda_error(e, "event");
            if ((e = launch_heavy_r(dR, nR, hkeys, hcnt, hstart, hcur, w.misc.as<uint32_t>(), 1, w.nsm, st)) !=
                cudaSuccess)
                return cuda_error(e, "heavy R");
        } else {
            // counting: the S histogram counts S rows per heavy key; R's heavy
            // rows are counted on the main stream meanwhile (after R's passes)
            if ((e = cudaEventRecord(w.table, s2)) != cudaSuccess ||
                (e = cudaStreamWaitEvent(st, w.table, 0)) != cudaSuccess)
                return cuda_error(e, "event");
            if ((e = launch_heavy_r(dR, nR, hkeys, hcnt, nullptr, nullptr, nullptr, 0, w.nsm, st)) !=
                cudaSuccess)
                return cuda_error(e, "heavy R");
        }
        if ((e = cudaMemcpyAsync(&ctrl->heavy_keys, hinserted, 4, cudaMemcpyDeviceToDevice, s2)) != cudaSuccess)
            return cuda_error(e, "copy");
        bp.keys = hkeys;
        bp.cnt = hcnt;
        bp.scnt = hscnt;
        bp.hpairs = hpairs;
        bp.hkept = hkeptc;
    } else {
        run->used_fallback = 1;  // no heavy mass: S is partitioned whole, as in RHO
    }
    if (timing) cudaEventRecord(w.ev[6], s2);
    // S: histogram (heavy rows joined or set aside on the way), passes
    if ((rc = part_histogram(1, g, dS, cfg, w, s2, bypass ? &bp : nullptr))) return rc;
    if (bypass && mat) {
        // the heavy pairs: output places reserved here, written on the main
        // stream while S's kept rows are partitioned
        HeavyEmitArgs ea;
        ea.hs = w.sc.as<Row>();
        ea.n = g.n[1];
        ea.chunk = g.ch[1];
        ea.G = g.G[1];
        ea.hkept = hkeptc;
        ea.hbase = hbase;
        ea.hkeys = hkeys;
        ea.hcnt = hcnt;
        ea.hstart = hstart;
        ea.rpay = w.misc.as<uint32_t>();
        ea.rows = d_rows;
        ea.cap = d_rows ? cap : 0;
        if ((e = launch_heavy_plan(hpairs, g.G[1], hbase, &ctrl->rows, s2)) != cudaSuccess ||
            (e = cudaEventRecord(w.emit, s2)) != cudaSuccess || (e = cudaStreamWaitEvent(st, w.emit, 0)) != cudaSuccess ||
            (e = launch_heavy_emit(ea, w.nsm, st)) != cudaSuccess)
            return cuda_error(e, "heavy pairs");
    }
    if ((rc = part_pass(1, 1, g, dS, w, s2, bypass))) return rc;
    if ((rc = part_pass(1, 2, g, dS, w, s2, bypass))) return rc;
    if ((e = cudaEventRecord(w.joined, s2)) != cudaSuccess) return cuda_error(e, "event");
    // main stream: both relations partitioned -> items -> build/probe
    if ((e = cudaStreamWaitEvent(st, w.joined, 0)) != cudaSuccess) return cuda_error(e, "event");
    if ((rc = plan_items(g, w, st))) return rc;
    if (timing) {
        cudaEventRecord(w.ev[1], st);
        cudaEventRecord(w.ev[2], st);
        cudaEventRecord(w.ev[3], st);
    }
    rc = radix_join_phase(cfg, d_rows, cap, w, st, run, capR, g.join_grid);
    if (!rc && bypass && !mat && (e = launch_heavy_sum(hcnt, hscnt, &ctrl->matches, st)) != cudaSuccess)
        return cuda_error(e, "heavy matches");
    if (timing) {
        float ms = 0;
        cudaEventSynchronize(w.ev[6]);
        cudaEventElapsedTime(&ms, w.ev[0], w.ev[6]);
        run->ms_learn = ms;
    }
    return rc;
}

}  // namespace tbg

using namespace tbg;

extern "C" {

int tbg_mlp_param_count(void) { return MLP_PARAMS; }

int tbg_mlp_init(float *params, uint64_t seed) {
    if (!params) return set_error(TBG_ERR_ARG, "null params");
    float *d = nullptr;
    cudaError_t e = cudaMalloc(&d, MLP_PARAMS * 4);
    if (e == cudaSuccess) e = launch_mlp_init(d, seed, 0);
    if (e == cudaSuccess) e = cudaMemcpy(params, d, MLP_PARAMS * 4, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? TBG_OK : cuda_error(e, "mlp init");
}

int tbg_mlp_grad(const float *params, const float *x, const float *y, uint64_t n, float *grad, float *loss) {
    if (!params || (n && (!x || !y)) || !grad || !loss || n > 0xFFFFFFFFull) return set_error(TBG_ERR_ARG, "bad arguments");
    float *d = nullptr;
    const size_t bytes = (MLP_PARAMS + 2 * n + MLP_PARAMS + 1) * 4;
    cudaError_t e = cudaMalloc(&d, bytes);
    if (e != cudaSuccess) return cuda_error(e, "cudaMalloc");
    float *dp = d, *dx = d + MLP_PARAMS, *dy = dx + n, *dg = dy + n, *dl = dg + MLP_PARAMS;
    e = cudaMemcpy(dp, params, MLP_PARAMS * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n) e = cudaMemcpy(dx, x, n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && n) e = cudaMemcpy(dy, y, n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_mlp_grad(dp, dx, dy, (uint32_t)n, dg, dl, 0);
    if (e == cudaSuccess) e = cudaMemcpy(grad, dg, MLP_PARAMS * 4, cudaMemcpyDeviceToHost);
    float ls = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&ls, dl, 4, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_error(e, "mlp grad");
    *loss = n ? ls / (float)n : 0.f;
    return TBG_OK;
}

int tbg_mlp_train(float *params, const float *x, const float *y, uint64_t n, int steps, float lr, uint64_t seed) {
    if (!params || !x || !y || n == 0 || n > 0xFFFFFFFFull || steps < 0) return set_error(TBG_ERR_ARG, "bad arguments");
    float *d = nullptr;
    cudaError_t e = cudaMalloc(&d, (MLP_PARAMS + 2 * n) * 4);
    if (e != cudaSuccess) return cuda_error(e, "cudaMalloc");
    float *dp = d, *dx = d + MLP_PARAMS, *dy = dx + n;
    e = cudaMemcpy(dp, params, MLP_PARAMS * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dx, x, n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dy, y, n * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_mlp_train(dx, dy, nullptr, nullptr, (uint32_t)n, dp, steps, lr, seed, 0);
    if (e == cudaSuccess) e = cudaMemcpy(params, dp, MLP_PARAMS * 4, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? TBG_OK : cuda_error(e, "mlp train");
}

float tbg_mlp_feature(uint32_t rank) { return rank_feature((double)rank); }

}  // extern "C"
