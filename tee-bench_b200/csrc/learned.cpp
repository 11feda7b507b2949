// Host pipeline of LRN, the learned skew-aware join, and the C-ABI entry
// points of its model.
//
//   1. sample 1% of S's keys (seeded) and sort the sample (LSD radix sort);
//   2. list the keys the sample repeats with their sample estimates, and
//      train the MLP on them (log-key feature -> log2(rows) / 32) on the GPU;
//   3. score the candidates with the model (predicted S rows) and keep the
//      largest (up to HEAVY_MAX) as heavy keys;
//   4. fall back to plain radix (RHO) when the keys the model selected hold,
//      by the sample's measure, less than 5% of S: the bypass would not pay
//      for its set-up;
//   5. otherwise build the heavy table, count (and, materialising, collect)
//      R's heavy rows, radix partition R and the non-heavy rows of S (the S
//      histogram joins heavy rows on the spot) and join the partitions.
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
static constexpr unsigned kCandCap = 1u << 20;

struct LearnCounters {
    unsigned ncand;
    unsigned inserted;
    float loss_sum;
    unsigned pad;
    unsigned bins[64];
    unsigned long long mass[64];
};

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
            (e = cudaEventCreateWithFlags(&w.joined, cudaEventDisableTiming)) != cudaSuccess)
            return cuda_error(e, "stream");
    }
    cudaStream_t s2 = w.side;
    double rate = cfg.sample_rate > 0 ? cfg.sample_rate : 0.01;
    uint64_t m = (uint64_t)((double)nS * rate);
    m = std::max<uint64_t>(m, 65536);
    m = std::min<uint64_t>(m, nS);
    const uint64_t tiles = (m + SCATTER_TILE - 1) / SCATTER_TILE + 1;
    const int capR = join_capacity(nR);
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
    ENSURE(w.aux[0], m * 8);                     // sample, sort ping
    ENSURE(w.aux[1], m * 8);                     // sort pong
    ENSURE(w.aux[4], 8192);                      // digit histograms of the sample, then candidate counts
    ENSURE(w.aux[5], 4 * 256 * 8);
    ENSURE(w.aux[2], (size_t)16384 * 8);         // training set x, y
    ENSURE(w.aux[3], (size_t)MLP_PARAMS_PAD * 4 * 2 + sizeof(LearnCounters));
    ENSURE(w.aux[6], (size_t)kCandCap * sizeof(HeavyCand));
    ENSURE(w.aux[7], (size_t)HEAVY_CAP * 4 * 4 + (1 << FILTER_LOG2) / 8);  // keys, cnt, start, cur, filter
    ENSURE(w.status, tiles * SCATTER_FMAX * 8);
#undef ENSURE
    Ctrl *ctrl = w.ctrl.as<Ctrl>();
    float *xs = w.aux[2].as<float>(), *ys = xs + 16384;
    float *params = w.aux[3].as<float>();
    float *grad = params + MLP_PARAMS_PAD;
    LearnCounters *lc = reinterpret_cast<LearnCounters *>(grad + MLP_PARAMS_PAD);
    uint32_t *hkeys = w.aux[7].as<uint32_t>();
    unsigned *hcnt = hkeys + HEAVY_CAP, *hstart = hcnt + HEAVY_CAP, *hcur = hstart + HEAVY_CAP;
    uint32_t *hfilter = hcur + HEAVY_CAP;
    HeavyCand *cand = w.aux[6].as<HeavyCand>();

    // main stream: R's partitioning needs nothing from the model
    if (timing) cudaEventRecord(w.ev[0], st);
    if ((e = cudaMemsetAsync(ctrl, 0, sizeof(Ctrl), st)) != cudaSuccess) return cuda_error(e, "memset");
    if ((e = cudaEventRecord(w.fork, st)) != cudaSuccess) return cuda_error(e, "event");
    if ((rc = part_histogram(0, g, dR, cfg, w, st, nullptr))) return rc;
    if ((rc = part_pass(0, 1, g, dR, w, st, false))) return rc;
    if ((rc = part_pass(0, 2, g, dR, w, st, false))) return rc;

    // side stream: learn the heavy keys meanwhile
    if ((e = cudaStreamWaitEvent(s2, w.fork, 0)) != cudaSuccess) return cuda_error(e, "event");
    if ((e = cudaMemsetAsync(lc, 0, sizeof(LearnCounters), s2)) != cudaSuccess) return cuda_error(e, "memset");
    // 1. sample and sort
    if ((e = launch_sample(dS, nS, w.aux[0].as<Row>(), m, cfg.seed, s2)) != cudaSuccess) return cuda_error(e, "sample");
    if ((e = launch_digit_hist(w.aux[0].as<Row>(), m, w.aux[4].as<uint32_t>(), w.aux[5].as<uint64_t>(), w.nsm, s2)) !=
        cudaSuccess)
        return cuda_error(e, "sample digits");
    uint32_t hh[1024];
    if ((e = cudaMemcpyAsync(hh, w.aux[4].p, sizeof hh, cudaMemcpyDeviceToHost, s2)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s2)) != cudaSuccess)
        return cuda_error(e, "sample digits");
    const Row *sorted = nullptr;
    int npass = 0;
    // ping-pong aux[1] -> aux[0] -> ...: the first pass never writes its input
    if ((rc = lsd_sort(w.aux[0].as<Row>(), m, w.aux[1], w.aux[0], hh, w.aux[5].as<uint64_t>(), 8, w, s2, &sorted,
                       &npass)))
        return rc;
    // 2. candidates (distinct sampled keys) and the frequency model
    if ((e = launch_candidates(sorted, m, (double)nS, cand, &lc->ncand, kCandCap, w.aux[4].as<unsigned>(), s2)) !=
        cudaSuccess)
        return cuda_error(e, "candidates");
    unsigned ncand_raw = 0;
    if ((e = cudaMemcpyAsync(&ncand_raw, &lc->ncand, 4, cudaMemcpyDeviceToHost, s2)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s2)) != cudaSuccess)
        return cuda_error(e, "candidates");
    const unsigned ncand = std::min(ncand_raw, kCandCap);
    const uint32_t T = std::min<uint32_t>(ncand, 16384);
    if ((e = launch_mlp_init(params, cfg.seed, s2)) != cudaSuccess) return cuda_error(e, "mlp init");
    const int steps = cfg.model == TBG_MODEL_MLP && T ? std::min(std::max(cfg.train_steps, 1), 500) : 0;
    if (T) {
        if ((e = launch_freq_points(cand, ncand, xs, ys, T, s2)) != cudaSuccess) return cuda_error(e, "points");
        if (steps && (e = launch_mlp_train(xs, ys, T, params, steps, 0.03f, cfg.seed, s2)) != cudaSuccess)
            return cuda_error(e, "mlp train");
        if ((e = launch_mlp_grad(params, xs, ys, T, grad, &lc->loss_sum, s2)) != cudaSuccess)
            return cuda_error(e, "mlp loss");
    }
    // 3. score: the model (or, for the ablation, the sample) proposes; keys the
    // sample saw once are not scored (they cannot reach the threshold)
    const double tau_min = std::max(64.0, (double)nS / (double)(1 << 20));
    const int use_model = cfg.model == TBG_MODEL_SAMPLE ? 0 : 1;
    const double single = (double)nS / (double)m;
    if ((e = launch_heavy_score(cand, ncand, params, use_model, tau_min, 1.5 * single, lc->bins, lc->mass, s2)) !=
        cudaSuccess)
        return cuda_error(e, "heavy score");
    LearnCounters h;
    if ((e = cudaMemcpyAsync(&h, lc, sizeof h, cudaMemcpyDeviceToHost, s2)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s2)) != cudaSuccess)
        return cuda_error(e, "heavy score");
    run->train_steps = steps;
    run->train_loss = T ? h.loss_sum / (float)T : 0.f;
    // 4. largest bins first while the table has room; the sample measures them
    unsigned taken = 0;
    double heavy_mass = 0;
    int lowest = 64;
    for (int b = 63; b >= 0; b--) {
        if (!h.bins[b]) continue;
        if (taken + h.bins[b] > (unsigned)HEAVY_MAX) break;
        taken += h.bins[b];
        heavy_mass += (double)h.mass[b];
        lowest = b;
    }
    run->predicted_imbalance = lowest < 64 ? std::ldexp(1.0, lowest) / ((double)nS / (double)g.P) : 0.0;
    const bool bypass = taken > 0 && heavy_mass >= kMinHeavyFraction * (double)nS;
    if (dbg)
        fprintf(stderr, "[lrn] m=%llu T=%u ncand=%u taken=%u lowest=%d heavy_mass=%.0f loss=%.3e bypass=%d\n",
                (unsigned long long)m, T, ncand, taken, lowest, heavy_mass, (double)run->train_loss, (int)bypass);
    if (timing) cudaEventRecord(w.ev[5], s2);
    SBypass bp;
    memset(&bp, 0, sizeof bp);
    if (bypass) {
        const float tau = (float)std::ldexp(1.0, lowest);
        if ((e = cudaMemsetAsync(hkeys, 0xFF, HEAVY_CAP * 4, s2)) != cudaSuccess) return cuda_error(e, "memset");
        if ((e = cudaMemsetAsync(hcnt, 0, HEAVY_CAP * 4 * 3 + (1 << FILTER_LOG2) / 8, s2)) != cudaSuccess)
            return cuda_error(e, "memset");
        if ((e = launch_heavy_build(cand, ncand, tau, hkeys, hfilter, &lc->inserted, s2)) != cudaSuccess)
            return cuda_error(e, "heavy build");
        uint32_t *rpay = nullptr;
        if ((e = launch_heavy_r(dR, nR, hkeys, hfilter, hcnt, nullptr, nullptr, nullptr, 0, w.nsm, s2)) !=
            cudaSuccess)
            return cuda_error(e, "heavy R");
        if (mat) {  // heavy R payload lists: at most |R| entries, so no count read-back
            if ((e = w.misc.ensure(std::max<uint64_t>(nR, 1) * 4 + 64)) != cudaSuccess)
                return cuda_error(e, "cudaMalloc");
            rpay = w.misc.as<uint32_t>();
            if ((e = launch_heavy_r(dR, nR, hkeys, hfilter, hcnt, hstart, hcur, rpay, 1, w.nsm, s2)) != cudaSuccess)
                return cuda_error(e, "heavy R");
        }
        if ((e = cudaMemcpyAsync(&ctrl->heavy_keys, &lc->inserted, 4, cudaMemcpyDeviceToDevice, s2)) != cudaSuccess)
            return cuda_error(e, "copy");
        bp.filter = hfilter;
        bp.keys = hkeys;
        bp.cnt = hcnt;
        bp.start = hstart;
        bp.rpay = rpay;
        bp.rows = d_rows;
        bp.cap = d_rows ? cap : 0;
    } else {
        run->used_fallback = 1;  // no heavy mass: S is partitioned whole, as in RHO
    }
    if (timing) cudaEventRecord(w.ev[6], s2);
    // S: histogram (joining heavy rows on the way), passes
    if ((rc = part_histogram(1, g, dS, cfg, w, s2, bypass ? &bp : nullptr))) return rc;
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
    if (e == cudaSuccess) e = launch_mlp_train(dx, dy, (uint32_t)n, dp, steps, lr, seed, 0);
    if (e == cudaSuccess) e = cudaMemcpy(params, dp, MLP_PARAMS * 4, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? TBG_OK : cuda_error(e, "mlp train");
}

float tbg_mlp_feature(uint32_t key) { return key_feature((double)key); }

}  // extern "C"
