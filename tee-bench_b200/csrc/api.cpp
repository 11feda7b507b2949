// Host runtime and C ABI of tee-bench-b200.
//
// The drop-in layer mirrors the reference's join entry points
// (Joins/radix_join.h:20-24, Joins/radix_sortmerge_join.h:4,
// Joins/psm/parallel_sortmerge_join.h:61) and registry (native.cpp:34-46);
// the device layer runs the GPU pipeline on caller buffers.  The per-thread
// task queues and barriers of the reference (Include/task_queue.h,
// Include/barrier.h, Joins/radix_join.c:1237-1396 join_init_run) have no
// counterpart: every phase is one kernel launch on one stream.
#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "tbg_internal.h"
#include "tbg_runtime.h"

namespace tbg {

static std::atomic<uint64_t> g_launches{0};
void count_launch(unsigned n) { g_launches += n; }

// ---------------------------------------------------------------- errors
static thread_local int t_err = TBG_OK;
static thread_local char t_msg[512] = "";
static std::atomic<int> g_errmode{TBG_ERRMODE_EXIT};

int dropin_errmode() { return g_errmode.load(); }

int set_error(int code, const char *fmt, ...) {
    t_err = code;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_msg, sizeof t_msg, fmt, ap);
    va_end(ap);
    return code;
}

int cuda_error(cudaError_t e, const char *what) {
    if (e == cudaErrorMemoryAllocation)
        return set_error(TBG_ERR_OOM, "%s: %s", what, cudaGetErrorString(e));
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return set_error(TBG_ERR_NO_DEVICE, "%s: %s", what, cudaGetErrorString(e));
    return set_error(TBG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// ---------------------------------------------------------------- buffers
cudaError_t DevBuf::ensure(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = bytes + bytes / 8;  // headroom for slightly larger calls
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            p = nullptr;
            return e;
        }
        want = bytes;
    }
    cap = want;
    fresh = true;
    return cudaSuccess;
}

void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
}

static std::mutex g_ws_mu;
static std::map<std::pair<int, cudaStream_t>, Workspace *> g_ws;

Workspace *workspace_for(cudaStream_t st) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    std::lock_guard<std::mutex> g(g_ws_mu);
    auto key = std::make_pair(dev, st);
    auto it = g_ws.find(key);
    if (it != g_ws.end()) return it->second;
    Workspace *w = new Workspace();
    w->device = dev;
    cudaDeviceGetAttribute(&w->nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaMallocHost(&w->host_ctrl, sizeof(Ctrl)) != cudaSuccess) {
        delete w;
        return nullptr;
    }
    for (auto &e : w->ev) cudaEventCreate(&e);
    g_ws[key] = w;
    return w;
}

uint32_t Workspace::next_epoch(cudaStream_t st) {
    if (status.fresh) {
        cudaMemsetAsync(status.p, 0, status.cap, st);
        status.fresh = false;
        epoch = 0;
    }
    if (++epoch > 255) {
        cudaMemsetAsync(status.p, 0, status.cap, st);
        epoch = 1;
    }
    return epoch;
}

static int ceil_log2(uint64_t x) {
    int k = 0;
    while ((1ull << k) < x) k++;
    return k;
}

void choose_radix(const tbg_config &cfg, uint64_t nR, int capR, int *B, int *passes) {
    int b = cfg.radix_bits;
    if (b <= 0) {
        // R partitions of about capR / 2 rows: room for uneven radix buckets
        uint64_t target = (uint64_t)capR / 2;
        b = ceil_log2((nR + target - 1) / target);
        if (b < 1) b = 1;
    }
    if (b > 15) b = 15;  // the histogram keeps 2^bits 32-bit counters in shared memory
    int p = cfg.passes;
    if (p <= 0 || p > 2) p = b <= 8 ? 1 : 2;
    if (p == 1 && b > 8) p = 2;
    *B = b;
    *passes = p;
}

// Records a timing event when cfg.timing is on.
static void mark(Workspace &w, bool timing, int i, cudaStream_t st) {
    if (timing) cudaEventRecord(w.ev[i], st);
}

// The radix-partitioned join: RHO (layout 0) and RHT (layout 1).
int run_radix_join(const tbg_config &cfg, const Row *dR, uint64_t nR, const Row *dS, uint64_t nS,
                   tbg_row_out *d_rows, uint64_t cap, Workspace &w, cudaStream_t st,
                   JoinRun *run) {
    const bool timing = cfg.timing != 0;
    const int capR = JOIN_CAPR_DEFAULT;
    int B, passes;
    choose_radix(cfg, nR, capR, &B, &passes);
    const int b1 = B / passes, b2 = B - b1;
    const uint64_t P = 1ull << B;
    const uint64_t F1 = 1ull << b1;
    run->B = B;
    run->passes = passes;
    run->P = P;

    const int join_per_sm = join_ctas_per_sm(capR);
    const int join_grid = w.nsm * join_per_sm;
    uint64_t capS = 0;
    if (cfg.skew_split) {
        capS = nS / ((uint64_t)join_grid * 4);
        if (capS < 65536) capS = 65536;
    }
    const uint64_t item_cap = nR / capR + (capS ? nS / capS : 0) + 2 * P + 16;
    const uint64_t tiles_max = (std::max(nR, nS) + SCATTER_TILE - 1) / SCATTER_TILE + F1 + 1;

    cudaError_t e;
#define ENSURE(buf, bytes)                                      \
    do {                                                        \
        e = (buf).ensure(bytes);                                \
        if (e != cudaSuccess) return cuda_error(e, "cudaMalloc"); \
    } while (0)
    ENSURE(w.ctrl, sizeof(Ctrl));
    ENSURE(w.histR, P * 4);
    ENSURE(w.histS, P * 4);
    ENSURE(w.baseR, (P + 1) * 8);
    ENSURE(w.baseS, (P + 1) * 8);
    ENSURE(w.segStartR, (F1 + 1) * 8);
    ENSURE(w.segStartS, (F1 + 1) * 8);
    ENSURE(w.segTileR, (F1 + 1) * 4);
    ENSURE(w.segTileS, (F1 + 1) * 4);
    ENSURE(w.status, tiles_max * SCATTER_FMAX * 8);
    ENSURE(w.partR, std::max<uint64_t>(nR, 1) * 8);
    ENSURE(w.partS, std::max<uint64_t>(nS, 1) * 8);
    if (passes == 2) {
        ENSURE(w.tmpR, std::max<uint64_t>(nR, 1) * 8);
        ENSURE(w.tmpS, std::max<uint64_t>(nS, 1) * 8);
    }
    ENSURE(w.items, item_cap * sizeof(Item));
#undef ENSURE

    Ctrl *ctrl = w.ctrl.as<Ctrl>();
    mark(w, timing, 0, st);
    if ((e = cudaMemsetAsync(ctrl, 0, sizeof(Ctrl), st)) != cudaSuccess) return cuda_error(e, "memset");
    if ((e = cudaMemsetAsync(w.histR.p, 0, P * 4, st)) != cudaSuccess) return cuda_error(e, "memset");
    if ((e = cudaMemsetAsync(w.histS.p, 0, P * 4, st)) != cudaSuccess) return cuda_error(e, "memset");

    RadixF rf;
    if (passes == 1) {
        rf = RadixF{(uint32_t)(P - 1), 0, 0, 0};
    } else {
        rf = RadixF{(uint32_t)(F1 - 1), (uint32_t)b1, (uint32_t)((1u << b2) - 1), (uint32_t)b2};
    }
    const bool agg = true;
    if ((e = launch_hist(dR, nR, w.histR.as<uint32_t>(), B, rf, agg, w.nsm, st)) != cudaSuccess)
        return cuda_error(e, "hist R");
    if ((e = launch_hist(dS, nS, w.histS.as<uint32_t>(), B, rf, agg, w.nsm, st)) != cudaSuccess)
        return cuda_error(e, "hist S");

    PlanArgs pa;
    pa.r = RelPlan{w.histR.as<uint32_t>(), w.baseR.as<uint64_t>(), w.segStartR.as<uint64_t>(),
                   w.segTileR.as<uint32_t>()};
    pa.s = RelPlan{w.histS.as<uint32_t>(), w.baseS.as<uint64_t>(), w.segStartS.as<uint64_t>(),
                   w.segTileS.as<uint32_t>()};
    pa.nR = nR;
    pa.nS = nS;
    pa.P_log2 = B;
    pa.b1 = b1;
    pa.b2 = b2;
    pa.passes = passes;
    pa.capR = capR;
    pa.capS = capS;
    pa.items = w.items.as<Item>();
    pa.item_cap = item_cap;
    pa.ctrl = ctrl;
    if ((e = launch_plan(pa, st)) != cudaSuccess) return cuda_error(e, "plan");
    mark(w, timing, 1, st);

    // pass 1 (and pass 2)
    auto scatter = [&](const Row *in, Row *out, uint64_t n, int slot, bool second,
                       const RelPlan &rp) -> cudaError_t {
        ScatterArgs a;
        a.in = in;
        a.out = out;
        a.out_n = n;
        a.tile_ctr = &ctrl->tiles[slot];
        a.err = &ctrl->error;
        a.status = w.status.as<uint64_t>();
        a.epoch = w.next_epoch(st);
        a.rf = rf;
        a.flat_n = n;
        uint64_t max_tiles = (n + SCATTER_TILE - 1) / SCATTER_TILE;
        if (passes == 1) {
            a.seg_start = nullptr;
            a.seg_tile = nullptr;
            a.nseg = 0;
            a.bases = rp.base;
            a.dshift = 0;
            a.dbits = B;
        } else if (!second) {
            a.seg_start = nullptr;
            a.seg_tile = nullptr;
            a.nseg = 0;
            a.bases = rp.seg_start;
            a.dshift = b2;
            a.dbits = b1;
        } else {
            a.seg_start = rp.seg_start;
            a.seg_tile = rp.seg_tile;
            a.nseg = (uint32_t)F1;
            a.bases = rp.base;
            a.dshift = 0;
            a.dbits = b2;
            max_tiles += F1;
        }
        return launch_scatter(a, n ? max_tiles : 0, st);
    };
    Row *outR = w.partR.as<Row>(), *outS = w.partS.as<Row>();
    if (passes == 1) {
        if ((e = scatter(dR, outR, nR, 0, false, pa.r)) != cudaSuccess) return cuda_error(e, "scatter R");
        if ((e = scatter(dS, outS, nS, 1, false, pa.s)) != cudaSuccess) return cuda_error(e, "scatter S");
        mark(w, timing, 2, st);
        mark(w, timing, 3, st);
    } else {
        Row *tR = w.tmpR.as<Row>(), *tS = w.tmpS.as<Row>();
        if ((e = scatter(dR, tR, nR, 0, false, pa.r)) != cudaSuccess) return cuda_error(e, "scatter R1");
        if ((e = scatter(dS, tS, nS, 1, false, pa.s)) != cudaSuccess) return cuda_error(e, "scatter S1");
        mark(w, timing, 2, st);
        if ((e = scatter(tR, outR, nR, 2, true, pa.r)) != cudaSuccess) return cuda_error(e, "scatter R2");
        if ((e = scatter(tS, outS, nS, 3, true, pa.s)) != cudaSuccess) return cuda_error(e, "scatter S2");
        mark(w, timing, 3, st);
    }

    JoinArgs ja;
    ja.R = outR;
    ja.S = outS;
    ja.items = w.items.as<Item>();
    ja.nitems = &ctrl->nitems;
    ja.item_ctr = &ctrl->item_ctr[0];
    ja.capR = capR;
    ja.hash_shift = B;
    ja.layout = cfg.algo == TBG_RHT ? 1 : 0;
    ja.matches = &ctrl->matches;
    ja.rows_ctr = &ctrl->rows;
    ja.out = d_rows;
    ja.cap = d_rows ? cap : 0;
    ja.err = &ctrl->error;
    if ((e = launch_join(ja, cfg.materialize != 0, join_grid, st)) != cudaSuccess)
        return cuda_error(e, "join");
    mark(w, timing, 4, st);
    run->timed = timing;
    return TBG_OK;
}

// Reads back the control block and fills stats; waits for the stream.
int finish_join(const tbg_config &cfg, Workspace &w, cudaStream_t st, const JoinRun &run,
                uint64_t nR, uint64_t nS, uint64_t cap, uint64_t *matches, tbg_stats *stats) {
    cudaError_t e = cudaMemcpyAsync(w.host_ctrl, w.ctrl.p, sizeof(Ctrl), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return cuda_error(e, "readback");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_error(e, "join");
    const Ctrl &c = *w.host_ctrl;
    if (matches) *matches = c.matches;
    if (stats) {
        memset(stats, 0, sizeof *stats);
        stats->matches = c.matches;
        stats->partitions = run.P;
        stats->work_items = c.nitems;
        stats->max_part_R = c.max_part_R;
        stats->max_part_S = c.max_part_S;
        stats->mean_part_R = run.P ? (double)nR / run.P : 0;
        stats->mean_part_S = run.P ? (double)nS / run.P : 0;
        double mr = stats->mean_part_R > 0 ? c.max_part_R / stats->mean_part_R : 0;
        double ms = stats->mean_part_S > 0 ? c.max_part_S / stats->mean_part_S : 0;
        stats->imbalance = std::max(mr, ms);
        stats->radix_bits = run.B;
        stats->passes = run.passes;
        stats->heavy_keys = c.heavy_keys;
        stats->heavy_rows_S = c.heavy_rows_S;
        stats->used_fallback = run.used_fallback;
        stats->predicted_imbalance = run.predicted_imbalance;
        stats->train_steps = run.train_steps;
        stats->train_loss = run.train_loss;
        stats->kernel_launches = (uint32_t)run.launches;
        if (run.timed) {
            float t;
            cudaEventElapsedTime(&t, w.ev[0], w.ev[1]); stats->ms_hist = t;
            cudaEventElapsedTime(&t, w.ev[1], w.ev[2]); stats->ms_pass1 = t;
            cudaEventElapsedTime(&t, w.ev[2], w.ev[3]); stats->ms_pass2 = t;
            cudaEventElapsedTime(&t, w.ev[3], w.ev[4]); stats->ms_join = t;
            cudaEventElapsedTime(&t, w.ev[0], w.ev[4]); stats->ms_total = t;
            stats->ms_learn = run.ms_learn;
        }
    }
    if (c.error) {
        if (c.error == TBG_ERR_TIMEOUT)
            return set_error(TBG_ERR_TIMEOUT, "a device-side wait gave up (look-back or queue)");
        return set_error((int)c.error, "device reported error %u", c.error);
    }
    if (cfg.materialize && c.matches > cap)
        return set_error(TBG_ERR_CAPACITY, "%llu result rows exceed capacity %llu",
                         (unsigned long long)c.matches, (unsigned long long)cap);
    return TBG_OK;
}

static int validate(const tbg_config *cfg, const void *dR, uint64_t nR, const void *dS, uint64_t nS) {
    if (!cfg) return set_error(TBG_ERR_ARG, "null config");
    if ((nR && !dR) || (nS && !dS)) return set_error(TBG_ERR_ARG, "null relation with rows");
    if (cfg->algo < TBG_RHO || cfg->algo > TBG_LRN) return set_error(TBG_ERR_ARG, "unknown algo %d", cfg->algo);
    if ((reinterpret_cast<uintptr_t>(dR) | reinterpret_cast<uintptr_t>(dS)) & 7)
        return set_error(TBG_ERR_ARG, "relations must be 8-byte aligned");
    if (nR > 0xFFFFFFFFull || nS > (1ull << 40)) return set_error(TBG_ERR_ARG, "relation too large");
    return TBG_OK;
}

int join_device_impl(const tbg_config *cfg, const Row *dR, uint64_t nR, const Row *dS, uint64_t nS,
                     tbg_row_out *d_rows, uint64_t rows_cap, cudaStream_t st, JoinRun *run,
                     Workspace **wout) {
    int rc = validate(cfg, dR, nR, dS, nS);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_error(TBG_ERR_NO_DEVICE, "no CUDA device");
    }
    Workspace *w = workspace_for(st);
    if (!w) return set_error(TBG_ERR_CUDA, "workspace");
    *wout = w;
    const uint64_t l0 = g_launches.load();
    cudaError_t e = w->ctrl.ensure(sizeof(Ctrl));
    if (e != cudaSuccess) return cuda_error(e, "cudaMalloc");
    if (nR == 0 || nS == 0) {
        e = cudaMemsetAsync(w->ctrl.p, 0, sizeof(Ctrl), st);
        run->P = 0;
        return e == cudaSuccess ? TBG_OK : cuda_error(e, "memset");
    }
    switch (cfg->algo) {
    case TBG_RHO:
    case TBG_RHT: rc = run_radix_join(*cfg, dR, nR, dS, nS, d_rows, rows_cap, *w, st, run); break;
    case TBG_RSM: rc = run_sortmerge_join(*cfg, dR, nR, dS, nS, d_rows, rows_cap, *w, st, run); break;
    case TBG_PSM: rc = run_psm_join(*cfg, dR, nR, dS, nS, d_rows, rows_cap, *w, st, run); break;
    case TBG_LRN: rc = run_learned_join(*cfg, dR, nR, dS, nS, d_rows, rows_cap, *w, st, run); break;
    }
    run->launches = g_launches.load() - l0;
    return rc;
}

}  // namespace tbg

using namespace tbg;

extern "C" {

void tbg_config_init(tbg_config *cfg) {
    if (!cfg) return;
    memset(cfg, 0, sizeof *cfg);
    cfg->algo = TBG_RHO;
    cfg->skew_split = 1;
    cfg->model = TBG_MODEL_MLP;
    cfg->train_steps = 300;
    cfg->heavy_bypass = 1;
    cfg->sample_rate = 0.01;
    cfg->imbalance_limit = 4.0;
    cfg->seed = 0x5eed;
}

int tbg_join_device(const tbg_config *cfg, const struct row_t *dR, uint64_t nR,
                    const struct row_t *dS, uint64_t nS, tbg_row_out *d_rows, uint64_t rows_cap,
                    uint64_t *matches, tbg_stats *stats, void *stream) {
    t_err = TBG_OK;
    cudaStream_t st = (cudaStream_t)stream;
    JoinRun run;
    Workspace *w = nullptr;
    int rc = join_device_impl(cfg, reinterpret_cast<const Row *>(dR), nR,
                              reinterpret_cast<const Row *>(dS), nS, d_rows, rows_cap, st, &run, &w);
    if (rc) return rc;
    return finish_join(*cfg, *w, st, run, nR, nS, cfg->materialize ? rows_cap : 0, matches, stats);
}

int tbg_join_device_async(const tbg_config *cfg, const struct row_t *dR, uint64_t nR,
                          const struct row_t *dS, uint64_t nS, tbg_row_out *d_rows,
                          uint64_t rows_cap, uint64_t *d_matches, void *stream) {
    t_err = TBG_OK;
    cudaStream_t st = (cudaStream_t)stream;
    JoinRun run;
    Workspace *w = nullptr;
    int rc = join_device_impl(cfg, reinterpret_cast<const Row *>(dR), nR,
                              reinterpret_cast<const Row *>(dS), nS, d_rows, rows_cap, st, &run, &w);
    if (rc) return rc;
    if (d_matches) {
        cudaError_t e = cudaMemcpyAsync(d_matches, &w->ctrl.as<Ctrl>()->matches, 8,
                                        cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return cuda_error(e, "copy count");
    }
    return TBG_OK;
}

int tbg_sync_status(void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    Workspace *w = workspace_for(st);
    if (!w || !w->ctrl.p) return set_error(TBG_ERR_ARG, "no join ran on this stream");
    unsigned err = 0;
    cudaError_t e = cudaMemcpyAsync(&err, &w->ctrl.as<Ctrl>()->error, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_error(e, "sync");
    if (err) return set_error((int)err, "device reported error %u", err);
    return TBG_OK;
}

uint64_t tbg_kernel_launches(void) { return g_launches.load(); }

int tbg_set_error_mode(int mode) { return g_errmode.exchange(mode); }
int tbg_last_error(void) { return t_err; }
const char *tbg_last_error_string(void) { return t_msg; }

int tbg_gen_pk(struct row_t *d, uint64_t n, uint64_t seed, void *stream) {
    if (n && !d) return set_error(TBG_ERR_ARG, "null buffer");
    cudaError_t e = launch_gen_pk(reinterpret_cast<Row *>(d), n, seed, (cudaStream_t)stream);
    return e == cudaSuccess ? TBG_OK : cuda_error(e, "gen_pk");
}

int tbg_gen_fk(struct row_t *d, uint64_t n, uint64_t maxid, uint64_t seed, void *stream) {
    if ((n && !d) || maxid == 0) return set_error(TBG_ERR_ARG, "bad arguments");
    cudaError_t e = launch_gen_fk(reinterpret_cast<Row *>(d), n, maxid, seed, (cudaStream_t)stream);
    return e == cudaSuccess ? TBG_OK : cuda_error(e, "gen_fk");
}

int tbg_gen_zipf(struct row_t *d, uint64_t n, uint64_t alphabet, double z, int scatter,
                 uint64_t seed, void *stream) {
    if ((n && !d) || alphabet == 0 || z < 0) return set_error(TBG_ERR_ARG, "bad arguments");
    cudaError_t e = launch_gen_zipf(reinterpret_cast<Row *>(d), n, alphabet, z, scatter, seed,
                                    (cudaStream_t)stream);
    return e == cudaSuccess ? TBG_OK : cuda_error(e, "gen_zipf");
}

int tbg_rows_checksum(const tbg_row_out *d_rows, uint64_t n, uint64_t *checksum, void *stream) {
    if ((n && !d_rows) || !checksum) return set_error(TBG_ERR_ARG, "bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    Workspace *w = workspace_for(st);
    if (!w) return set_error(TBG_ERR_CUDA, "workspace");
    cudaError_t e = w->misc.ensure(64);
    if (e == cudaSuccess)
        e = launch_checksum(d_rows, n, w->misc.as<unsigned long long>(), st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(w->host_ctrl, w->misc.p, 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_error(e, "checksum");
    *checksum = *reinterpret_cast<unsigned long long *>(w->host_ctrl);
    return TBG_OK;
}

}  // extern "C"
