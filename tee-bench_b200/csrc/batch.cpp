// Batched joins: planner, autotuner and CUDA graph behind tbg_batch_*.
//
// A plan fixes, per join, the partitioning (direct, or one radix pass of B
// bits), the table layout, the S rows per work item (capS) and the rows per
// histogram/scatter chunk; lays out every partitioned copy, histogram, base
// array and item list in one device allocation (256-byte aligned regions, so
// no cache line is shared by two joins); and lists the tickets of the
// persistent kernel.  The autotuner picks those choices per size class
// (floor(log2 |R_i|)) by timing candidate plans over the batch's own joins
// of that class.  The final plan is captured as one CUDA graph: a memset of
// the progress counters and results, the persistent kernel, and a copy of
// the device error word to pinned host memory.
//
// The reference has no batched mode: its driver runs one join per call
// (native.cpp:125), so each join's count here is checked against the
// reference's RHO count of that join.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "batch.h"
#include "tbg_runtime.h"

namespace tbg {
namespace {

constexpr int NCLASS = 33;
constexpr size_t ALIGN = 256;

size_t align_up(size_t x) { return (x + ALIGN - 1) & ~(ALIGN - 1); }
uint64_t ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

int size_class(uint64_t nR) { return nR <= 1 ? 0 : 63 - __builtin_clzll(nR); }

struct Choice {
    int B = 0;               // 0: direct join, > 0: radix bits of the single pass
    int layout = 0;          // table layout: 0 bucket chain, 1 histogram
    uint32_t capS = 65536;   // S rows per work item / direct slice
    uint32_t chunk = 262144;  // rows per histogram and scatter chunk
    double ms = 0;           // tuned time of the class sample (0: not tuned)
    int joins = 0;           // joins of the batch in this class
    int tuned = 0;
};

// Partitions of about capR / 2 rows for the largest |R| of the class;
// classes whose R fits one table are joined directly.
Choice heuristic(int cls) {
    Choice c;
    const uint64_t rmax = (2ull << cls) - 1;
    if (rmax <= (uint64_t)BATCH_CAPR) {
        c.B = 0;
    } else {
        int B = cls + 1 - 12;
        c.B = std::max(1, std::min(B, 8));
    }
    return c;
}

struct Plan {
    int grid = 0;
    int njoins = 0;     // caller's join count (result slots)
    DevBuf part, meta, ctl;
    size_t ctl_bytes = 0, counts_off = 0;
    BatchArgs args{};
    uint64_t rows = 0;  // input rows covered by the plan
    uint32_t tickets = 0;
};

int validate(const tbg_batch_join *joins, int njoins) {
    if (njoins < 0 || (njoins > 0 && !joins)) return set_error(TBG_ERR_ARG, "tbg_batch_create: bad join array");
    for (int i = 0; i < njoins; i++) {
        const tbg_batch_join &j = joins[i];
        if ((j.nR && !j.dR) || (j.nS && !j.dS))
            return set_error(TBG_ERR_ARG, "join %d: null relation with nonzero size", i);
        if (j.nR >= (1ull << 32) || j.nS >= (1ull << 32))
            return set_error(TBG_ERR_ARG, "join %d: relations must hold fewer than 2^32 rows", i);
        if ((reinterpret_cast<uintptr_t>(j.dR) | reinterpret_cast<uintptr_t>(j.dS)) & 7)
            return set_error(TBG_ERR_ARG, "join %d: relations must be 8-byte aligned", i);
    }
    return TBG_OK;
}

// Builds the plan of joins `sel` (indices into `joins`) with choice
// `ch[size_class]`; allocates and uploads everything the kernel reads.
// Uploads are ordered on `st` and complete when this returns.
int build_plan(const tbg_batch_join *joins, int njoins, const std::vector<int> &sel, const Choice *ch,
               int grid, Plan &p, cudaStream_t st) {
    std::vector<int> order(sel);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return joins[a].nR + joins[a].nS > joins[b].nR + joins[b].nS;
    });
    std::vector<BatchJoin> bj;
    std::vector<uint2> chunks, jt;
    std::vector<uint32_t> scans;
    struct Off { size_t rp, sp, hr, hs, br, bs, it; };
    std::vector<Off> off;
    size_t part_bytes = 0, meta2 = 0;  // partitioned rows | histograms, bases, items
    uint64_t rows = 0;
    for (int idx : order) {
        const tbg_batch_join &in = joins[idx];
        if (in.nR == 0 || in.nS == 0) continue;  // count stays 0
        const Choice &c = ch[size_class(in.nR)];
        BatchJoin J{};
        J.R = reinterpret_cast<const Row *>(in.dR);
        J.S = reinterpret_cast<const Row *>(in.dS);
        J.nR = in.nR;
        J.nS = in.nS;
        J.B = (uint32_t)c.B;
        J.P = 1u << c.B;
        J.layout = (uint32_t)c.layout;
        J.capS = c.capS;
        J.chunk = c.chunk;
        J.orig = (uint32_t)idx;
        const uint32_t j = (uint32_t)bj.size();
        rows += in.nR + in.nS;
        Off o{};
        if (c.B > 0) {
            J.GR = (uint32_t)ceil_div(in.nR, c.chunk);
            J.GS = (uint32_t)ceil_div(in.nS, c.chunk);
            J.item_cap = (uint32_t)(J.P + ceil_div(in.nS, c.capS));
            o.rp = part_bytes; part_bytes = align_up(part_bytes + in.nR * sizeof(Row));
            o.sp = part_bytes; part_bytes = align_up(part_bytes + in.nS * sizeof(Row));
            o.hr = meta2; meta2 = align_up(meta2 + (size_t)J.GR * J.P * 4);
            o.hs = meta2; meta2 = align_up(meta2 + (size_t)J.GS * J.P * 4);
            o.br = meta2; meta2 = align_up(meta2 + (size_t)J.P * 4);
            o.bs = meta2; meta2 = align_up(meta2 + (size_t)J.P * 4);
            o.it = meta2; meta2 = align_up(meta2 + (size_t)J.item_cap * sizeof(Item));
            for (uint32_t k = 0; k < J.GR; k++) chunks.push_back(make_uint2(j, k));
            for (uint32_t k = 0; k < J.GS; k++) chunks.push_back(make_uint2(j, 0x80000000u | k));
            scans.push_back(j);
            const uint64_t workers = std::min<uint64_t>(J.item_cap, std::max<uint64_t>(1, (in.nR + in.nS) >> 18));
            for (uint64_t w = 0; w < workers; w++) jt.push_back(make_uint2(j, (uint32_t)w));
        } else {
            const uint64_t slices = ceil_div(in.nS, c.capS);
            for (uint64_t k = 0; k < slices; k++) jt.push_back(make_uint2(j, (uint32_t)k));
        }
        bj.push_back(J);
        off.push_back(o);
    }
    if (chunks.size() >= (1u << 30) || jt.size() >= (1u << 30))
        return set_error(TBG_ERR_ARG, "batch too large: %zu chunks", chunks.size());
    // device memory: [partitioned rows][histograms, bases, items] and the plan arrays
    const size_t meta_off = part_bytes;
    cudaError_t e = p.part.ensure(std::max<size_t>(ALIGN, part_bytes + meta2));
    if (e != cudaSuccess) return cuda_error(e, "cudaMalloc (batch partitions)");
    char *base = p.part.as<char>();
    for (size_t k = 0; k < bj.size(); k++) {
        BatchJoin &J = bj[k];
        if (J.B == 0) continue;
        const Off &o = off[k];
        J.Rp = reinterpret_cast<Row *>(base + o.rp);
        J.Sp = reinterpret_cast<Row *>(base + o.sp);
        J.histR = reinterpret_cast<uint32_t *>(base + meta_off + o.hr);
        J.histS = reinterpret_cast<uint32_t *>(base + meta_off + o.hs);
        J.baseR = reinterpret_cast<uint32_t *>(base + meta_off + o.br);
        J.baseS = reinterpret_cast<uint32_t *>(base + meta_off + o.bs);
        J.items = reinterpret_cast<Item *>(base + meta_off + o.it);
    }
    // histograms start zeroed, so a run whose waits gave up still reads in-range sizes
    if (meta2) {
        e = cudaMemsetAsync(base + meta_off, 0, meta2, st);
        if (e != cudaSuccess) return cuda_error(e, "cudaMemsetAsync");
    }
    const size_t m_joins = 0;
    const size_t m_chunks = align_up(m_joins + bj.size() * sizeof(BatchJoin));
    const size_t m_scans = align_up(m_chunks + chunks.size() * sizeof(uint2));
    const size_t m_jt = align_up(m_scans + scans.size() * sizeof(uint32_t));
    const size_t m_end = align_up(m_jt + jt.size() * sizeof(uint2));
    std::vector<char> host(m_end);
    if (!bj.empty()) memcpy(host.data() + m_joins, bj.data(), bj.size() * sizeof(BatchJoin));
    if (!chunks.empty()) memcpy(host.data() + m_chunks, chunks.data(), chunks.size() * sizeof(uint2));
    if (!scans.empty()) memcpy(host.data() + m_scans, scans.data(), scans.size() * sizeof(uint32_t));
    if (!jt.empty()) memcpy(host.data() + m_jt, jt.data(), jt.size() * sizeof(uint2));
    e = p.meta.ensure(std::max<size_t>(ALIGN, m_end));
    if (e != cudaSuccess) return cuda_error(e, "cudaMalloc (batch plan)");
    if (m_end) {
        e = cudaMemcpyAsync(p.meta.p, host.data(), m_end, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_error(e, "cudaMemcpyAsync (batch plan)");
    }
    // control block: ticket, error word, per-join progress, results
    const size_t sync_off = ALIGN;
    p.counts_off = align_up(sync_off + bj.size() * sizeof(BatchSync));
    p.ctl_bytes = p.counts_off + (size_t)njoins * sizeof(unsigned long long);
    e = p.ctl.ensure(std::max<size_t>(ALIGN, p.ctl_bytes));
    if (e != cudaSuccess) return cuda_error(e, "cudaMalloc (batch control)");
    if (meta2 && (e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_error(e, "cudaStreamSynchronize");
    char *m = p.meta.as<char>();
    char *c = p.ctl.as<char>();
    BatchArgs &a = p.args;
    a.joins = reinterpret_cast<const BatchJoin *>(m + m_joins);
    a.chunks = reinterpret_cast<const uint2 *>(m + m_chunks);
    a.scans = reinterpret_cast<const uint32_t *>(m + m_scans);
    a.jt = reinterpret_cast<const uint2 *>(m + m_jt);
    a.ticket = reinterpret_cast<unsigned *>(c);
    a.err = reinterpret_cast<unsigned *>(c) + 1;
    a.sync = reinterpret_cast<BatchSync *>(c + sync_off);
    a.counts = reinterpret_cast<unsigned long long *>(c + p.counts_off);
    a.n_chunks = (uint32_t)chunks.size();
    a.n_scans = (uint32_t)scans.size();
    a.n_jt = (uint32_t)jt.size();
    a.capR = BATCH_CAPR;
    p.grid = grid;
    p.njoins = njoins;
    p.rows = rows;
    p.tickets = 2 * a.n_chunks + a.n_scans + a.n_jt;
    return TBG_OK;
}

cudaError_t enqueue(const Plan &p, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(p.ctl.p, 0, p.ctl_bytes, st);
    if (e != cudaSuccess) return e;
    if (p.tickets == 0) return cudaSuccess;
    return launch_batch(p.args, p.grid, st);
}

// Device time of one run of the plan (best of `reps` after one warm-up).
int time_plan(const Plan &p, cudaStream_t st, int reps, double *ms, unsigned *err_host) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    double best = 1e30;
    cudaError_t e = cudaSuccess;
    for (int r = 0; r <= reps && e == cudaSuccess; r++) {
        cudaEventRecord(a, st);
        e = enqueue(p, st);
        cudaEventRecord(b, st);
        if (e == cudaSuccess) e = cudaEventSynchronize(b);
        float t = 0;
        cudaEventElapsedTime(&t, a, b);
        if (r > 0) best = std::min(best, (double)t);
    }
    unsigned err = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&err, p.args.err, sizeof(unsigned), cudaMemcpyDeviceToHost);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e != cudaSuccess) return cuda_error(e, "batch autotune run");
    *err_host = err;
    if (err) return set_error((int)err, "batch autotune run: device status %u", err);
    *ms = best;
    return TBG_OK;
}

}  // namespace
}  // namespace tbg

using namespace tbg;

struct tbg_batch {
    Plan plan;
    Choice cls[NCLASS];
    cudaStream_t st = nullptr;       // capture / tuning stream
    cudaStream_t last = nullptr;     // stream of the last run
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned *host_err = nullptr;    // pinned copy of the device error word
    int device = 0;
    double tune_ms = 0;
};

static void batch_free(tbg_batch *b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->host_err) cudaFreeHost(b->host_err);
    if (b->st) cudaStreamDestroy(b->st);
    b->plan.part.release();
    b->plan.meta.release();
    b->plan.ctl.release();
    delete b;
}

// Picks the choice of every size class present in the batch by timing
// candidates on up to ~2^25 rows of that class's own joins: first the
// partitioning (direct or B bits), then the table layout, the S rows per
// item and the chunk size, keeping each winner.
static int autotune(tbg_batch *b, const tbg_batch_join *joins, int njoins, int grid, int force_layout) {
    std::vector<int> members[NCLASS];
    for (int i = 0; i < njoins; i++)
        if (joins[i].nR && joins[i].nS) members[size_class(joins[i].nR)].push_back(i);
    for (int c = 0; c < NCLASS; c++) {
        if (members[c].empty()) continue;
        std::vector<int> sample;
        uint64_t rows = 0;
        for (int i : members[c]) {
            if (!sample.empty() && rows + joins[i].nR + joins[i].nS > (1ull << 25)) break;
            sample.push_back(i);
            rows += joins[i].nR + joins[i].nS;
        }
        Choice best = b->cls[c];
        best.ms = 1e30;
        Plan trial;
        auto run = [&](Choice cand) -> int {
            Choice tab[NCLASS];
            tab[c] = cand;
            int rc = build_plan(joins, njoins, sample, tab, grid, trial, b->st);
            if (rc) return rc;
            double ms = 0;
            unsigned err = 0;
            rc = time_plan(trial, b->st, 2, &ms, &err);
            if (rc) return rc;
            if (ms < best.ms) {
                best = cand;
                best.ms = ms;
            }
            return TBG_OK;
        };
        const Choice h = heuristic(c);
        std::vector<int> bits;
        const uint64_t rmax = (2ull << c) - 1;
        if (rmax <= 4ull * BATCH_CAPR) bits.push_back(0);  // direct: R re-read at most 4 times
        const int b0 = std::max(1, h.B);
        for (int B = b0 - 1; B <= b0 + 2; B++)
            if (B >= 1 && B <= 8 && (rmax >> B) <= 4ull * BATCH_CAPR) bits.push_back(B);
        int rc = TBG_OK;
        for (int B : bits) {
            Choice cand = h;
            cand.B = B;
            cand.layout = force_layout >= 0 ? force_layout : 0;
            if ((rc = run(cand))) break;
        }
        if (!rc && force_layout < 0) {
            Choice cand = best;
            cand.layout = 1;
            rc = run(cand);
        }
        for (uint32_t capS : {16384u, 262144u}) {
            if (rc) break;
            Choice cand = best;
            cand.capS = capS;
            rc = run(cand);
        }
        if (!rc && best.B > 0) {
            for (uint32_t chunk : {65536u, 1048576u}) {
                Choice cand = best;
                cand.chunk = chunk;
                if ((rc = run(cand))) break;
            }
        }
        trial.part.release();
        trial.meta.release();
        trial.ctl.release();
        if (rc) return rc;
        best.tuned = 1;
        best.joins = (int)members[c].size();
        b->cls[c] = best;
    }
    return TBG_OK;
}

extern "C" {

TBG_API int tbg_batch_create(const tbg_batch_join *joins, int njoins, const tbg_config *cfg, void *stream,
                             tbg_batch **out) {
    if (!out) return set_error(TBG_ERR_ARG, "tbg_batch_create: out is NULL");
    *out = nullptr;
    tbg_config def;
    tbg_config_init(&def);
    const tbg_config &c = cfg ? *cfg : def;
    if (c.algo != TBG_RHO && c.algo != TBG_RHT)
        return set_error(TBG_ERR_ARG, "tbg_batch_create: batched joins are radix hash joins (RHO or RHT)");
    if (c.materialize) return set_error(TBG_ERR_ARG, "tbg_batch_create: batched joins return counts only");
    if (c.radix_bits > 8) return set_error(TBG_ERR_ARG, "tbg_batch_create: radix_bits above 8 (one pass)");
    int rc = validate(joins, njoins);
    if (rc) return rc;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    // the inputs may still be in flight on the caller's stream; tuning runs on a private one
    e = stream ? cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) : cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_error(e, "tbg_batch_create: synchronize");
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int grid = nsm * batch_ctas_per_sm();
    tbg_batch *b = new tbg_batch();
    b->device = dev;
    const int force_layout = c.algo == TBG_RHT ? 1 : -1;
    for (int k = 0; k < NCLASS; k++) {
        b->cls[k] = heuristic(k);
        if (force_layout >= 0) b->cls[k].layout = force_layout;
        if (c.radix_bits > 0) b->cls[k].B = c.radix_bits;
    }
    for (int i = 0; i < njoins; i++)
        if (joins[i].nR && joins[i].nS && c.radix_bits != 0) b->cls[size_class(joins[i].nR)].joins++;
    if ((e = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaMallocHost(&b->host_err, sizeof(unsigned))) != cudaSuccess) {
        batch_free(b);
        return cuda_error(e, "tbg_batch_create");
    }
    *b->host_err = 0;
    if (c.radix_bits == 0) {
        cudaEvent_t t0, t1;
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, b->st);
        rc = autotune(b, joins, njoins, grid, force_layout);
        cudaEventRecord(t1, b->st);
        cudaEventSynchronize(t1);
        float ms = 0;
        cudaEventElapsedTime(&ms, t0, t1);
        b->tune_ms = ms;
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        if (rc) {
            batch_free(b);
            return rc;
        }
    }
    std::vector<int> all(njoins);
    for (int i = 0; i < njoins; i++) all[i] = i;
    rc = build_plan(joins, njoins, all, b->cls, grid, b->plan, b->st);
    if (rc) {
        batch_free(b);
        return rc;
    }
    // one graph: reset counters and results, the persistent kernel, error word to the host
    e = cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaError_t e1 = enqueue(b->plan, b->st);
        cudaError_t e2 = cudaMemcpyAsync(b->host_err, b->plan.args.err, sizeof(unsigned), cudaMemcpyDeviceToHost,
                                         b->st);
        e = cudaStreamEndCapture(b->st, &b->graph);
        if (e1 != cudaSuccess) e = e1;
        else if (e2 != cudaSuccess) e = e2;
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (e != cudaSuccess) {
        batch_free(b);
        return cuda_error(e, "tbg_batch_create: graph capture");
    }
    *out = b;
    return TBG_OK;
}

TBG_API int tbg_batch_run(tbg_batch *b, uint64_t *d_counts, void *stream) {
    if (!b) return set_error(TBG_ERR_ARG, "tbg_batch_run: NULL batch");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaGraphLaunch(b->exec, st);
    if (e != cudaSuccess) return cuda_error(e, "cudaGraphLaunch");
    if (b->plan.tickets) count_launch();
    if (d_counts && b->plan.njoins) {
        e = cudaMemcpyAsync(d_counts, b->plan.args.counts, (size_t)b->plan.njoins * sizeof(uint64_t),
                            cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return cuda_error(e, "cudaMemcpyAsync (batch counts)");
    }
    b->last = st;
    return TBG_OK;
}

TBG_API int tbg_batch_sync(tbg_batch *b) {
    if (!b) return set_error(TBG_ERR_ARG, "tbg_batch_sync: NULL batch");
    cudaError_t e = cudaStreamSynchronize(b->last);
    if (e != cudaSuccess) return cuda_error(e, "cudaStreamSynchronize");
    const unsigned err = *b->host_err;
    if (err) return set_error((int)err, "batched join: device status %u (a bounded wait gave up)", err);
    return TBG_OK;
}

TBG_API int tbg_batch_describe(const tbg_batch *b, char *buf, size_t cap) {
    if (!b) return set_error(TBG_ERR_ARG, "tbg_batch_describe: NULL batch");
    std::string s = "{\"grid\": " + std::to_string(b->plan.grid) + ", \"tickets\": " +
                    std::to_string(b->plan.tickets) + ", \"chunks\": " + std::to_string(b->plan.args.n_chunks) +
                    ", \"rows\": " + std::to_string(b->plan.rows) + ", \"tune_ms\": " +
                    std::to_string(b->tune_ms) + ", \"classes\": [";
    bool first = true;
    for (int c = 0; c < NCLASS; c++) {
        const Choice &x = b->cls[c];
        if (!x.joins) continue;
        char item[256];
        snprintf(item, sizeof item,
                 "%s{\"log2_R\": %d, \"joins\": %d, \"bits\": %d, \"layout\": %d, \"capS\": %u, \"chunk\": %u, "
                 "\"tuned\": %d, \"sample_ms\": %.4f}",
                 first ? "" : ", ", c, x.joins, x.B, x.layout, x.capS, x.chunk, x.tuned, x.tuned ? x.ms : 0.0);
        s += item;
        first = false;
    }
    s += "]}";
    if (buf && cap) {
        const size_t n = std::min(cap - 1, s.size());
        memcpy(buf, s.data(), n);
        buf[n] = 0;
    }
    return (int)s.size();
}

TBG_API void tbg_batch_destroy(tbg_batch *b) {
    if (!b) return;
    if (b->last) cudaStreamSynchronize(b->last);
    cudaStreamSynchronize(b->st);
    batch_free(b);
}

}  // extern "C"
