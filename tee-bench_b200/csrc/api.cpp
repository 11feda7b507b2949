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
#include <functional>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "tbg_internal.h"
#include "tbg_learned.h"
#include "tbg_runtime.h"

namespace tbg {

static std::atomic<uint64_t> g_launches{0};
void count_launch(unsigned n) { g_launches += n; }

cudaError_t smem_limit(const void *func, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, size_t> set;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> g(mu);
    size_t &cur = set[std::make_pair(dev, func)];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

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
    if (cudaMallocHost(&w->host_ctrl, sizeof(Ctrl)) != cudaSuccess ||
        cudaMallocHost(&w->host_small, Workspace::HOST_SMALL_BYTES) != cudaSuccess) {
        cudaGetLastError();
        if (w->host_ctrl) cudaFreeHost(w->host_ctrl);
        delete w;
        return nullptr;
    }
    for (auto &e : w->ev) cudaEventCreate(&e);
    g_ws[key] = w;
    return w;
}

// Pass 2 processes units of at least this many rows (consecutive chunks of
// one pass-1 partition).  Measured on the 2^28 x 2^28 headline join: 128K-row
// units with two chunks per SM take 12.35 ms against 12.81 ms for 64K-row
// units with four (fewer, longer CTAs: less prologue and tail per row).
#ifndef TBG_PASS2_UNIT_ROWS
#define TBG_PASS2_UNIT_ROWS 131072
#endif
static constexpr uint64_t PASS2_UNIT_ROWS = TBG_PASS2_UNIT_ROWS;
// Pass-1 chunks (and histogram rows) per SM: a whole number of waves of the
// resident partitioning CTAs.
#ifndef TBG_PASS1_CHUNKS_PER_SM
#define TBG_PASS1_CHUNKS_PER_SM 2
#endif
static constexpr uint64_t PASS1_CHUNKS_PER_SM = TBG_PASS1_CHUNKS_PER_SM;

static int ceil_log2(uint64_t x) {
    int k = 0;
    while ((1ull << k) < x) k++;
    return k;
}

void choose_radix(const tbg_config &cfg, uint64_t nR, int capR, int *B, int *passes) {
    int b = cfg.radix_bits;
#ifdef TBG_RADIX_BITS_FORCE  // a build option for A/B timing of other geometries
    if (b <= 0) b = TBG_RADIX_BITS_FORCE;
#endif
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
void mark(Workspace &w, bool timing, int i, cudaStream_t st) {
    if (timing) cudaEventRecord(w.ev[i], st);
}

// Geometry of the chunked radix partitioning of R and S into 2^B final
// partitions (shared by RHO, RHT, RSM and LRN).
// R rows per shared-memory join table that the planner plans with (R
// partitions larger than that are joined in chunks).  choose_radix aims the
// average R partition at half of it.
//   Counting joins, |R| <= 2^28: JOIN_CAPR_WIDE, so the radix geometry is the
//   one whose average R partition fills a JOIN_CAPR_FIT-row table (14 bits,
//   7 + 7, at |R| = 2^27, where half-full 5120-row tables need 15 bits,
//   7 + 8).  The join then launches a JOIN_CAPR_FIT-row table kernel and a
//   JOIN_CAPR_WIDE one, each gated on the largest R partition (device
//   memory).  Measured at 2^27 x 2^30: 11.41 ms against 12.28 ms; the
//   8-bit fan-out of the second pass costs more than the bigger tables.
//   Otherwise: JOIN_CAPR_DEFAULT (three CTAs per SM) while R's partitions at
//   the largest radix (15 bits) fit it, else the next power of two, up to
//   16384 (one CTA per SM), so a partition of R is built once and S is not
//   probed twice.
int join_capacity(uint64_t nR, bool counting) {
#ifdef TBG_JOIN_CAPR_FORCE  // a build option for A/B timing of other table sizes
    if (nR) return TBG_JOIN_CAPR_FORCE;
#endif
    if (counting && nR <= ((uint64_t)JOIN_CAPR_FIT << 15)) return JOIN_CAPR_WIDE;
    const uint64_t per = (nR + (1u << 15) - 1) >> 15;
    if (per <= (uint64_t)JOIN_CAPR_DEFAULT) return JOIN_CAPR_DEFAULT;
    uint64_t c = 8192;
    while (c < per && c < 16384) c <<= 1;
    return (int)c;
}

RadixGeom radix_geometry(const tbg_config &cfg, uint64_t nR, uint64_t nS, int capR, Workspace &w) {
    RadixGeom g;
    choose_radix(cfg, nR, capR, &g.B, &g.passes);
    // an odd B gives pass 1 the smaller digit (7 + 8 at 15 bits), or with
    // TBG_PASS1_WIDER the larger (8 + 7); a build option for A/B timing
#ifndef TBG_PASS1_WIDER
#define TBG_PASS1_WIDER 0
#endif
    g.b1 = g.passes == 2 ? (TBG_PASS1_WIDER ? (g.B + 1) / 2 : g.B / 2) : g.B;
    g.b2 = g.B - g.b1;
    g.P = 1ull << g.B;
    g.F1 = 1ull << g.b1;
    g.capR = capR;
    g.join_grid = w.nsm * join_ctas_per_sm(capR, cfg.materialize != 0, cfg.algo == TBG_RHT ? 1 : 0);
    g.capS = 0;
    if (cfg.skew_split) {
        g.capS = nS / ((uint64_t)g.join_grid * 4);
        if (g.capS < 65536) g.capS = 65536;
    }
    // room for every R chunk of a partition to split its S side (k_plan
    // keeps oversized S sides whole if a skewed input still overflows this)
    g.item_cap = 2 * (nR / capR + (g.capS ? nS / g.capS : 0) + 2 * g.P) + 16;
    // four chunks per SM (two resident partitioning CTAs each).  A chunk's
    // CTA reads its row of the per-chunk prefix (2^B counters) to set up its
    // cursors, so a chunk holds at least max(4096, 2^B) rows: at 15 bits 32K
    // rows, while small joins still get enough chunks to fill the GPU.
    const uint64_t min_chunk = std::max<uint64_t>(4096, g.P);
    auto chunks = [&](uint64_t n) {
        uint64_t c = std::min<uint64_t>((uint64_t)w.nsm * PASS1_CHUNKS_PER_SM, (n + min_chunk - 1) / min_chunk);
        return (int)std::max<uint64_t>(c, 1);
    };
    g.G[0] = chunks(nR);
    g.G[1] = chunks(nS);
    g.ch[0] = ((nR + g.G[0] - 1) / g.G[0] + 1) & ~1ull;
    g.ch[1] = ((nS + g.G[1] - 1) / g.G[1] + 1) & ~1ull;
    g.n[0] = nR;
    g.n[1] = nS;
    // f = (key & (F1 - 1)) << b2 | (key >> b1) & (F2 - 1): pass 1 by the low b1
    // bits, pass 2 by the next b2
    g.rf = g.passes == 1 ? RadixF{(uint32_t)(g.P - 1), 0, 0, 0}
                         : RadixF{(uint32_t)(g.F1 - 1), (uint32_t)g.b1, (uint32_t)((1u << g.b2) - 1), (uint32_t)g.b2};
    g.d1 = DigitOp{0u, (uint32_t)(g.F1 - 1)};
    g.d2 = DigitOp{(uint32_t)g.b1, (uint32_t)((1u << g.b2) - 1)};
    return g;
}

// Geometry of an MSD partitioning of R and S by the top B bits of key - sub
// (PSM): final partition f = (key - sub) >> lowbits holds a contiguous key
// range, and partitions in order hold increasing keys.  Pass 1 takes the top
// b1 bits of f, pass 2 the low b2 (one pass when B <= 8).  Chunking as in
// radix_geometry.
RadixGeom radix_geometry_msd(uint64_t nR, uint64_t nS, uint32_t sub, int B, int lowbits, Workspace &w) {
    RadixGeom g;
    g.B = B;
    g.passes = B <= 8 ? 1 : 2;
    g.b1 = g.passes == 2 ? B / 2 : B;
    g.b2 = B - g.b1;
    g.P = 1ull << B;
    g.F1 = 1ull << g.b1;
    g.capR = 0;
    g.join_grid = 0;
    g.capS = 0;
    g.item_cap = 16;
    const uint64_t min_chunk = std::max<uint64_t>(4096, g.P);
    auto chunks = [&](uint64_t n) {
        uint64_t c = std::min<uint64_t>((uint64_t)w.nsm * PASS1_CHUNKS_PER_SM, (n + min_chunk - 1) / min_chunk);
        return (int)std::max<uint64_t>(c, 1);
    };
    g.G[0] = chunks(nR);
    g.G[1] = chunks(nS);
    g.ch[0] = ((nR + g.G[0] - 1) / g.G[0] + 1) & ~1ull;
    g.ch[1] = ((nS + g.G[1] - 1) / g.G[1] + 1) & ~1ull;
    g.n[0] = nR;
    g.n[1] = nS;
    g.rf = RadixF{0u, (uint32_t)lowbits, (uint32_t)(g.P - 1), 0u};
    g.rf.sub = sub;
    if (g.passes == 2) {
        g.d1 = DigitOp{(uint32_t)(lowbits + g.b2), (uint32_t)(g.F1 - 1), sub};
        g.d2 = DigitOp{(uint32_t)lowbits, (uint32_t)((1u << g.b2) - 1), sub};
    } else {
        g.d1 = DigitOp{(uint32_t)lowbits, (uint32_t)(g.P - 1), sub};
        g.d2 = DigitOp{0u, 0u, sub};
    }
    return g;
}

int ensure_radix_buffers(const RadixGeom &g, bool bypass, Workspace &w) {
    cudaError_t e;
#define ENSURE(buf, bytes)                                        \
    do {                                                          \
        e = (buf).ensure(bytes);                                  \
        if (e != cudaSuccess) return cuda_error(e, "cudaMalloc"); \
    } while (0)
    const uint64_t nR = g.n[0], nS = g.n[1];
    ENSURE(w.ctrl, sizeof(Ctrl));
    ENSURE(w.histR, (uint64_t)g.G[0] * g.P * 4);
    ENSURE(w.histS, (uint64_t)g.G[1] * g.P * 4);
    ENSURE(w.totR, g.P * 4);
    ENSURE(w.totS, g.P * 4);
    ENSURE(w.baseR, (g.P + 1) * 8);
    ENSURE(w.baseS, (g.P + 1) * 8);
    ENSURE(w.off1R, (uint64_t)g.G[0] * g.F1 * 4);
    ENSURE(w.off1S, (uint64_t)g.G[1] * g.F1 * 4);
    ENSURE(w.cnt1R, (uint64_t)g.G[0] * g.F1 * 4);
    ENSURE(w.cnt1S, (uint64_t)g.G[1] * g.F1 * 4);
    ENSURE(w.partR, std::max<uint64_t>(nR, 1) * 8);
    ENSURE(w.partS, std::max<uint64_t>(nS, 1) * 8);
    if (g.passes == 2) {
        ENSURE(w.tmpR, std::max<uint64_t>(nR, 1) * 8);
        ENSURE(w.tmpS, std::max<uint64_t>(nS, 1) * 8);
    }
    ENSURE(w.items, g.item_cap * sizeof(Item));
    if (bypass) {
        ENSURE(w.sc, std::max<uint64_t>(nS, 1) * 8);
        ENSURE(w.kept, (uint64_t)g.G[1] * 4);
    }
#undef ENSURE
    return TBG_OK;
}

// Histogram of one relation (with the heavy bypass for S when given), column
// prefix and partition bases.
int part_histogram(int rel, const RadixGeom &g, const Row *d, const tbg_config &cfg, Workspace &w, cudaStream_t st,
                   const SBypass *bypass) {
    Ctrl *ctrl = w.ctrl.as<Ctrl>();
    DevBuf &hist = rel ? w.histS : w.histR;
    DevBuf &tot = rel ? w.totS : w.totR;
    DevBuf &base = rel ? w.baseS : w.baseR;
    cudaError_t e;
    if (!bypass) {
        const bool check = rel == 1 && g.s_range_max != 0xFFFFFFFFu;
        e = launch_hist_chunks(d, g.n[rel], g.ch[rel], g.G[rel], hist.as<uint32_t>(), g.B, g.rf, st,
                               check ? &ctrl->out_of_range : nullptr, g.s_range_max);
    } else {
        BypassArgs ba;
        ba.in = d;
        ba.n = g.n[rel];
        ba.chunk = g.ch[rel];
        ba.G = g.G[rel];
        ba.nbins = (int)g.P;
        ba.rf = g.rf;
        ba.out = w.sc.as<Row>();
        ba.hist = hist.as<uint32_t>();
        ba.kept = w.kept.as<uint32_t>();
        ba.hkept = bypass->hkept;
        ba.hpairs = bypass->hpairs;
        ba.hkeys = bypass->keys;
        ba.hcnt = bypass->cnt;
        ba.scnt = bypass->scnt;
        ba.matches = &ctrl->matches;
        ba.heavy_rows = &ctrl->heavy_rows_S;
        e = launch_hist_bypass(ba, cfg.materialize != 0, st);
    }
    if (e != cudaSuccess) return cuda_error(e, "histogram");
    if ((e = launch_colscan(hist.as<uint32_t>(), g.G[rel], (int)g.P, tot.as<uint32_t>(), st)) != cudaSuccess)
        return cuda_error(e, "colscan");
    if ((e = launch_plan_bases(tot.as<uint32_t>(), base.as<uint64_t>(), g.B,
                               rel ? &ctrl->max_part_S : &ctrl->max_part_R, st)) != cudaSuccess)
        return cuda_error(e, "bases");
    return TBG_OK;
}

// Pass `which` (1 or 2) of one relation.  Pass 1 reads the relation (or, with
// the bypass, the compacted S); the last pass writes partR / partS.
int part_pass(int rel, int which, const RadixGeom &g, const Row *d, Workspace &w, cudaStream_t st, bool bypass) {
    Ctrl *ctrl = w.ctrl.as<Ctrl>();
    const uint64_t n = g.n[rel];
    PartArgs a;
    a.n = n;
    a.chunk = g.ch[rel];
    a.chunk_len = nullptr;
    a.G = g.G[rel];
    const uint64_t per_unit = std::max<uint64_t>(n / ((uint64_t)a.G * g.F1), 1);
    // pass-2 units of PASS2_UNIT_ROWS rows, smaller for small relations so
    // that there are about two units per SM (at least 4096 rows each)
    const uint64_t unit_rows =
        std::min<uint64_t>(PASS2_UNIT_ROWS, std::max<uint64_t>(4096, n / ((uint64_t)w.nsm * 2)));
    a.group = (int)std::min<uint64_t>((uint64_t)a.G, std::max<uint64_t>(1, unit_rows / per_unit));
    a.b1 = g.b1;
    a.b2 = g.b2;
    a.rf = g.rf;
    a.d1 = g.d1;
    a.d2 = g.d2;
    a.pre = (rel ? w.histS : w.histR).as<uint32_t>();
    a.totals = (rel ? w.totS : w.totR).as<uint32_t>();
    a.base = (rel ? w.baseS : w.baseR).as<uint64_t>();
    a.off1 = g.passes == 2 ? (rel ? w.off1S : w.off1R).as<uint32_t>() : nullptr;
    a.cnt1 = g.passes == 2 ? (rel ? w.cnt1S : w.cnt1R).as<uint32_t>() : nullptr;
    a.err = &ctrl->error;
    Row *part = (rel ? w.partS : w.partR).as<Row>();
    Row *tmp = g.passes == 2 ? (rel ? w.tmpS : w.tmpR).as<Row>() : part;
    cudaError_t e;
    if (which == 1) {
        a.in = bypass ? w.sc.as<Row>() : d;
        if (bypass) a.chunk_len = w.kept.as<uint32_t>();
        a.out = tmp;
        e = launch_part_pass1(a, st);
    } else {
        if (g.passes != 2) return TBG_OK;
        a.in = tmp;
        a.out = part;
        e = launch_part_pass2(a, st);
    }
    return e == cudaSuccess ? TBG_OK : cuda_error(e, "partition pass");
}

int plan_items(const RadixGeom &g, Workspace &w, cudaStream_t st) {
    PlanArgs pa;
    pa.r = RelPlan{w.totR.as<uint32_t>(), w.baseR.as<uint64_t>()};
    pa.s = RelPlan{w.totS.as<uint32_t>(), w.baseS.as<uint64_t>()};
    pa.nR = g.n[0];
    pa.nS = g.n[1];
    pa.P_log2 = g.B;
    pa.b1 = g.b1;
    pa.b2 = g.b2;
    pa.passes = g.passes;
    pa.capR = g.capR;
    pa.capS = g.capS;
    pa.items = w.items.as<Item>();
    pa.item_cap = g.item_cap;
    pa.ctrl = w.ctrl.as<Ctrl>();
    cudaError_t e = launch_plan(pa, st);
    return e == cudaSuccess ? TBG_OK : cuda_error(e, "plan");
}

// Single-stream radix partitioning of R and S (RHO, RHT, RSM).
int radix_partition(const tbg_config &cfg, const Row *dR, uint64_t nR, const Row *dS, uint64_t nS,
                    int capR, Workspace &w, cudaStream_t st, JoinRun *run, int *join_grid_out) {
    const bool timing = cfg.timing != 0;
    const RadixGeom g = radix_geometry(cfg, nR, nS, capR, w);
    run->B = g.B;
    run->passes = g.passes;
    run->P = g.P;
    *join_grid_out = g.join_grid;
    int rc = ensure_radix_buffers(g, false, w);
    if (rc) return rc;
    mark(w, timing, 0, st);
    cudaError_t e = cudaMemsetAsync(w.ctrl.p, 0, sizeof(Ctrl), st);
    if (e != cudaSuccess) return cuda_error(e, "memset");
    if ((rc = part_histogram(0, g, dR, cfg, w, st, nullptr))) return rc;
    if ((rc = part_histogram(1, g, dS, cfg, w, st, nullptr))) return rc;
    if ((rc = plan_items(g, w, st))) return rc;
    mark(w, timing, 1, st);
    if ((rc = part_pass(0, 1, g, dR, w, st, false))) return rc;
    if ((rc = part_pass(1, 1, g, dS, w, st, false))) return rc;
    mark(w, timing, 2, st);
    if ((rc = part_pass(0, 2, g, dR, w, st, false))) return rc;
    if ((rc = part_pass(1, 2, g, dS, w, st, false))) return rc;
    mark(w, timing, 3, st);
    return TBG_OK;
}

// The radix-partitioned join: RHO (layout 0) and RHT (layout 1).
int run_radix_join(const tbg_config &cfg, const Row *dR, uint64_t nR, const Row *dS, uint64_t nS,
                   tbg_row_out *d_rows, uint64_t cap, Workspace &w, cudaStream_t st,
                   JoinRun *run) {
    const int capR = join_capacity(nR, !cfg.materialize);
    int join_grid = 0;
    int rc = radix_partition(cfg, dR, nR, dS, nS, capR, w, st, run, &join_grid);
    if (rc) return rc;
    return radix_join_phase(cfg, d_rows, cap, w, st, run, capR, join_grid);
}

// RHO / RHT with S arriving in slices, for callers that copy S from the host
// on another stream: slice k is [s_lo[k], s_lo[k+1]) of dS.  issue(-1)
// starts R's copy and issue(k) slice k's; each records r_ready / s_ready[k]
// when its copy is done.  Slice k + 1's copy is issued before slice k's work
// is queued, so copies from pageable memory (which block the host) still
// overlap the work.  R is
// partitioned once; each slice is partitioned with R's radix geometry
// (which depends on |R| only), planned against R's partitions and joined.
// Matches and output rows accumulate in the control block across slices,
// so the count and the row multiset equal the whole join's, and slice k's
// work overlaps the copy of slice k + 1.
int run_radix_join_sliced(const tbg_config &cfg, const Row *dR, uint64_t nR, const Row *dS, const uint64_t *s_lo,
                          int nslices, const std::function<int(int)> &issue, cudaEvent_t r_ready,
                          const cudaEvent_t *s_ready, tbg_row_out *d_rows, uint64_t cap, Workspace &w,
                          cudaStream_t st, JoinRun *run) {
    const int capR = join_capacity(nR, !cfg.materialize);
    uint64_t smax = 1;
    for (int k = 0; k < nslices; k++) smax = std::max(smax, s_lo[k + 1] - s_lo[k]);
    const RadixGeom gmax = radix_geometry(cfg, nR, smax, capR, w);
    run->B = gmax.B;
    run->passes = gmax.passes;
    run->P = gmax.P;
    int rc = ensure_radix_buffers(gmax, false, w);
    if (rc) return rc;
    Ctrl *ctrl = w.ctrl.as<Ctrl>();
    if ((rc = issue(-1)) || (nslices > 0 && (rc = issue(0)))) return rc;
    cudaError_t e = cudaMemsetAsync(w.ctrl.p, 0, sizeof(Ctrl), st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, r_ready, 0);
    if (e != cudaSuccess) return cuda_error(e, "sliced join: setup");
    // R: histogram, bases and both passes, while S is still arriving
    if ((rc = part_histogram(0, gmax, dR, cfg, w, st, nullptr))) return rc;
    if ((rc = part_pass(0, 1, gmax, dR, w, st, false))) return rc;
    if ((rc = part_pass(0, 2, gmax, dR, w, st, false))) return rc;
    for (int k = 0; k < nslices; k++) {
        if (k + 1 < nslices && (rc = issue(k + 1))) return rc;
        const uint64_t n = s_lo[k + 1] - s_lo[k];
        if (!n) continue;
        const Row *d = dS + s_lo[k];
        const RadixGeom g = radix_geometry(cfg, nR, n, capR, w);
        if ((e = cudaStreamWaitEvent(st, s_ready[k], 0)) != cudaSuccess) return cuda_error(e, "sliced join: wait");
        if ((rc = part_histogram(1, g, d, cfg, w, st, nullptr))) return rc;
        if ((rc = plan_items(g, w, st))) return rc;
        if ((rc = part_pass(1, 1, g, d, w, st, false))) return rc;
        if ((rc = part_pass(1, 2, g, d, w, st, false))) return rc;
        // the join's work-item ticket restarts for every slice
        if ((e = cudaMemsetAsync(&ctrl->item_ctr[0], 0, sizeof(unsigned), st)) != cudaSuccess)
            return cuda_error(e, "memset");
        if ((rc = radix_join_phase(cfg, d_rows, cap, w, st, run, capR, g.join_grid))) return rc;
    }
    return TBG_OK;
}

// Build/probe over the partitions radix_partition left in partR / partS.
int radix_join_phase(const tbg_config &cfg, tbg_row_out *d_rows, uint64_t cap, Workspace &w, cudaStream_t st,
                     JoinRun *run, int capR, int join_grid) {
    Ctrl *ctrl = w.ctrl.as<Ctrl>();
    JoinArgs ja;
    ja.R = w.partR.as<Row>();
    ja.S = w.partS.as<Row>();
    ja.items = w.items.as<Item>();
    ja.nitems = &ctrl->nitems;
    ja.item_ctr = &ctrl->item_ctr[0];
    ja.capR = capR;
    ja.hash_shift = run->B;
    ja.layout = cfg.algo == TBG_RHT ? 1 : 0;
    ja.matches = &ctrl->matches;
    ja.rows_ctr = &ctrl->rows;
    ja.out = d_rows;
    ja.cap = d_rows ? cap : 0;
    ja.err = &ctrl->error;
    ja.gate = nullptr;
    ja.gate_max = 0;
    ja.gate_le = 0;
    cudaError_t e;
    // Counting with a smaller table takes less shared memory per CTA and is
    // faster, but only fits when no R partition is larger; that size is
    // known on the device only (the planner's max_part_R).  So both table
    // sizes are launched, each gated on it: one does the join, the other
    // returns at once, and no host read-back is needed.  The geometry of
    // JOIN_CAPR_WIDE plans aims R's partitions at JOIN_CAPR_FIT rows.
    const int small_cap = cfg.materialize ? 0
                          : capR == JOIN_CAPR_WIDE    ? JOIN_CAPR_FIT
                          : capR == JOIN_CAPR_DEFAULT ? JOIN_CAPR_SMALL
                                                      : 0;
    if (small_cap) {
        JoinArgs small = ja;
        small.capR = small_cap;
        small.gate = &ctrl->max_part_R;
        small.gate_max = (unsigned long long)small_cap;
        small.gate_le = 1;
        if ((e = launch_join(small, false, w.nsm * join_ctas_per_sm(small_cap, false, ja.layout), st)) != cudaSuccess)
            return cuda_error(e, "join");
        ja.gate = small.gate;
        ja.gate_max = (unsigned long long)small_cap;
        ja.gate_le = 0;
    }
    e = launch_join(ja, cfg.materialize != 0, join_grid, st);
    if (e != cudaSuccess) return cuda_error(e, "join");
    mark(w, cfg.timing != 0, 4, st);
    run->timed = cfg.timing != 0;
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
        stats->heavy_rows_predicted = run.heavy_pred;
        stats->heavy_rows_sampled = run.heavy_sampled;
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
    if (nR > 0xFFFFFFFFull || nS > 0xFFFFFFFFull) return set_error(TBG_ERR_ARG, "relations hold at most 2^32 - 1 rows");
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
    cfg->train_steps = 30;
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
