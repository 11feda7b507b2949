// Host pipelines of the sort-merge joins RSM and PSM.
//
// RSM (Joins/radix_sortmerge_join.c:102-105) shares RHO's radix partitioning
// and swaps the build/probe kernel for a per-partition sort + merge-path join.
// PSM (Joins/psm/parallel_sortmerge_join.h:61-111) sorts both relations by key
// (LSD radix sort, 8-bit digits, chunked stable passes; a pass whose digit is
// the same for every row is skipped) and merges them.
#include <algorithm>
#include <cstring>
#include <vector>

#include "tbg_internal.h"
#include "tbg_runtime.h"

namespace tbg {

cudaError_t launch_join_rsm(const JoinArgs &a, bool materialize, int grid, cudaStream_t st);
int rsm_ctas_per_sm(int capR, bool materialize);
cudaError_t launch_merge_join(const Row *R, uint64_t nr, const Row *S, uint64_t ns, uint64_t *splits,
                              unsigned long long *matches, unsigned long long *rows_ctr, tbg_row_out *out,
                              uint64_t cap, bool mat, cudaStream_t st);
uint64_t merge_ctas(uint64_t nr, uint64_t ns);

constexpr int RSM_CAPR = 4096;

static void mark_ev(Workspace &w, bool timing, int i, cudaStream_t st) {
    if (timing) cudaEventRecord(w.ev[i], st);
}

int run_sortmerge_join(const tbg_config &cfg, const Row *dR, uint64_t nR, const Row *dS, uint64_t nS,
                       tbg_row_out *d_rows, uint64_t cap, Workspace &w, cudaStream_t st, JoinRun *run) {
    // one shared-memory radix-sorted tile (512 threads x 8 rows) of R per item
    const int capR = RSM_CAPR;
    int join_grid = 0;
    int rc = radix_partition(cfg, dR, nR, dS, nS, capR, w, st, run, &join_grid);
    if (rc) return rc;
    Ctrl *ctrl = w.ctrl.as<Ctrl>();
    JoinArgs ja;
    memset(&ja, 0, sizeof ja);
    ja.R = w.partR.as<Row>();
    ja.S = w.partS.as<Row>();
    ja.items = w.items.as<Item>();
    ja.nitems = &ctrl->nitems;
    ja.item_ctr = &ctrl->item_ctr[0];
    ja.capR = capR;
    ja.hash_shift = run->B;
    ja.matches = &ctrl->matches;
    ja.rows_ctr = &ctrl->rows;
    ja.out = d_rows;
    ja.cap = d_rows ? cap : 0;
    ja.err = &ctrl->error;
    cudaError_t e =
        launch_join_rsm(ja, cfg.materialize != 0, w.nsm * rsm_ctas_per_sm(capR, cfg.materialize != 0), st);
    if (e != cudaSuccess) return cuda_error(e, "rsm join");
    mark_ev(w, cfg.timing != 0, 4, st);
    run->timed = cfg.timing != 0;
    return TBG_OK;
}

cudaError_t launch_sort_pass(const Row *in, Row *out, uint64_t n, uint64_t chunk, int G, const uint32_t *pre,
                             const uint32_t *totals, uint32_t shift, int digit_bits, unsigned *err, cudaStream_t st);

// LSD sort of n rows by key with chunked stable passes (per-chunk digit
// histograms, column prefix, k_sort_pass): 24 B per row per pass and no
// inter-CTA waits.  hhist holds the four 8-bit digit histograms of the input:
// 8-bit digits that are the same for every row are skipped, and when the key
// bits that vary fit fewer 9-bit digits than the remaining 8-bit passes, the
// sort uses 9-bit digits instead (e.g. 3 passes for 27-bit keys, not 4); at
// an equal pass count narrower digits win (4 passes of 7 bits for 28-bit
// keys).
int lsd_sort_chunked(const Row *in, uint64_t n, DevBuf &a, DevBuf &b, const uint32_t *hhist, Workspace &w,
                     cudaStream_t st, const Row **out, int *passes) {
    const Row *src = in;
    Row *bufs[2] = {a.as<Row>(), b.as<Row>()};
    int which = 0;
    *passes = 0;
    const int G = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)w.nsm * 4, (n + 32767) / 32768));
    const uint64_t chunk = (n + G - 1) / G;
    cudaError_t e = w.sorthist.ensure(((size_t)G + 1) * 512 * 4);
    if (e != cudaSuccess) return cuda_error(e, "cudaMalloc");
    uint32_t *hist = w.sorthist.as<uint32_t>(), *totals = hist + (size_t)G * 512;
    unsigned *err = &w.ctrl.as<Ctrl>()->error;
    if (n <= 1) {
        *out = src;
        return TBG_OK;
    }
    // the passes: (shift, digit bits)
    std::vector<std::pair<uint32_t, int>> plan;
    int lo_bit = -1, hi_bit = -1;
    for (int p = 0; p < 4; p++) {
        bool trivial = false;
        int top = 0;
        for (int d = 0; d < 256; d++) {
            if (hhist[p * 256 + d] == n) trivial = true;
            if (hhist[p * 256 + d]) top = d;
        }
        if (trivial) continue;
        plan.push_back({8u * p, 8});
        if (lo_bit < 0) lo_bit = 8 * p;
        hi_bit = 8 * p + (top ? 31 - __builtin_clz((unsigned)top) : 0);
    }
    if (lo_bit >= 0) {
        // the fewest passes of at most 9 bits over the varying span, with the
        // bits spread evenly (at least 7 per pass); taken when it saves a
        // pass, or at equal passes when its digits are narrower (cheaper
        // ranking, longer runs per digit)
        const int bits = hi_bit - lo_bit + 1;
        const int np = (bits + 8) / 9;
        const int db = std::max(7, (bits + np - 1) / np);
        if (np < (int)plan.size() || (np == (int)plan.size() && db < 8)) {
            plan.clear();
            for (int i = 0; i < np; i++) plan.push_back({(uint32_t)(lo_bit + db * i), db});
        }
    }
    for (const auto &pp : plan) {
        const uint32_t shift = pp.first;
        const int db = pp.second;
        const uint32_t m2 = (1u << db) - 1;
        if ((e = launch_hist_chunks(src, n, chunk, G, hist, db, RadixF{0u, shift, m2, 0u}, st)) != cudaSuccess ||
            (e = launch_colscan(hist, G, 1 << db, totals, st)) != cudaSuccess ||
            (e = launch_sort_pass(src, bufs[which], n, chunk, G, hist, totals, shift, db, err, st)) != cudaSuccess)
            return cuda_error(e, "sort pass");
        src = bufs[which];
        which ^= 1;
        (*passes)++;
    }
    *out = src;
    return TBG_OK;
}

// LSD sort of n rows by key with the one-sweep scatter (one launch per pass,
// decoupled look-back): used for small inputs (LRN's sample), where launch
// count matters more than bandwidth.  Returns the buffer holding the sorted
// rows.
int lsd_sort(const Row *in, uint64_t n, DevBuf &a, DevBuf &b, const uint32_t *hhist,
                    const uint64_t *dbases, int slot0, Workspace &w, cudaStream_t st, const Row **out,
                    int *passes) {
    const Row *src = in;
    Row *bufs[2] = {a.as<Row>(), b.as<Row>()};
    int which = 0;
    *passes = 0;
    for (int p = 0; p < 4; p++) {
        bool trivial = false;
        for (int d = 0; d < 256; d++)
            if (hhist[p * 256 + d] == n) trivial = true;
        if (trivial || n <= 1) continue;
        ScatterArgs s;
        memset(&s, 0, sizeof s);
        s.in = src;
        s.out = bufs[which];
        s.out_n = n;
        s.seg_start = nullptr;
        s.seg_tile = nullptr;
        s.nseg = 0;
        s.flat_n = n;
        s.bases = dbases + p * 256;
        s.status = w.status.as<uint64_t>();
        s.tile_ctr = &w.ctrl.as<Ctrl>()->tiles[slot0 + p];
        s.err = &w.ctrl.as<Ctrl>()->error;
        s.epoch = w.next_epoch(st);
        s.dshift = 8 * p;
        s.dbits = 8;
        s.rf = RadixF{0xFFFFFFFFu, 0, 0, 0};
        cudaError_t e = launch_scatter(s, (n + SCATTER_TILE - 1) / SCATTER_TILE, st);
        if (e != cudaSuccess) return cuda_error(e, "sort pass");
        src = bufs[which];
        which ^= 1;
        (*passes)++;
    }
    *out = src;
    return TBG_OK;
}

int run_psm_join(const tbg_config &cfg, const Row *dR, uint64_t nR, const Row *dS, uint64_t nS,
                 tbg_row_out *d_rows, uint64_t cap, Workspace &w, cudaStream_t st, JoinRun *run) {
    const bool timing = cfg.timing != 0;
    cudaError_t e;
    const uint64_t tiles = (std::max(nR, nS) + SCATTER_TILE - 1) / SCATTER_TILE + 1;
#define ENSURE(buf, bytes)                                        \
    do {                                                          \
        e = (buf).ensure(bytes);                                  \
        if (e != cudaSuccess) return cuda_error(e, "cudaMalloc"); \
    } while (0)
    ENSURE(w.ctrl, sizeof(Ctrl));
    ENSURE(w.aux[0], nR * 8);
    ENSURE(w.aux[1], nR * 8);
    ENSURE(w.aux[2], nS * 8);
    ENSURE(w.aux[3], nS * 8);
    ENSURE(w.aux[4], 2 * 4 * 256 * 4);
    ENSURE(w.aux[5], 2 * 4 * 256 * 8);
    ENSURE(w.aux[6], (merge_ctas(nR, nS) + 2) * 8);
    ENSURE(w.status, tiles * SCATTER_FMAX * 8);
#undef ENSURE
    Ctrl *ctrl = w.ctrl.as<Ctrl>();
    uint32_t *hist = w.aux[4].as<uint32_t>();
    uint64_t *bases = w.aux[5].as<uint64_t>();
    mark_ev(w, timing, 0, st);
    if ((e = cudaMemsetAsync(ctrl, 0, sizeof(Ctrl), st)) != cudaSuccess) return cuda_error(e, "memset");
    if ((e = launch_digit_hist(dR, nR, hist, bases, w.nsm, st)) != cudaSuccess) return cuda_error(e, "digits R");
    if ((e = launch_digit_hist(dS, nS, hist + 1024, bases + 1024, w.nsm, st)) != cudaSuccess)
        return cuda_error(e, "digits S");
    // which digit passes are needed decides the buffer chain: read the counts back
    uint32_t hh[2048];
    if ((e = cudaMemcpyAsync(hh, hist, sizeof hh, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return cuda_error(e, "digits");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_error(e, "digits");
    mark_ev(w, timing, 1, st);
    const Row *sR = nullptr, *sS = nullptr;
    int pr = 0, ps = 0;
    int rc = lsd_sort_chunked(dR, nR, w.aux[0], w.aux[1], hh, w, st, &sR, &pr);
    if (rc) return rc;
    mark_ev(w, timing, 2, st);
    rc = lsd_sort_chunked(dS, nS, w.aux[2], w.aux[3], hh + 1024, w, st, &sS, &ps);
    if (rc) return rc;
    mark_ev(w, timing, 3, st);
    e = launch_merge_join(sR, nR, sS, nS, w.aux[6].as<uint64_t>(), &ctrl->matches, &ctrl->rows, d_rows,
                          d_rows ? cap : 0, cfg.materialize != 0, st);
    if (e != cudaSuccess) return cuda_error(e, "merge join");
    mark_ev(w, timing, 4, st);
    run->B = 8;
    run->passes = std::max(pr, ps);
    run->P = 0;
    run->timed = timing;
    return TBG_OK;
}

}  // namespace tbg
