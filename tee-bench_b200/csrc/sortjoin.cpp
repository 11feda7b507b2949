// Host pipelines of the sort-merge joins RSM and PSM.
//
// RSM (Joins/radix_sortmerge_join.c:102-105) shares RHO's radix partitioning
// and swaps the build/probe kernel for a per-partition sort + merge-path join.
// PSM (Joins/psm/parallel_sortmerge_join.h:61-111) sorts both relations by key
// and merges them.  The sort is MSD: RHO's histogram and passes partition by
// the top bits of key - min (at most 15), then every bucket is sorted by the
// remaining 12 or 13 bits in one counting pass.  Relations whose key range
// leaves more low bits, or with a bucket over a million rows (a heavy key),
// take an LSD radix sort (7- to 9-bit digits, chunked stable passes).
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
                             const uint32_t *totals, uint32_t shift, uint32_t sub, int digit_bits, unsigned *err,
                             cudaStream_t st);

// Passes of the LSD sort of keys in [kmin, kmax]: (shift, digit bits) over
// the bits of key - kmin, the fewest passes of at most 9 bits with the bits
// spread evenly (at least 7 per pass: at an equal pass count narrower digits
// are cheaper to rank and give longer runs per digit).  Sorting by key - kmin
// keeps the key order and needs only the bits of the range: 3 passes for
// the keys 1..2^27 (27 bits of range), where the raw keys span 28 bits.
std::vector<std::pair<uint32_t, int>> sort_plan(uint32_t kmin, uint32_t kmax) {
    std::vector<std::pair<uint32_t, int>> plan;
    if (kmax <= kmin) return plan;
    const uint32_t span = kmax - kmin;
    const int bits = 32 - __builtin_clz(span);
    const int np = (bits + 8) / 9;
    const int db = std::max(7, (bits + np - 1) / np);
    for (int i = 0, lo = 0; i < np; i++, lo += db) plan.push_back({(uint32_t)lo, std::min(db, 32 - lo)});
    return plan;
}

// LSD sort of n rows by key with chunked stable passes (per-chunk digit
// histograms, column prefix, k_sort_pass): 24 B per row per pass and no
// inter-CTA waits.  Digits are taken from key - kmin.
int lsd_sort_chunked(const Row *in, uint64_t n, uint32_t kmin, uint32_t kmax, DevBuf &a, DevBuf &b, Workspace &w,
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
    for (const auto &pp : sort_plan(kmin, kmax)) {
        const uint32_t shift = pp.first;
        const int db = pp.second;
        const uint32_t m2 = (1u << db) - 1;
        RadixF rf{0u, shift, m2, 0u};
        rf.sub = kmin;
        if ((e = launch_hist_chunks(src, n, chunk, G, hist, db, rf, st)) != cudaSuccess ||
            (e = launch_colscan(hist, G, 1 << db, totals, st)) != cudaSuccess ||
            (e = launch_sort_pass(src, bufs[which], n, chunk, G, hist, totals, shift, kmin, db, err, st)) !=
                cudaSuccess)
            return cuda_error(e, "sort pass");
        src = bufs[which];
        which ^= 1;
        (*passes)++;
    }
    *out = src;
    return TBG_OK;
}

cudaError_t launch_bucket_sort(const Row *in, Row *out, const uint64_t *base, uint32_t nb, uint64_t n, uint32_t sub,
                               int lowbits, int nsm, cudaStream_t st);

// MSD sort of both relations: radix partitioning by the top B bits of
// key - sub (RHO's histogram and passes), then each bucket sorted by the low
// `lowbits` bits (k_bucket_sort), into sorted[0] (R) and sorted[1] (S).  A
// relation with a bucket over kBucketMax rows (a heavy key) is left for the
// LSD sort instead: msd_done[rel] says which ones were sorted.
static constexpr uint64_t kBucketMax = 1u << 20;
static constexpr int kLowBits = 12, kLowBitsMax = 13;

// With check_s, the range [sub, sub + 2^span) is R's alone: S's histogram
// also counts S's keys outside it, and if there are any, nothing is sorted
// and *s_outside is set (the caller then takes both relations' range).
static int msd_sort(const tbg_config &cfg, const Row *dR, uint64_t nR, const Row *dS, uint64_t nS, uint32_t sub,
                    int span, bool check_s, Row *sorted[2], bool msd_done[2], bool *s_outside, Workspace &w,
                    cudaStream_t st, JoinRun *run) {
    msd_done[0] = msd_done[1] = false;
    *s_outside = false;
    int lowbits = std::min(span, kLowBits), B = span - lowbits;
    if (B > 15) {
        B = 15;
        lowbits = span - B;
    }
    if (B < 1 || lowbits > kLowBitsMax) return TBG_OK;  // the LSD sort takes both
    RadixGeom g = radix_geometry_msd(nR, nS, sub, B, lowbits, w);
    if (check_s) g.s_range_max = (uint32_t)((1ull << span) - 1);
    int rc = ensure_radix_buffers(g, false, w);
    if (rc) return rc;
    Ctrl *ctrl = w.ctrl.as<Ctrl>();
    cudaError_t e;
    if ((e = cudaMemsetAsync(&ctrl->max_part_R, 0, 24, st)) != cudaSuccess) return cuda_error(e, "memset");
    if ((rc = part_histogram(0, g, dR, cfg, w, st, nullptr)) || (rc = part_histogram(1, g, dS, cfg, w, st, nullptr)))
        return rc;
    // the largest bucket of each relation decides between this sort and LSD;
    // S's keys outside R's range void the histograms
    unsigned long long *hm = static_cast<unsigned long long *>(w.host_small);
    if ((e = cudaMemcpyAsync(hm, &ctrl->max_part_R, 24, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_error(e, "bucket sizes");
    if (check_s && hm[2]) {
        *s_outside = true;
        return TBG_OK;
    }
    const unsigned long long maxp[2] = {hm[0], hm[1]};
    const Row *in[2] = {dR, dS};
    for (int rel = 0; rel < 2; rel++) {
        if (maxp[rel] > kBucketMax) continue;
        if ((rc = part_pass(rel, 1, g, in[rel], w, st, false)) || (rc = part_pass(rel, 2, g, in[rel], w, st, false)))
            return rc;
        const Row *part = (rel ? w.partS : w.partR).as<Row>();
        const uint64_t *base = (rel ? w.baseS : w.baseR).as<uint64_t>();
        if ((e = launch_bucket_sort(part, sorted[rel], base, (uint32_t)g.P, rel ? nS : nR, sub, lowbits, w.nsm,
                                    st)) != cudaSuccess)
            return cuda_error(e, "bucket sort");
        msd_done[rel] = true;
        mark_ev(w, cfg.timing != 0, 2 + rel, st);
    }
    run->B = B;
    run->passes = g.passes + 1;
    run->P = g.P;
    return TBG_OK;
}

int run_psm_join(const tbg_config &cfg, const Row *dR, uint64_t nR, const Row *dS, uint64_t nS,
                 tbg_row_out *d_rows, uint64_t cap, Workspace &w, cudaStream_t st, JoinRun *run) {
    const bool timing = cfg.timing != 0;
    cudaError_t e;
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
    ENSURE(w.aux[4], 64);
    ENSURE(w.aux[6], (merge_ctas(nR, nS) + 2) * 8);
#undef ENSURE
    Ctrl *ctrl = w.ctrl.as<Ctrl>();
    uint32_t *mm = w.aux[4].as<uint32_t>();  // min, max of R's keys, then of S's
    uint32_t *hm = static_cast<uint32_t *>(w.host_small);
    mark_ev(w, timing, 0, st);
    if ((e = cudaMemsetAsync(ctrl, 0, sizeof(Ctrl), st)) != cudaSuccess) return cuda_error(e, "memset");
    // R's key range decides the MSD geometry (S's keys usually lie inside it:
    // S's histogram checks that, so S's own range read is only needed when
    // they do not, or for the LSD sort)
    uint32_t rmin = 0, rmax = 0, smin = 0, smax = 0;
    bool have_s = false;
    auto read_range = [&](const Row *d, uint64_t n, uint32_t *lo, uint32_t *hi) -> int {
        if ((e = launch_key_range(d, n, mm, w.nsm, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(hm, mm, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return cuda_error(e, "key range");
        *lo = hm[0];
        *hi = hm[1];
        return TBG_OK;
    };
    auto span_of = [](uint32_t lo, uint32_t hi) { return hi > lo ? 32 - __builtin_clz(hi - lo) : 0; };
    int rc = read_range(dR, nR, &rmin, &rmax);
    if (rc) return rc;
    mark_ev(w, timing, 1, st);
    Row *sorted[2] = {w.aux[0].as<Row>(), w.aux[2].as<Row>()};
    bool msd_done[2] = {false, false};
    run->B = 8;
    run->P = 0;
    run->passes = 0;
    if (nR && nS) {
        bool s_outside = false;
        if ((rc = msd_sort(cfg, dR, nR, dS, nS, rmin, span_of(rmin, rmax), true, sorted, msd_done, &s_outside, w, st,
                           run)))
            return rc;
        if (s_outside) {  // both relations' range, histograms again
            if ((rc = read_range(dS, nS, &smin, &smax))) return rc;
            have_s = true;
            const uint32_t lo = std::min(rmin, smin), hi = std::max(rmax, smax);
            if ((rc = msd_sort(cfg, dR, nR, dS, nS, lo, span_of(lo, hi), false, sorted, msd_done, &s_outside, w,
                               st, run)))
                return rc;
        }
    }
    const Row *sR = sorted[0], *sS = sorted[1];
    int pr = 0, ps = 0;
    if (!msd_done[0]) {
        if ((rc = lsd_sort_chunked(dR, nR, rmin, rmax, w.aux[0], w.aux[1], w, st, &sR, &pr))) return rc;
        mark_ev(w, timing, 2, st);
    }
    if (!msd_done[1]) {
        if (!have_s && (rc = read_range(dS, nS, &smin, &smax))) return rc;
        if ((rc = lsd_sort_chunked(dS, nS, smin, smax, w.aux[2], w.aux[3], w, st, &sS, &ps))) return rc;
        mark_ev(w, timing, 3, st);
    }
    e = launch_merge_join(sR, nR, sS, nS, w.aux[6].as<uint64_t>(), &ctrl->matches, &ctrl->rows, d_rows,
                          d_rows ? cap : 0, cfg.materialize != 0, st);
    if (e != cudaSuccess) return cuda_error(e, "merge join");
    mark_ev(w, timing, 4, st);
    if (!msd_done[0] || !msd_done[1]) run->passes = std::max(run->passes, std::max(pr, ps));
    run->timed = timing;
    return TBG_OK;
}

}  // namespace tbg
