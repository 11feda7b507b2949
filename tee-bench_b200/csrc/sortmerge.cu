// Sort-merge joins for sm_100a.
//
// RSM (Joins/radix_sortmerge_join.c:74-100): the radix partitions of RHO,
// then per work item R's chunk is sorted in shared memory over the key bits
// that vary in it (one counting pass, or a stable LSD radix sort when they
// span more than 12 bits) and S is sorted in tiles and merged against it.
// Count-only joins sort S in 16384-row tiles by a counting sort ranked
// against R's key range (k_join_rsm_count); materialising joins sort packed
// (key, payload) words in 4096-row tiles (k_join_rsm).  PSM
// (Joins/psm/parallel_sortmerge_join.h:61-111): R and S are sorted globally
// (the MSD bucket sort or the LSD passes of sortpass.cu) and merged
// (k_merge_count, k_merge_join).
//
// The merges are merge paths (Green, McColl, Bader 2012); diagonals split the
// path evenly over threads (and, for PSM, over CTAs).  The count-only merges
// take R[i] before S[j] iff R[i].key <= S[j].key, so when S[j] is taken every
// R row of its key is behind it and a running count of the last R key's rows
// gives its matches.  The materialising merges take R[i] first iff
// R[i].key < S[j].key, so S[j]'s matches are the run of equal R keys from the
// current R position, which it emits.  The reference's merge()
// (Joins/radix_sortmerge_join.c:40-71, parallel_sortmerge_join.h:18-51) has
// unbounded inner loops and a stale S cursor that miscount duplicates and
// misses; these merges count exactly the equi-join.
#include <algorithm>

#include "part_dev.cuh"

namespace tbg {

__device__ __forceinline__ uint64_t pack_row(uint32_t k, uint32_t p) { return ((uint64_t)k << 32) | p; }
__device__ __forceinline__ uint32_t row_key(uint64_t x) { return (uint32_t)(x >> 32); }
__device__ __forceinline__ uint32_t row_pay(uint64_t x) { return (uint32_t)x; }

// Skewed layout of a sorted tile: row i at i + i / 16, so threads that walk
// merge-path segments about 8 rows apart hit different banks.
__device__ __forceinline__ uint32_t pad16(uint32_t i) { return i + (i >> 4); }
__host__ __device__ constexpr uint32_t padded_rows(uint32_t n) { return n + n / 16 + 1; }

// The sorts below run on packed rows (key in the high 32 bits) or on bare
// keys (count-only RSM).  Bare keys are 4 bytes, one bank each, so their
// skewed layout puts key i at i + i / 8 for the same effect.
__device__ __forceinline__ uint32_t elem_key(uint64_t x) { return row_key(x); }
__device__ __forceinline__ uint32_t elem_key(uint32_t x) { return x; }
template <typename T>
__device__ __forceinline__ uint32_t skew(uint32_t i) {
    return sizeof(T) == 8 ? pad16(i) : i + (i >> 3);
}
template <typename T>
__host__ __device__ constexpr uint32_t skewed_size(uint32_t n) {
    return sizeof(T) == 8 ? padded_rows(n) : n + n / 8 + 1;
}

// Block-wide stable LSD radix sort of n <= THREADS * 8 packed rows (by their
// high 32 bits) or bare keys in shared memory.  Only the key bits that differ
// inside the tile are sorted, 8 per pass.  In a pass, thread (w, lane) holds
// rows e = w * 256 + i * 32 + lane (i < 8); a row's rank counts the rows of
// the same digit before it in that order (per-warp counters advanced slot by
// slot, ballot-built peer masks inside a slot), so every pass is stable.  `a` holds
// the rows, `b` is scratch for n rows, `cnt` 256 * THREADS / 32 counters,
// `scratch` THREADS / 32 + 1 words, `red` 2 words.  `a` is read in plain
// layout; the sorted rows are left in the skewed layout (skew<T>) in the
// returned buffer, a or b, each sized skewed_size<T>(n).
template <int THREADS, typename T>
__device__ T *block_radix_sort(T *a, T *b, uint32_t n, uint16_t *cnt, uint64_t *scratch, uint32_t *red) {
    constexpr int NW = THREADS / 32, ITEMS = 8, C = 256 * NW / THREADS;
    static_assert(THREADS * ITEMS <= 65535 && 256 * NW % THREADS == 0 && NW % C == 0,
                  "16-bit counters; a thread's counters belong to one digit");
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tid == 0) {
        red[0] = 0;
        red[1] = ~0u;
    }
    __syncthreads();
    uint32_t vor = 0, vand = ~0u;
    for (uint32_t e = tid; e < n; e += THREADS) {
        const uint32_t k = elem_key(a[e]);
        vor |= k;
        vand &= k;
    }
    for (int o = 16; o > 0; o >>= 1) {
        vor |= __shfl_xor_sync(0xffffffffu, vor, o);
        vand &= __shfl_xor_sync(0xffffffffu, vand, o);
    }
    if (lane == 0) {
        atomicOr(&red[0], vor);
        atomicAnd(&red[1], vand);
    }
    __syncthreads();
    const uint32_t varying = red[0] & ~red[1];
    __syncthreads();  // red is reused by the next call
    T *src = a, *dst = b;
    if (!varying) {  // every key equal: already sorted, only the layout changes
        for (uint32_t e = tid; e < n; e += THREADS) b[skew<T>(e)] = a[e];
        __syncthreads();
        return b;
    }
    const int lo = __ffs(varying) - 1, hi = 31 - __clz(varying);
    for (int shift = lo; shift <= hi; shift += 8) {
        const bool last = shift + 8 > hi;
        for (int i = tid; i < 256 * NW; i += THREADS) cnt[i] = 0;
        __syncthreads();
        // only the ranks stay in registers across the scan; rows and digits
        // are read again from src for the scatter
        uint32_t r[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const uint32_t e = (uint32_t)w * 32 * ITEMS + i * 32 + lane;
            const bool valid = e < n;
            const uint32_t d = valid ? (elem_key(src[e]) >> shift) & 255 : 256;
            const unsigned peers = warp_peers9(d);
            uint32_t base = 0;
            if (valid) base = cnt[w * 256 + d];  // warp-major: lanes with different digits hit different banks
            __syncwarp();
            if (valid && (peers & lanemask_lt()) == 0) cnt[w * 256 + d] = (uint16_t)(base + __popc(peers));
            __syncwarp();
            r[i] = base + __popc(peers & lanemask_lt());
        }
        __syncthreads();
        // exclusive scan over (digit, warp), digit-major: thread t owns the C
        // counters of digit t * C / NW for warps (t * C) % NW ...
        const int dgt = tid * C / NW, w0 = (tid * C) % NW;
        uint32_t sum = 0;
#pragma unroll
        for (int c = 0; c < C; c++) sum += cnt[(w0 + c) * 256 + dgt];
        uint64_t tot;
        uint32_t run = (uint32_t)block_excl_scan<THREADS>(sum, &tot, scratch);
#pragma unroll
        for (int c = 0; c < C; c++) {
            const uint32_t x = cnt[(w0 + c) * 256 + dgt];
            cnt[(w0 + c) * 256 + dgt] = (uint16_t)run;
            run += x;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const uint32_t e = (uint32_t)w * 32 * ITEMS + i * 32 + lane;
            if (e < n) {
                const T x = src[e];
                const uint32_t p = cnt[w * 256 + ((elem_key(x) >> shift) & 255)] + r[i];
                dst[last ? skew<T>(p) : p] = x;
            }
        }
        __syncthreads();
        T *t = src;
        src = dst;
        dst = t;
    }
    return src;
}

// Widest key field (bits) that load_sorted sorts in one counting pass.
constexpr int COUNT_SORT_BITS = 12;

// Loads rows [off, off + n) (n <= THREADS * 8) and sorts them by key; returns
// the buffer holding the sorted rows in the skewed layout (s, or tmp after a
// multi-pass sort).  Every thread issues its 8 loads before the first use.
// When the key bits that vary in the tile span at most COUNT_SORT_BITS
// (12 at the 2^27-key, 15-bit radix workloads), one counting pass sorts
// them: ranks from shared atomics on 2^span bins kept in tmp, an exclusive
// scan of the bins, then each row goes straight from registers to its
// place.  Rows with equal keys then sit in no particular order, which the
// merge does not need (a join's rows are a multiset).  Wider spans take
// block_radix_sort.
template <int THREADS>
__device__ uint64_t *load_sorted(const Row *__restrict__ src, uint64_t off, uint32_t n, uint64_t *s, uint64_t *tmp,
                                 uint16_t *cnt, uint64_t *scratch, uint32_t *red) {
    constexpr int ITEMS = 8;
    const int tid = threadIdx.x, lane = tid & 31;
    const uint2 *v = reinterpret_cast<const uint2 *>(src) + off;
    if (tid == 0) {
        red[0] = 0;
        red[1] = ~0u;
    }
    // tmp (sized for THREADS * 8 skewed rows) holds the payloads, parked
    // there to free registers, and the counting pass's 2^span <= 4096 bins
    uint32_t *c32 = reinterpret_cast<uint32_t *>(tmp);
    uint32_t *pay = c32 + (1u << COUNT_SORT_BITS);
    uint32_t key[ITEMS];
    uint32_t vor = 0, vand = ~0u;
    {
        uint2 x[ITEMS];
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const uint32_t e = i * THREADS + tid;
            if (e < n) x[i] = v[e];
        }
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const uint32_t e = i * THREADS + tid;
            key[i] = x[i].x;
            if (e < n) {
                pay[e] = x[i].y;
                vor |= x[i].x;
                vand &= x[i].x;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        vor |= __shfl_xor_sync(0xffffffffu, vor, o);
        vand &= __shfl_xor_sync(0xffffffffu, vand, o);
    }
    __syncthreads();  // red initialised
    if (lane == 0) {
        atomicOr(&red[0], vor);
        atomicAnd(&red[1], vand);
    }
    __syncthreads();
    const uint32_t varying = red[0] & ~red[1];
    const int lo = varying ? __ffs(varying) - 1 : 0;
    const int span = varying ? 32 - __clz(varying) - lo : 0;
    if (span > COUNT_SORT_BITS) {
#pragma unroll
        for (int i = 0; i < ITEMS; i++) {
            const uint32_t e = i * THREADS + tid;
            if (e < n) s[e] = pack_row(key[i], pay[e]);
        }
        __syncthreads();  // also: red is reused by the sort
        return block_radix_sort<THREADS, uint64_t>(s, tmp, n, cnt, scratch, red);
    }
    const uint32_t bins = 1u << span;
    for (uint32_t b = tid; b < bins; b += THREADS) c32[b] = 0;
    __syncthreads();
    uint32_t r[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        const bool valid = i * THREADS + tid < n;
        const uint32_t d = valid ? (key[i] >> lo) & (bins - 1) : 0;
        r[i] = rank_warp(c32, d, valid, warp_has_dups(d, valid));
    }
    __syncthreads();
    {
        // exclusive scan of the bins; thread t owns bins [t * per, (t + 1) * per)
        const uint32_t per = (bins + THREADS - 1) / THREADS;
        const uint32_t b0 = min(bins, tid * per), b1 = min(bins, b0 + per);
        uint32_t sum = 0;
        for (uint32_t b = b0; b < b1; b++) sum += c32[b];
        uint64_t tot;
        uint32_t run = (uint32_t)block_excl_scan<THREADS>(sum, &tot, scratch);
        for (uint32_t b = b0; b < b1; b++) {
            const uint32_t c = c32[b];
            c32[b] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < ITEMS; i++)
        if (i * THREADS + tid < n)
            s[pad16(c32[(key[i] >> lo) & (bins - 1)] + r[i])] = pack_row(key[i], pay[i * THREADS + tid]);
    __syncthreads();
    return s;
}

// Merge-path split of diagonal d over sorted arrays A (na) and B (nb):
// the number of A elements among the first d of the merged order, where A[i]
// precedes B[j] iff key(A[i]) < key(B[j]).
// With A_FIRST, A[i] precedes B[j] iff key(A[i]) <= key(B[j]) instead.
template <bool A_FIRST = false, class GetA, class GetB>
__device__ __forceinline__ uint64_t merge_split(uint64_t d, uint64_t na, uint64_t nb, GetA ka, GetB kb) {
    uint64_t lo = d > nb ? d - nb : 0, hi = d < na ? d : na;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (A_FIRST ? ka(mid) <= kb(d - mid - 1) : ka(mid) < kb(d - mid - 1)) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// RSM: per work item, sorted R chunk in shared memory against sorted S tiles.
// ---------------------------------------------------------------------------
constexpr int RSM_THREADS = 512;
constexpr int RSM_STILE = RSM_THREADS * 8;  // one radix-sorted S tile

// R rows, an S tile, sort scratch (each in the skewed layout), 16-bit sort
// counters
size_t rsm_smem_bytes(int capR) {
    return ((size_t)padded_rows(capR) + padded_rows(RSM_STILE) + padded_rows(std::max(capR, RSM_STILE))) * 8 +
           256 * (RSM_THREADS / 32) * 2;
}

template <bool MAT>
__global__ void __launch_bounds__(RSM_THREADS, 2) k_join_rsm(JoinArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t *Rs = reinterpret_cast<uint64_t *>(smem);
    uint64_t *Sbuf = Rs + padded_rows(a.capR);
    uint64_t *tmp = Sbuf + padded_rows(RSM_STILE);
    uint16_t *cnt = reinterpret_cast<uint16_t *>(tmp + padded_rows(max(a.capR, RSM_STILE)));
    __shared__ uint32_t s_item;
    __shared__ unsigned long long s_base;
    __shared__ uint64_t scan_scratch[RSM_THREADS / 32 + 1];
    __shared__ uint32_t red[2];
    const int tid = threadIdx.x;
    const unsigned nitems = *a.err ? 0u : *a.nitems;  // a planner error leaves the item list unusable
    unsigned long long local = 0;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(a.item_ctr, 1u);
        __syncthreads();
        const uint32_t it = s_item;
        if (it >= nitems) break;
        const Item m = a.items[it];
        const uint32_t nr = m.r_len;
        if (load_sorted<RSM_THREADS>(a.R, m.r_off, nr, Rs, tmp, cnt, scan_scratch, red) != Rs) {
            for (uint32_t q = tid; q < padded_rows(nr); q += RSM_THREADS) Rs[q] = tmp[q];  // sorted R stays in Rs
            __syncthreads();
        }
        for (uint64_t s0 = 0; s0 < m.s_len; s0 += RSM_STILE) {
            const uint32_t ns = (uint32_t)umin64(RSM_STILE, m.s_len - s0);
            const uint64_t *Ss = load_sorted<RSM_THREADS>(a.S, m.s_off + s0, ns, Sbuf, tmp, cnt, scan_scratch, red);
            // each thread walks an equal share of the merge path of R[0..nr) and S[0..ns)
            const uint32_t L = nr + ns;
            const uint32_t per = (L + RSM_THREADS - 1) / RSM_THREADS;
            const uint32_t d0 = min(L, tid * per), d1 = min(L, d0 + per);
            auto kr = [&](uint32_t i) { return row_key(Rs[pad16(i)]); };
            auto ks = [&](uint32_t j) { return row_key(Ss[pad16(j)]); };
            uint32_t i;
            {
                uint32_t lo = d0 > ns ? d0 - ns : 0, hi = min(d0, nr);
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (kr(mid) < ks(d0 - mid - 1)) lo = mid + 1;
                    else hi = mid;
                }
                i = lo;
            }
            uint32_t j = d0 - i;
            // pass 1: count this thread's matches.  The current keys stay in
            // registers; at a side's end they read the padded slot past its
            // last row (inside the buffer, never used).
            uint32_t cnt = 0;
            {
                uint32_t ii = i, jj = j;
                uint32_t rk = kr(ii), sk = ks(jj);
                uint32_t last_key = 0, last_cnt = 0;
                bool have = false;
                for (uint32_t d = d0; d < d1; d++) {
                    if (ii < nr && (jj >= ns || rk < sk)) {
                        rk = kr(++ii);
                    } else {
                        if (!have || sk != last_key) {
                            last_cnt = 0;
                            if (ii < nr && rk == sk)
                                for (uint32_t q = ii; q < nr && kr(q) == sk; q++) last_cnt++;
                            last_key = sk;
                            have = true;
                        }
                        cnt += last_cnt;
                        sk = ks(++jj);
                    }
                }
            }
            local += cnt;
            if (MAT) {
                uint64_t tot;
                const uint64_t off = block_excl_scan<RSM_THREADS>(cnt, &tot, scan_scratch);
                if (tid == 0) s_base = tot ? atomicAdd(a.rows_ctr, (unsigned long long)tot) : 0;
                __syncthreads();
                uint64_t pos = s_base + off;
                for (uint32_t d = d0; d < d1; d++) {
                    if (i < nr && (j >= ns || kr(i) < ks(j))) {
                        i++;
                    } else {
                        const uint32_t k = ks(j);
                        for (uint32_t q = i; q < nr && kr(q) == k; q++) {
                            if (pos < a.cap) {
                                tbg_row_out o;
                                o.key = k;
                                o.Rpayload = row_pay(Rs[pad16(q)]);
                                o.Spayload = row_pay(Ss[pad16(j)]);
                                a.out[pos] = o;
                            }
                            pos++;
                        }
                        j++;
                    }
                }
            }
            __syncthreads();  // S tile reused
        }
    }
    const unsigned long long ws = warp_sum_u64(local);
    if ((tid & 31) == 0 && ws) atomicAdd(a.matches, ws);
}

// Count-only RSM works on bare keys (4 bytes in shared memory instead of 8),
// which leaves room to load the next S tile's keys into registers while the
// current tile is merged.

// Keys of rows [off, off + n) (n <= THREADS * 8): key[i] is row i * THREADS +
// tid.  All loads are issued before the first use.
template <int THREADS>
__device__ __forceinline__ void load_keys(const Row *__restrict__ src, uint64_t off, uint32_t n, uint32_t (&key)[8]) {
    const uint2 *v = reinterpret_cast<const uint2 *>(src) + off;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const uint32_t e = i * THREADS + threadIdx.x;
        if (e < n) key[i] = __ldcs(v + e).x;
    }
}

// cnt[0, bins) -> exclusive offsets in place; returns the total.  Ends with
// the counters written but not yet synchronised.  When bins is a multiple of
// 4 * THREADS (and cnt 16-byte aligned) a thread's run of bins moves as
// 16-byte words: strided 4-byte reads of the runs conflict (8-way for runs
// of 8 bins).
template <int THREADS>
__device__ __forceinline__ uint32_t scan_bins(uint32_t *cnt, uint32_t bins, uint64_t *scratch) {
    const uint32_t per = (bins + THREADS - 1) / THREADS;
    if (per % 4 == 0) {
        uint4 *c4 = reinterpret_cast<uint4 *>(cnt) + threadIdx.x * (per / 4);
        uint32_t sum = 0;
        for (uint32_t q = 0; q < per / 4; q++) {
            const uint4 c = c4[q];
            sum += c.x + c.y + c.z + c.w;
        }
        uint64_t tot;
        uint32_t run = (uint32_t)block_excl_scan<THREADS>(sum, &tot, scratch);
        for (uint32_t q = 0; q < per / 4; q++) {
            const uint4 c = c4[q];
            uint4 o;
            o.x = run;
            o.y = o.x + c.x;
            o.z = o.y + c.y;
            o.w = o.z + c.z;
            run = o.w + c.w;
            c4[q] = o;
        }
        return (uint32_t)tot;
    }
    const uint32_t b0 = min(bins, threadIdx.x * per), b1 = min(bins, b0 + per);
    uint32_t sum = 0;
    for (uint32_t b = b0; b < b1; b++) sum += cnt[b];
    uint64_t tot;
    uint32_t run = (uint32_t)block_excl_scan<THREADS>(sum, &tot, scratch);
    for (uint32_t b = b0; b < b1; b++) {
        const uint32_t c = cnt[b];
        cnt[b] = run;
        run += c;
    }
    return (uint32_t)tot;
}

// Sorts the n keys held as load_keys left them into `out` (skewed 4-byte
// layout): one counting pass on the 2^COUNT_SORT_BITS counters `c32`
// (16-byte aligned) when the varying bits span at most COUNT_SORT_BITS, else
// the stable LSD sort through `tmp`.  `out` and `tmp` hold
// skewed_size<uint32_t>(THREADS * 8) keys.
template <int THREADS>
__device__ void sort_keys(const uint32_t (&key)[8], uint32_t n, uint32_t *out, uint32_t *tmp, uint32_t *c32,
                          uint16_t *cnt, uint64_t *scratch, uint32_t *red) {
    constexpr int ITEMS = 8;
    const int tid = threadIdx.x, lane = tid & 31;
    if (tid == 0) {
        red[0] = 0;
        red[1] = ~0u;
    }
    uint32_t vor = 0, vand = ~0u;
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        if (i * THREADS + tid < n) {
            vor |= key[i];
            vand &= key[i];
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        vor |= __shfl_xor_sync(0xffffffffu, vor, o);
        vand &= __shfl_xor_sync(0xffffffffu, vand, o);
    }
    __syncthreads();  // red initialised
    if (lane == 0) {
        atomicOr(&red[0], vor);
        atomicAnd(&red[1], vand);
    }
    __syncthreads();
    const uint32_t varying = red[0] & ~red[1];
    const int lo = varying ? __ffs(varying) - 1 : 0;
    const int span = varying ? 32 - __clz(varying) - lo : 0;
    if (span > COUNT_SORT_BITS) {
#pragma unroll
        for (int i = 0; i < ITEMS; i++)
            if (i * THREADS + tid < n) tmp[i * THREADS + tid] = key[i];
        __syncthreads();  // also: red is reused by the sort
        const uint32_t *res = block_radix_sort<THREADS, uint32_t>(tmp, out, n, cnt, scratch, red);
        if (res != out) {
            for (uint32_t q = tid; q < skewed_size<uint32_t>(n); q += THREADS) out[q] = res[q];
            __syncthreads();
        }
        return;
    }
    const uint32_t bins = 1u << span;
    for (uint32_t b = tid; b < bins; b += THREADS) c32[b] = 0;
    __syncthreads();
    uint32_t r[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; i++) {
        const bool valid = i * THREADS + tid < n;
        const uint32_t d = valid ? (key[i] >> lo) & (bins - 1) : 0;
        r[i] = rank_warp(c32, d, valid, warp_has_dups(d, valid));
    }
    __syncthreads();
    scan_bins<THREADS>(c32, bins, scratch);
    __syncthreads();
#pragma unroll
    for (int i = 0; i < ITEMS; i++)
        if (i * THREADS + tid < n) out[skew<uint32_t>(c32[(key[i] >> lo) & (bins - 1)] + r[i])] = key[i];
    __syncthreads();
}

// Matches of this thread's share of the merge path of sorted keys A (na, the
// R chunk) and B (nb, an S tile), skewed 4-byte layout.  Here the merged
// order takes A[i] before B[j] iff A[i] <= B[j], so when B[j] is taken every
// A key equal to it is behind: `run` counts the A keys equal to the last A
// key taken (`pk`), and B[j] matches run of them when its key is pk.  No
// step walks a run of equal keys, so the steps cost the same under skew.
template <int THREADS>
__device__ __forceinline__ uint32_t merge_count(const uint32_t *A, uint32_t na, const uint32_t *B, uint32_t nb) {
    const uint32_t L = na + nb;
    const uint32_t per = (L + THREADS - 1) / THREADS;
    const uint32_t d0 = min(L, threadIdx.x * per), d1 = min(L, d0 + per);
    auto ka = [&](uint32_t i) { return A[skew<uint32_t>(i)]; };
    auto kb = [&](uint32_t j) { return B[skew<uint32_t>(j)]; };
    uint32_t lo = d0 > nb ? d0 - nb : 0, hi = min(d0, na);
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (ka(mid) <= kb(d0 - mid - 1)) lo = mid + 1;
        else hi = mid;
    }
    uint32_t i = lo, j = d0 - lo;
    uint32_t pk = 0, run = 0;  // with no A key behind, run 0 matches nothing
    if (i > 0 && d0 < d1) {
        // the A keys equal to A[i - 1] end at i - 1: a short walk back, then
        // a binary search for the first of them
        pk = ka(i - 1);
        uint32_t q = i - 1;
        for (int w = 0; w < 4 && q > 0 && ka(q - 1) == pk; w++) q--;
        if (q > 0 && ka(q - 1) == pk) {
            uint32_t l = 0, h = q - 1;
            while (l < h) {
                const uint32_t m = (l + h) >> 1;
                if (ka(m) < pk) l = m + 1;
                else h = m;
            }
            q = l;
        }
        run = i - q;
    }
    // the current keys stay in registers; at a side's end they read the
    // padding slot past its last key (inside the buffer, never used)
    uint32_t ak = ka(i), bk = kb(j);
    uint32_t cnt = 0;
    for (uint32_t d = d0; d < d1; d++) {
        if (i < na && (j >= nb || ak <= bk)) {
            run = ak == pk ? run + 1 : 1;
            pk = ak;
            ak = ka(++i);
        } else {
            if (bk == pk) cnt += run;
            bk = kb(++j);
        }
    }
    return cnt;
}

constexpr uint32_t RSM_KEYS = skewed_size<uint32_t>(RSM_STILE);
// S tiles of the ranged counting sort (below) and the bins it ranks on.
constexpr uint32_t RSM_SBIG = RSM_STILE * 4;
constexpr uint32_t RSM_SBIG_KEYS = skewed_size<uint32_t>(RSM_SBIG);
constexpr uint32_t RSM_BINS = 1u << COUNT_SORT_BITS;
static_assert(RSM_BINS % (4 * RSM_THREADS) == 0, "the rounded bin count fits");
// the per-tile path reuses the S buffer: 4096 sorted keys, the sort's
// scratch keys and its 16-bit counters
static_assert(2 * RSM_KEYS + 256 * (RSM_THREADS / 32) / 2 <= RSM_SBIG_KEYS, "per-tile buffers fit the S buffer");

size_t rsm_count_smem_bytes() { return (size_t)(RSM_KEYS + RSM_SBIG_KEYS + RSM_BINS) * 4; }

// One read of S rows [off, off + ns) for the ranged counting sort.  Rows whose
// key lies in [rmin, rmin + rspan] (R's key range) have the digit
// (key - rmin) >> shift: RANK false counts the digits, RANK true takes each
// row's slot from its digit's running offset and stores the key there.  Rows
// outside R's range cannot match and stay out of the sorted tile.  All keys of
// a work item share their low `shift` bits (the partition's radix), so keys
// in range have distinct digits for distinct values and the slots sort them;
// equal keys sit in any order among themselves.  The counting read keeps S in
// L2 (ld.global.cg) for the ranking read, which streams it (ld.global.cs).
template <bool RANK, bool FULL>
__device__ __forceinline__ void rsm_ranged_pass(const Row *__restrict__ S, uint64_t off, uint32_t ns, uint32_t rmin,
                                                uint32_t rspan, int shift, uint32_t *cnt, uint32_t *Sk) {
    const uint2 *v = reinterpret_cast<const uint2 *>(S) + off;
    constexpr uint32_t BATCH = RSM_THREADS * 8;
    if (FULL) ns = RSM_SBIG;
    for (uint32_t b0 = 0; b0 < ns; b0 += BATCH) {
        uint32_t k[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const uint32_t e = b0 + i * RSM_THREADS + threadIdx.x;
            k[i] = 0;
            if (FULL || e < ns) k[i] = RANK ? __ldcs(v + e).x : __ldcg(v + e).x;
        }
        const bool dup =
            warp_has_dups((k[0] - rmin) >> shift, (FULL || b0 + threadIdx.x < ns) && k[0] - rmin <= rspan);
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const uint32_t dk = k[i] - rmin;
            const bool in = (FULL || b0 + i * RSM_THREADS + threadIdx.x < ns) && dk <= rspan;
            const uint32_t slot = rank_warp(cnt, in ? dk >> shift : 0u, in, dup);
            if (RANK && in) Sk[skew<uint32_t>(slot)] = k[i];
        }
    }
}

// Count-only RSM for items with r_len <= RSM_STILE.  The R chunk's keys are
// sorted once (sort_keys).  When R's keys span at most RSM_BINS digits above
// the partition's radix bits, S is sorted in tiles of RSM_SBIG rows by the
// ranged counting sort (a counting read, a scan of the bins, a ranking read
// that places the keys) and each sorted tile is merged against R.  Otherwise
// S tiles of RSM_STILE keys are sorted by sort_keys, tile k + 1's keys
// loading while tile k merges.
__global__ void __launch_bounds__(RSM_THREADS, 2) k_join_rsm_count(JoinArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t *bins_cnt = reinterpret_cast<uint32_t *>(smem);  // 16-byte aligned for the scan
    uint32_t *Rk = bins_cnt + RSM_BINS;
    uint32_t *Sk = Rk + RSM_KEYS;
    uint32_t *tmp = Sk + RSM_KEYS;  // per-tile sorts: scratch keys and counters inside the S buffer
    uint16_t *cnt = reinterpret_cast<uint16_t *>(tmp + RSM_KEYS);
    __shared__ uint32_t s_item;
    __shared__ uint64_t scan_scratch[RSM_THREADS / 32 + 1];
    __shared__ uint32_t red[2];
    const int tid = threadIdx.x;
    const int shift = a.hash_shift;
    const unsigned nitems = *a.err ? 0u : *a.nitems;  // a planner error leaves the item list unusable
    unsigned long long local = 0;
    uint32_t key[8];
    for (;;) {
        if (tid == 0) s_item = atomicAdd(a.item_ctr, 1u);
        __syncthreads();
        const uint32_t it = s_item;
        if (it >= nitems) break;
        const Item m = a.items[it];
        const uint32_t nr = min(m.r_len, (uint32_t)RSM_STILE);  // the planner's capR is RSM_STILE
        __syncthreads();  // s_item read by every thread before thread 0 rewrites it
        if (nr == 0 || m.s_len == 0) continue;
        load_keys<RSM_THREADS>(a.R, m.r_off, nr, key);
        sort_keys<RSM_THREADS>(key, nr, Rk, tmp, bins_cnt, cnt, scan_scratch, red);
        const uint32_t rmin = Rk[0], rspan = Rk[skew<uint32_t>(nr - 1)] - rmin;
        if ((rspan >> shift) < RSM_BINS) {
            // digits in [0, bins); above 1024 bins the count runs to a
            // multiple of 4 * RSM_THREADS (the extra bins stay empty) so the
            // scan reads 16-byte words
            const uint32_t bins0 = (rspan >> shift) + 1;
            const uint32_t bins = bins0 > 1024 ? (bins0 + 4 * RSM_THREADS - 1) & ~(4u * RSM_THREADS - 1) : bins0;
            for (uint64_t s0 = 0; s0 < m.s_len; s0 += RSM_SBIG) {
                const uint32_t ns = (uint32_t)umin64(RSM_SBIG, m.s_len - s0);
                for (uint32_t b = tid; b < bins; b += RSM_THREADS) bins_cnt[b] = 0;
                __syncthreads();
                if (ns == RSM_SBIG) rsm_ranged_pass<false, true>(a.S, m.s_off + s0, ns, rmin, rspan, shift, bins_cnt, Sk);
                else rsm_ranged_pass<false, false>(a.S, m.s_off + s0, ns, rmin, rspan, shift, bins_cnt, Sk);
                __syncthreads();
                const uint32_t nin = scan_bins<RSM_THREADS>(bins_cnt, bins, scan_scratch);
                __syncthreads();
                if (ns == RSM_SBIG) rsm_ranged_pass<true, true>(a.S, m.s_off + s0, ns, rmin, rspan, shift, bins_cnt, Sk);
                else rsm_ranged_pass<true, false>(a.S, m.s_off + s0, ns, rmin, rspan, shift, bins_cnt, Sk);
                __syncthreads();
                local += merge_count<RSM_THREADS>(Rk, nr, Sk, nin);
                __syncthreads();  // Sk and the bins are rewritten by the next tile
            }
            continue;
        }
        uint32_t ns = (uint32_t)umin64(RSM_STILE, m.s_len);
        load_keys<RSM_THREADS>(a.S, m.s_off, ns, key);
        for (uint64_t s0 = 0; s0 < m.s_len;) {
            sort_keys<RSM_THREADS>(key, ns, Sk, tmp, bins_cnt, cnt, scan_scratch, red);
            const uint64_t s1 = s0 + ns;
            const uint32_t ns_next = (uint32_t)umin64(RSM_STILE, m.s_len - s1);
            if (ns_next) load_keys<RSM_THREADS>(a.S, m.s_off + s1, ns_next, key);  // in flight during the merge
            local += merge_count<RSM_THREADS>(Rk, nr, Sk, ns);
            __syncthreads();  // Sk and tmp are rewritten by the next tile
            s0 = s1;
            ns = ns_next;
        }
    }
    const unsigned long long ws = warp_sum_u64(local);
    if ((tid & 31) == 0 && ws) atomicAdd(a.matches, ws);
}

// Resident CTAs per SM of the RSM join kernel a launch would use.
// RSM's planner caps R chunks at RSM_STILE rows, so counting joins always
// take the bare-key kernel and k_join_rsm runs materialising only.
int rsm_ctas_per_sm(int capR, bool materialize) {
    int n = 0;
    if (!materialize) {
        const size_t smem = rsm_count_smem_bytes();
        smem_limit((const void *)k_join_rsm_count, smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_join_rsm_count, RSM_THREADS, smem);
    } else {
        const size_t smem = rsm_smem_bytes(capR);
        smem_limit((const void *)k_join_rsm<true>, smem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_join_rsm<true>, RSM_THREADS, smem);
    }
    return n < 1 ? 1 : n;
}

cudaError_t launch_join_rsm(const JoinArgs &a, bool materialize, int grid, cudaStream_t st) {
    if (a.capR > RSM_STILE) return cudaErrorInvalidValue;  // one shared-memory tile of R per item
    cudaError_t e;
    if (!materialize) {
        const size_t smem = rsm_count_smem_bytes();
        if ((e = smem_limit((const void *)k_join_rsm_count, smem)) !=
            cudaSuccess)
            return e;
        k_join_rsm_count<<<grid, RSM_THREADS, smem, st>>>(a);
    } else {
        const size_t smem = rsm_smem_bytes(a.capR);
        if ((e = smem_limit((const void *)k_join_rsm<true>, smem)) !=
            cudaSuccess)
            return e;
        k_join_rsm<true><<<grid, RSM_THREADS, smem, st>>>(a);
    }
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// PSM: the key range of a relation in one read (the sort's passes cover the
// bits of key - min that vary), then the merge join of the sorted relations.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512) k_key_range(const Row *__restrict__ in, uint64_t n, uint32_t *minmax) {
    uint32_t lo = 0xFFFFFFFFu, hi = 0;
    const uint64_t np = n / 2;  // row pairs, read as 16-byte vectors when the start is aligned
    const bool vec = (reinterpret_cast<uintptr_t>(in) & 15) == 0;
    const uint64_t stride = (uint64_t)gridDim.x * 512;
    if (vec) {
        const uint4 *v = reinterpret_cast<const uint4 *>(in);
        for (uint64_t i = (uint64_t)blockIdx.x * 512 + threadIdx.x; i < np; i += stride) {
            const uint4 x = ldg_stream(v + i);
            lo = min(lo, min(x.x, x.z));
            hi = max(hi, max(x.x, x.z));
        }
        if (blockIdx.x == 0 && threadIdx.x == 0 && (n & 1)) {
            lo = min(lo, in[n - 1].key);
            hi = max(hi, in[n - 1].key);
        }
    } else {
        for (uint64_t i = (uint64_t)blockIdx.x * 512 + threadIdx.x; i < n; i += stride) {
            const uint32_t k = in[i].key;
            lo = min(lo, k);
            hi = max(hi, k);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&minmax[0], lo);
        atomicMax(&minmax[1], hi);
    }
}

// minmax[0] = smallest key, minmax[1] = largest (0xFFFFFFFF, 0 for no rows).
cudaError_t launch_key_range(const Row *in, uint64_t n, uint32_t *minmax, int nsm, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(minmax, 0xFF, 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(minmax + 1, 0, 4, st);
    if (e != cudaSuccess || !n) return e;
    const uint64_t g = umin64((n / 2 + 511) / 512 + 1, (uint64_t)nsm * 4);
    k_key_range<<<(unsigned)g, 512, 0, st>>>(in, n, minmax);
    count_launch();
    return cudaGetLastError();
}

// Merge join of sorted R (nr) and sorted S (ns).  k_merge_splits finds, for
// every CTA boundary c * D, the merge-path split (one thread per boundary);
// CTA c then loads R[i_c, i_c+1) and S[j_c, j_c+1) (D rows together) into
// one shared array, each thread issuing a batch of loads before its first
// shared store, splits its D diagonals evenly over threads and walks them.
// Materialising (k_merge_join<true>): a run of equal R keys that continues
// past the tile is finished in global memory.  Count-only (k_merge_count): a
// run of equal R keys that starts before the tile is found by walking back.
// Merge tile shapes (build options for A/B timing).
#ifndef TBG_MERGE_THREADS
#define TBG_MERGE_THREADS 256
#endif
#ifndef TBG_MERGE_PER_THREAD
#define TBG_MERGE_PER_THREAD 16
#endif
#ifndef TBG_MCOUNT_PER_THREAD
#define TBG_MCOUNT_PER_THREAD 32
#endif
constexpr int MERGE_THREADS = TBG_MERGE_THREADS;
constexpr int MERGE_PER_THREAD = TBG_MERGE_PER_THREAD;
constexpr int MERGE_TILE = MERGE_THREADS * MERGE_PER_THREAD;
// the count-only merge walks longer segments (its per-thread search and
// set-up cost less per row) and loads its tile in batches of 16 rows
constexpr int MCOUNT_PER_THREAD = TBG_MCOUNT_PER_THREAD;
constexpr int MCOUNT_TILE = MERGE_THREADS * MCOUNT_PER_THREAD;
constexpr int MCOUNT_BATCH = 16;
static_assert(MCOUNT_PER_THREAD % MCOUNT_BATCH == 0 && MCOUNT_TILE >= MERGE_TILE, "batches; the splits buffer");

template <bool A_FIRST>
__global__ void k_merge_splits(const Row *__restrict__ R, uint64_t nr, const Row *__restrict__ S, uint64_t ns,
                               uint64_t *__restrict__ splits, uint64_t nsplits, uint32_t tile) {
    const uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nsplits) return;
    const uint64_t d = umin64(nr + ns, c * tile);
    auto kr = [&](uint64_t i) { return R[i].key; };
    auto ks = [&](uint64_t j) { return S[j].key; };
    splits[c] = merge_split<A_FIRST>(d, nr, ns, kr, ks);
}

// Count-only merge join.  The merged order takes R[i] before S[j] iff
// R[i].key <= S[j].key, so when S[j] is taken every R row of its key is
// behind it (in this tile or an earlier one): each thread keeps the last R
// key taken and the number of R rows with that key (`run`), and S[j] adds
// run when its key is that key.  A thread finds the run it starts inside once,
// walking back (into global memory before the tile's first R row when the run
// starts earlier); the steps themselves never walk a run.  Keys sit in shared
// memory at t + t / 16, so threads whose walks start 16 apart use different
// banks.
#ifndef TBG_MERGE_SKEW
#define TBG_MERGE_SKEW 1
#endif
__device__ __forceinline__ uint32_t mskew(uint32_t t) { return TBG_MERGE_SKEW ? t + (t >> 4) : t; }
constexpr uint32_t mskew_host(uint32_t t) { return t + (t >> 4); }

__global__ void __launch_bounds__(MERGE_THREADS, 6) k_merge_count(const Row *__restrict__ R, uint64_t nr,
                                                                const Row *__restrict__ S, uint64_t ns,
                                                                const uint64_t *__restrict__ splits,
                                                                unsigned long long *matches) {
    extern __shared__ __align__(16) uint32_t merge_smem[];
    uint32_t *K = merge_smem;  // mskew(MCOUNT_TILE) + 1 keys: R's, then S's, and a spare slot
    const uint64_t L = nr + ns;
    const uint64_t c = blockIdx.x;
    const uint64_t dc0 = c * MCOUNT_TILE, dc1 = umin64(L, dc0 + MCOUNT_TILE);
    const uint64_t ic0 = splits[c], ic1 = splits[c + 1];
    const uint64_t jc0 = dc0 - ic0, jc1 = dc1 - ic1;
    const uint32_t nrt = (uint32_t)(ic1 - ic0), nst = (uint32_t)(jc1 - jc0);
    const uint32_t Lt = nrt + nst;
    {
        const uint2 *Rv = reinterpret_cast<const uint2 *>(R) + ic0;
        const uint2 *Sv = reinterpret_cast<const uint2 *>(S) + jc0;
#pragma unroll
        for (int b = 0; b < MCOUNT_PER_THREAD; b += MCOUNT_BATCH) {
            uint32_t x[MCOUNT_BATCH];
#pragma unroll
            for (int q = 0; q < MCOUNT_BATCH; q++) {
                const uint32_t t = (b + q) * MERGE_THREADS + threadIdx.x;
                if (t < Lt) x[q] = __ldcs(t < nrt ? Rv + t : Sv + (t - nrt)).x;
            }
#pragma unroll
            for (int q = 0; q < MCOUNT_BATCH; q++) {
                const uint32_t t = (b + q) * MERGE_THREADS + threadIdx.x;
                if (t < Lt) K[mskew(t)] = x[q];
            }
        }
        if (threadIdx.x == 0) K[mskew(Lt)] = 0;
    }
    __syncthreads();
    auto kr = [&](uint32_t i) { return K[mskew(i)]; };
    auto ks = [&](uint32_t j) { return K[mskew(nrt + j)]; };
    const uint32_t d0 = min(Lt, threadIdx.x * MCOUNT_PER_THREAD), d1 = min(Lt, d0 + MCOUNT_PER_THREAD);
    uint32_t i;
    {
        uint32_t lo = d0 > nst ? d0 - nst : 0, hi = min(d0, nrt);
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (kr(mid) <= ks(d0 - mid - 1)) lo = mid + 1;
            else hi = mid;
        }
        i = lo;
    }
    uint32_t j = d0 - i;
    uint32_t pk = 0;
    uint64_t run = 0;  // with no R row behind, run 0 matches nothing
    const uint64_t gi = ic0 + i;
    if (gi > 0 && d0 < d1) {
        // the R rows of key R[gi - 1] end at gi - 1: find the first of them
        auto rkey = [&](uint64_t g) { return g >= ic0 ? kr((uint32_t)(g - ic0)) : R[g].key; };
        pk = rkey(gi - 1);
        uint64_t q = gi - 1;
        for (int w = 0; w < 4 && q > 0 && rkey(q - 1) == pk; w++) q--;
        if (q > 0 && rkey(q - 1) == pk) {
            uint64_t l = 0, h = q - 1;
            while (l < h) {
                const uint64_t m = (l + h) >> 1;
                if (rkey(m) < pk) l = m + 1;
                else h = m;
            }
            q = l;
        }
        run = gi - q;
    }
    // Current keys in registers.  A step takes R (ta) or S without a
    // branch: one shared load at the taken side's next position (past a
    // side's end: the other side's first key or the spare slot, which the
    // bounds keep unused) and selects.
    uint32_t jj = nrt + j;  // S's cursor in K
    uint32_t rk = kr(i), sk = K[mskew(jj)];
    uint32_t run32 = (uint32_t)run;  // a run of R rows is shorter than 2^32
    unsigned long long cnt = 0;
    const uint32_t steps = d1 - d0;
#pragma unroll
    for (uint32_t t = 0; t < (uint32_t)MCOUNT_PER_THREAD; t++) {
        if (t < steps) {
            const bool ta = i < nrt && (jj >= Lt || rk <= sk);
            const uint32_t key = ta ? rk : sk;
            const bool eq = key == pk;
            cnt += (!ta && eq) ? run32 : 0u;
            run32 = ta ? (eq ? run32 + 1 : 1u) : run32;
            pk = ta ? key : pk;
            const uint32_t nx = K[mskew((ta ? i : jj) + 1)];
            i += ta;
            jj += !ta;
            rk = ta ? nx : rk;
            sk = ta ? sk : nx;
        }
    }
    const unsigned long long ws = warp_sum_u64(cnt);
    if ((threadIdx.x & 31) == 0 && ws) atomicAdd(matches, ws);
}

template <bool MAT>
__global__ void __launch_bounds__(MERGE_THREADS) k_merge_join(const Row *__restrict__ R, uint64_t nr,
                                                               const Row *__restrict__ S, uint64_t ns,
                                                               const uint64_t *__restrict__ splits,
                                                               unsigned long long *matches,
                                                               unsigned long long *rows_ctr, tbg_row_out *out,
                                                               uint64_t cap) {
    // keys (and payloads when materialising) of the tile's R rows [0, nrt),
    // then of its S rows; one spare slot so a walk may read one row past
    // either side without a guard
    extern __shared__ __align__(16) uint32_t merge_smem[];
    uint32_t *K = merge_smem;                 // MERGE_TILE + 1 keys
    uint32_t *Pay = merge_smem + MERGE_TILE + 1;  // MERGE_TILE payloads (materialising)
    __shared__ unsigned long long s_base;
    __shared__ uint64_t scan_scratch[MERGE_THREADS / 32 + 1];
    const uint64_t L = nr + ns;
    const uint64_t c = blockIdx.x;
    const uint64_t dc0 = c * MERGE_TILE, dc1 = umin64(L, dc0 + MERGE_TILE);
    const uint64_t ic0 = splits[c], ic1 = splits[c + 1];
    const uint64_t jc0 = dc0 - ic0, jc1 = dc1 - ic1;
    const uint32_t nrt = (uint32_t)(ic1 - ic0), nst = (uint32_t)(jc1 - jc0);
    const uint32_t Lt = nrt + nst;
    {
        const uint2 *Rv = reinterpret_cast<const uint2 *>(R) + ic0;
        const uint2 *Sv = reinterpret_cast<const uint2 *>(S) + jc0;
        uint2 x[MERGE_PER_THREAD];
#pragma unroll
        for (int q = 0; q < MERGE_PER_THREAD; q++) {
            const uint32_t t = q * MERGE_THREADS + threadIdx.x;
            if (t < Lt) x[q] = *(t < nrt ? Rv + t : Sv + (t - nrt));
        }
#pragma unroll
        for (int q = 0; q < MERGE_PER_THREAD; q++) {
            const uint32_t t = q * MERGE_THREADS + threadIdx.x;
            if (t < Lt) {
                K[t] = x[q].x;
                if (MAT) Pay[t] = x[q].y;
            }
        }
        if (threadIdx.x == 0) K[Lt] = 0;
    }
    __syncthreads();
    const uint32_t *Ks = K + nrt;
    const uint32_t d0 = min(Lt, threadIdx.x * MERGE_PER_THREAD), d1 = min(Lt, d0 + MERGE_PER_THREAD);
    // merge-path split of diagonal d0 inside the tile (32-bit indices)
    uint32_t i0;
    {
        uint32_t lo = d0 > nst ? d0 - nst : 0, hi = min(d0, nrt);
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (K[mid] < Ks[d0 - mid - 1]) lo = mid + 1;
            else hi = mid;
        }
        i0 = lo;
    }
    const uint32_t j0 = d0 - i0;
    // rows of R equal to k from tile position i on (continuing past the tile)
    auto run_len = [&](uint32_t i, uint32_t k) {
        uint32_t q = i;
        while (q < nrt && K[q] == k) q++;
        uint32_t n = q - i;
        if (q == nrt)
            for (uint64_t g = ic0 + q; g < nr && R[g].key == k; g++) n++;
        return n;
    };
    uint32_t i = i0, j = j0, cnt = 0, last_key = 0, last_cnt = 0;
    uint32_t rk = K[i], sk = Ks[j];  // current keys (a spare or foreign slot past a side's end)
    bool have = false;
    for (uint32_t d = d0; d < d1; d++) {
        if (i < nrt && (j >= nst || rk < sk)) {
            rk = K[++i];
        } else {
            if (!have || sk != last_key) {
                // i == nrt: the run may continue in the R rows past the tile
                last_cnt = (i == nrt || rk == sk) ? run_len(i, sk) : 0;
                last_key = sk;
                have = true;
            }
            cnt += last_cnt;
            sk = Ks[++j];
        }
    }
    if (MAT) {
        uint64_t tot;
        const uint64_t off = block_excl_scan<MERGE_THREADS>(cnt, &tot, scan_scratch);
        if (threadIdx.x == 0) s_base = tot ? atomicAdd(rows_ctr, (unsigned long long)tot) : 0;
        __syncthreads();
        uint64_t pos = s_base + off;
        i = i0;
        j = j0;
        for (uint32_t d = d0; d < d1; d++) {
            if (i < nrt && (j >= nst || K[i] < Ks[j])) {
                i++;
            } else {
                const uint32_t k = Ks[j], sp = Pay[nrt + j];
                uint32_t q = i;
                for (; q < nrt && K[q] == k; q++, pos++)
                    if (pos < cap) out[pos] = tbg_row_out{k, Pay[q], sp};
                if (q == nrt)
                    for (uint64_t g = ic0 + q; g < nr && R[g].key == k; g++, pos++)
                        if (pos < cap) out[pos] = tbg_row_out{k, R[g].payload, sp};
                j++;
            }
        }
    }
    const unsigned long long ws = warp_sum_u64(cnt);
    if ((threadIdx.x & 31) == 0 && ws) atomicAdd(matches, ws);
}

uint64_t merge_ctas(uint64_t nr, uint64_t ns) { return (nr + ns + MERGE_TILE - 1) / MERGE_TILE; }

cudaError_t launch_merge_join(const Row *R, uint64_t nr, const Row *S, uint64_t ns, uint64_t *splits,
                              unsigned long long *matches, unsigned long long *rows_ctr, tbg_row_out *out,
                              uint64_t cap, bool mat, cudaStream_t st) {
    const uint64_t grid = merge_ctas(nr, ns);
    if (!grid) return cudaSuccess;
    const uint64_t nsplits = grid + 1;
    const unsigned sgrid = (unsigned)((nsplits + 255) / 256);
    cudaError_t e;
    if (!mat) {
        const uint64_t cgrid = (nr + ns + MCOUNT_TILE - 1) / MCOUNT_TILE;
        k_merge_splits<true><<<(unsigned)((cgrid + 256) / 256), 256, 0, st>>>(R, nr, S, ns, splits, cgrid + 1,
                                                                              MCOUNT_TILE);
        const size_t smem = (size_t)(mskew_host(MCOUNT_TILE) + 1) * 4;
        if ((e = smem_limit((const void *)k_merge_count, smem)) != cudaSuccess) return e;
        k_merge_count<<<(unsigned)cgrid, MERGE_THREADS, smem, st>>>(R, nr, S, ns, splits, matches);
    } else {
        k_merge_splits<false><<<sgrid, 256, 0, st>>>(R, nr, S, ns, splits, nsplits, MERGE_TILE);
        const size_t smem = (size_t)(2 * MERGE_TILE + 1) * 4;
        if ((e = smem_limit((const void *)k_merge_join<true>, smem)) != cudaSuccess) return e;
        k_merge_join<true><<<(unsigned)grid, MERGE_THREADS, smem, st>>>(R, nr, S, ns, splits, matches, rows_ctr,
                                                                        out, cap);
    }
    count_launch(2);
    return cudaGetLastError();
}

}  // namespace tbg
