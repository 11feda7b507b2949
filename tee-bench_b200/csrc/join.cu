// K4: per-partition build/probe out of shared memory, persistent CTAs pulling
// work items.  Replaces the reference's join phase (Joins/radix_join.c:1184-1192
// task loop) and its two table layouts:
//   layout 0  bucket_chaining_join (Joins/radix_join.c:187-244): bucket heads
//             over next_pow2(|R_p|) slots, index (key >> bits) & (N-1),
//             1-based chains through `next`;
//   layout 1  histogram_join (Joins/radix_join.c:374-440, RHT): bucket counts
//             over max(next_pow2(|R_p|)/4, 4) slots, prefix sum, R_p reordered
//             by bucket, probe scans the bucket's range.
// Counting uses per-thread counters folded once per CTA; materialisation
// reserves output rows once per CTA round (one global atomic for up to
// JOIN_THREADS * 8 probe rows) and places them in (row slot, lane) order, so
// consecutive lanes store consecutive rows (the reference's insert_output,
// Include/util.c:20-29, mallocs one node per row).
#include <algorithm>
#include <map>
#include <mutex>

#include "join_dev.cuh"

namespace tbg {

template <bool MAT>
__global__ void __launch_bounds__(JOIN_THREADS) k_join(JoinArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t s_item[2];
    __shared__ uint64_t scan_scratch[JOIN_THREADS / 32 + 1];
    if (a.gate) {  // the same value for every thread: the whole launch steps aside
        const unsigned long long v = *a.gate;
        if (a.gate_le ? v > a.gate_max : v <= a.gate_max) return;
    }
    Table t;
    t.key = reinterpret_cast<uint32_t *>(smem);
    t.pay = t.key + a.capR;
    t.heads = t.pay + a.capR;
    t.next = reinterpret_cast<uint16_t *>(t.heads + a.capR + 2);
    t.head64 = nullptr;
    t.hcap = floor_pow2((uint32_t)a.capR + 2);
    if (!MAT && a.layout == 0) {  // count only: keys, packed heads (capR * 4 is a multiple of 8), links
        t.hcap = count_head_slots(a.capR);
        t.head64 = reinterpret_cast<uint64_t *>(t.key + a.capR);
        t.next = reinterpret_cast<uint16_t *>(t.head64 + t.hcap);
    }
    if (!MAT && a.layout == 1) {  // count only: keys, then bucket starts and cursors (no payloads)
        t.pay = nullptr;
        t.heads = t.key + a.capR;
    }
    t.hs = a.hash_shift;
    t.layout = a.layout;
    const int tid = threadIdx.x;
    const unsigned nitems = *a.err ? 0u : *a.nitems;  // a planner error leaves the item list unusable
    unsigned long long local = 0;

    // an item is claimed one step ahead, and its R rows are prefetched into
    // L2 while the current item is probed, so its table build reads L2
    if (tid == 0) s_item[0] = atomicAdd(a.item_ctr, 1u);
    __syncthreads();
    for (uint32_t iter = 0;; iter++) {
        const uint32_t it = s_item[iter & 1];
        if (it >= nitems) break;
        if (tid == 0) {
            const uint32_t nx = atomicAdd(a.item_ctr, 1u);
            s_item[(iter + 1) & 1] = nx;  // read by all after this item's barriers
            if (nx < nitems) {
                const Item mn = a.items[nx];
                prefetch_l2(a.R + mn.r_off, (uint64_t)mn.r_len * sizeof(Row));
            }
        }
        const Item m = a.items[it];
        build_table<JOIN_THREADS>(t, a.R, m.r_off, m.r_len, scan_scratch);

        const Row *s = a.S + m.s_off;
        const uint64_t len = m.s_len;
        const uint64_t head = ((reinterpret_cast<uintptr_t>(s) & 15) && len) ? 1 : 0;
        const uint64_t body = len - head;
        const uint64_t nv = body / 2;
        const bool tail = body & 1;
        const uint4 *v = reinterpret_cast<const uint4 *>(s + head);

        if (!MAT) {
            local += probe_count<JOIN_THREADS>(t, s, len);
        } else {
            // block-synchronous rounds: 8 rows per thread, one reservation per round
            const uint64_t per_round = 4ull * JOIN_THREADS;
            const uint64_t rounds = (nv + per_round - 1) / per_round + ((head || tail) ? 1 : 0);
            for (uint64_t r = 0; r < rounds; r++) {
                uint32_t k[8], p[8];
                unsigned valid = 0;
                const bool edge = (head || tail) && r == rounds - 1;
                if (edge) {
                    if (tid == 0 && head) { k[0] = s[0].key; p[0] = s[0].payload; valid = 1; }
                    if (tid == 1 && tail) { k[0] = s[len - 1].key; p[0] = s[len - 1].payload; valid = 1; }
                } else {
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        uint64_t i = r * per_round + (uint64_t)u * JOIN_THREADS + tid;
                        if (i < nv) {
                            uint4 x = ldg_stream(v + i);
                            k[2 * u] = x.x; p[2 * u] = x.y;
                            k[2 * u + 1] = x.z; p[2 * u + 1] = x.w;
                            valid |= 3u << (2 * u);
                        }
                    }
                }
                uint32_t c[8];
                uint32_t csum = 0;
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    c[j] = (valid >> j & 1) ? t.count(k[j]) : 0;
                    csum += c[j];
                }
                uint64_t pos[8];
                block_emit_positions<JOIN_THREADS, 8>(c, pos, a.rows_ctr, scan_scratch);
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    if (c[j]) {
                        const uint32_t kk = k[j], pp = p[j];
                        uint64_t q = pos[j];
                        t.for_each(kk, [&](uint32_t rp) {
                            if (q < a.cap) {
                                tbg_row_out o;
                                o.key = kk; o.Rpayload = rp; o.Spayload = pp;
                                a.out[q] = o;
                            }
                            q++;
                        });
                    }
                }
                const uint32_t c_total = csum;
                local += c_total;
            }
        }
        __syncthreads();  // table reused by the next item
    }
    unsigned long long ws = warp_sum_u64(local);
    if ((tid & 31) == 0 && ws) atomicAdd(a.matches, ws);
}

size_t join_smem_bytes(int capR) {
    return (size_t)capR * 4 * 2 + ((size_t)capR + 2) * 4 + (size_t)capR * 2 + 16;
}
// Shared memory of a k_join launch: counting bucket-chain tables hold keys,
// packed heads and links only.
// Counting histogram tables (RHT) hold keys, the bucket starts and cursors.
size_t join_launch_smem(int capR, bool materialize, int layout) {
    if (!materialize && layout == 0)
        return (size_t)capR * 4 + (size_t)count_head_slots(capR) * 8 + (size_t)capR * 2 + 16;
    if (!materialize && layout == 1) {
        uint32_t p = 1;
        while (p < (uint32_t)capR) p <<= 1;
        const size_t nb = std::max<uint32_t>(p >> 2, 4);  // buckets of the largest partition
        return (size_t)capR * 4 + (2 * nb + 1) * 4 + 16;
    }
    return join_smem_bytes(capR);
}

// Resident CTAs per SM of a k_join launch at a table of capR rows, cached per
// (device, capR, materialize, layout): the occupancy query runs once per size.
int join_ctas_per_sm(int capR, bool materialize, int layout) {
    static std::mutex mu;
    static std::map<std::pair<int, int>, int> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> g(mu);
    const int key = capR * 4 + (materialize ? 2 : 0) + (layout ? 1 : 0);
    auto it = cache.find(std::make_pair(dev, key));
    if (it != cache.end()) return it->second;
    const size_t smem = join_launch_smem(capR, materialize, layout);
    int n = 0;
    if (smem_limit((const void *)k_join<false>, smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_join<false>, JOIN_THREADS, smem) != cudaSuccess) {
        cudaGetLastError();
        return 1;  // not cached: a later call retries
    }
    n = n < 1 ? 1 : n;
    cache[std::make_pair(dev, key)] = n;
    return n;
}

cudaError_t launch_join(const JoinArgs &a, bool materialize, int grid, cudaStream_t st) {
    const size_t smem = join_launch_smem(a.capR, materialize, a.layout);
    auto kern = materialize ? k_join<true> : k_join<false>;
    cudaError_t e = smem_limit((const void *)kern, smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, JOIN_THREADS, smem, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

}  // namespace tbg
