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
// reserves output rows once per CTA round with a block scan, so one global
// atomic covers up to JOIN_THREADS * 8 probe rows (the reference's
// insert_output, Include/util.c:20-29, mallocs one node per row).
#include "tbg_device.cuh"

namespace tbg {

struct Table {
    uint32_t *key;    // [capR]
    uint32_t *pay;    // [capR]
    uint32_t *heads;  // layout 0: [N] 1-based chain heads; layout 1: [Nb+1] starts, then cursors
    uint16_t *next;   // layout 0: [capR] 1-based next links
    uint32_t mask;    // bucket mask
    int hs;           // hash shift (radix bits already consumed)
    int layout;

    __device__ __forceinline__ uint32_t bucket(uint32_t k) const { return (k >> hs) & mask; }

    template <class Fn>
    __device__ __forceinline__ void for_each(uint32_t k, Fn fn) const {
        const uint32_t b = bucket(k);
        if (layout == 0) {
            for (uint32_t h = heads[b]; h; h = next[h - 1])
                if (key[h - 1] == k) fn(pay[h - 1]);
        } else {
            for (uint32_t j = heads[b], e = heads[b + 1]; j < e; j++)
                if (key[j] == k) fn(pay[j]);
        }
    }
    __device__ __forceinline__ uint32_t count(uint32_t k) const {
        uint32_t c = 0;
        const uint32_t b = bucket(k);
        if (layout == 0) {
            for (uint32_t h = heads[b]; h; h = next[h - 1]) c += (key[h - 1] == k);
        } else {
            for (uint32_t j = heads[b], e = heads[b + 1]; j < e; j++) c += (key[j] == k);
        }
        return c;
    }
};

size_t join_smem_bytes(int capR) {
    return (size_t)capR * 4 * 2 + ((size_t)capR + 2) * 4 + (size_t)capR * 2 + 16;
}

__device__ void build_table(Table &t, const Row *__restrict__ R, uint64_t r_off, uint32_t r_len,
                            uint64_t *scan_scratch) {
    const int tid = threadIdx.x;
    if (t.layout == 0) {
        const uint32_t N = next_pow2(r_len);
        t.mask = N - 1;
        for (uint32_t i = tid; i < r_len; i += JOIN_THREADS) {
            uint2 x = reinterpret_cast<const uint2 *>(R)[r_off + i];
            t.key[i] = x.x;
            t.pay[i] = x.y;
        }
        for (uint32_t i = tid; i < N; i += JOIN_THREADS) t.heads[i] = 0;
        __syncthreads();
        for (uint32_t i = tid; i < r_len; i += JOIN_THREADS) {
            uint32_t b = t.bucket(t.key[i]);
            t.next[i] = (uint16_t)atomicExch(&t.heads[b], i + 1);
        }
        __syncthreads();
    } else {
        uint32_t Nb = next_pow2(r_len) >> 2;
        if (Nb < 4) Nb = 4;
        t.mask = Nb - 1;
        uint32_t *cnt = t.heads;            // [Nb + 1]
        uint32_t *cur = t.heads + Nb + 1;   // cursors, Nb entries (fits: capR + 2 >= 2 Nb + 1)
        for (uint32_t i = tid; i <= Nb; i += JOIN_THREADS) cnt[i] = 0;
        __syncthreads();
        for (uint32_t i = tid; i < r_len; i += JOIN_THREADS)
            atomicAdd(&cnt[t.bucket(reinterpret_cast<const uint2 *>(R)[r_off + i].x)], 1u);
        __syncthreads();
        // exclusive scan of cnt[0..Nb) in place, cnt[Nb] = r_len
        const uint32_t per = (Nb + JOIN_THREADS - 1) / JOIN_THREADS;
        const uint32_t lo = min(Nb, tid * per), hi = min(Nb, lo + per);
        uint64_t s = 0;
        for (uint32_t i = lo; i < hi; i++) s += cnt[i];
        uint64_t tot;
        uint64_t run = block_excl_scan<JOIN_THREADS>(s, &tot, scan_scratch);
        for (uint32_t i = lo; i < hi; i++) {
            uint32_t c = cnt[i];
            cnt[i] = (uint32_t)run;
            cur[i] = (uint32_t)run;
            run += c;
        }
        if (tid == 0) cnt[Nb] = r_len;
        __syncthreads();
        for (uint32_t i = tid; i < r_len; i += JOIN_THREADS) {
            uint2 x = reinterpret_cast<const uint2 *>(R)[r_off + i];
            uint32_t pos = atomicAdd(&cur[t.bucket(x.x)], 1u);
            t.key[pos] = x.x;
            t.pay[pos] = x.y;
        }
        __syncthreads();
    }
}

template <bool MAT>
__global__ void __launch_bounds__(JOIN_THREADS) k_join(JoinArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t s_item;
    __shared__ unsigned long long s_base;
    __shared__ uint64_t scan_scratch[JOIN_THREADS / 32 + 1];
    Table t;
    t.key = reinterpret_cast<uint32_t *>(smem);
    t.pay = t.key + a.capR;
    t.heads = t.pay + a.capR;
    t.next = reinterpret_cast<uint16_t *>(t.heads + a.capR + 2);
    t.hs = a.hash_shift;
    t.layout = a.layout;
    const int tid = threadIdx.x;
    const unsigned nitems = *a.nitems;
    unsigned long long local = 0;

    for (;;) {
        if (tid == 0) s_item = atomicAdd(a.item_ctr, 1u);
        __syncthreads();
        const uint32_t it = s_item;
        if (it >= nitems) break;
        const Item m = a.items[it];
        build_table(t, a.R, m.r_off, m.r_len, scan_scratch);

        const Row *s = a.S + m.s_off;
        const uint64_t len = m.s_len;
        const uint64_t head = ((reinterpret_cast<uintptr_t>(s) & 15) && len) ? 1 : 0;
        const uint64_t body = len - head;
        const uint64_t nv = body / 2;
        const bool tail = body & 1;
        const uint4 *v = reinterpret_cast<const uint4 *>(s + head);

        if (!MAT) {
            if (head && tid == 0) local += t.count(s[0].key);
            if (tail && tid == JOIN_THREADS - 1) local += t.count(s[len - 1].key);
            uint64_t i = tid;
            for (; i + 3 * JOIN_THREADS < nv; i += 4 * JOIN_THREADS) {
                uint4 x0 = ldg_stream(v + i), x1 = ldg_stream(v + i + JOIN_THREADS);
                uint4 x2 = ldg_stream(v + i + 2 * JOIN_THREADS), x3 = ldg_stream(v + i + 3 * JOIN_THREADS);
                local += t.count(x0.x) + t.count(x0.z) + t.count(x1.x) + t.count(x1.z);
                local += t.count(x2.x) + t.count(x2.z) + t.count(x3.x) + t.count(x3.z);
            }
            for (; i < nv; i += JOIN_THREADS) {
                uint4 x0 = ldg_stream(v + i);
                local += t.count(x0.x) + t.count(x0.z);
            }
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
                uint32_t c = 0;
#pragma unroll
                for (int j = 0; j < 8; j++)
                    if (valid >> j & 1) c += t.count(k[j]);
                uint64_t tot;
                uint64_t off = block_excl_scan<JOIN_THREADS>(c, &tot, scan_scratch);
                if (tid == 0) s_base = tot ? atomicAdd(a.rows_ctr, (unsigned long long)tot) : 0;
                __syncthreads();
                uint64_t pos = s_base + off;
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    if (valid >> j & 1) {
                        const uint32_t kk = k[j], pp = p[j];
                        t.for_each(kk, [&](uint32_t rp) {
                            if (pos < a.cap) {
                                tbg_row_out o;
                                o.key = kk; o.Rpayload = rp; o.Spayload = pp;
                                a.out[pos] = o;
                            }
                            pos++;
                        });
                    }
                }
                local += c;
                __syncthreads();
            }
        }
        __syncthreads();  // table reused by the next item
    }
    unsigned long long ws = warp_sum_u64(local);
    if ((tid & 31) == 0 && ws) atomicAdd(a.matches, ws);
}

int join_ctas_per_sm(int capR) {
    int n = 0;
    const size_t smem = join_smem_bytes(capR);
    cudaFuncSetAttribute(k_join<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(k_join<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_join<false>, JOIN_THREADS, smem);
    return n < 1 ? 1 : n;
}

cudaError_t launch_join(const JoinArgs &a, bool materialize, int grid, cudaStream_t st) {
    const size_t smem = join_smem_bytes(a.capR);
    auto kern = materialize ? k_join<true> : k_join<false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, JOIN_THREADS, smem, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

}  // namespace tbg
