// Exchange step of a join split over several GPUs: tbg_shard_split.
//
// The reference runs one join on one machine and splits it over threads by
// contiguous chunks of R and S (Joins/radix_join.c:1285-1306), every thread
// partitioning its chunk into the shared radix partitions.  Across GPUs the
// relations live in separate memories, so the split has to be by key: every
// rank splits its rows of R and of S by destination shard (ShardOp, a hash of
// the key), an all-to-all (NCCL, in the caller) moves each piece to its
// shard's rank, and every rank joins what it received with the single-GPU
// join.  Equal keys always meet on the same rank, so the ranks' counts sum to
// the join's count, and each rank partitions only its share of R and S.
//
// The split is the chunked radix pass of partition.cu with the shard as the
// digit: per-chunk histograms over the shards, a column prefix over chunks,
// then the TMA-fed tile scatter with exact per-(chunk, shard) cursors.
#include "part_dev.cuh"
#include "tbg_runtime.h"

namespace tbg {

constexpr int SHARD_HIST_THREADS = 1024;
constexpr int SHARD_THREADS = 512;

// K1: chunk c's row count per shard -> hist[c][d].
__global__ void __launch_bounds__(SHARD_HIST_THREADS) k_shard_hist(const Row *__restrict__ in, uint64_t n,
                                                                   uint64_t chunk, uint32_t *__restrict__ hist,
                                                                   ShardOp op) {
    __shared__ uint32_t sh[SCATTER_FMAX];
    for (int i = threadIdx.x; i < (int)op.n; i += SHARD_HIST_THREADS) sh[i] = 0;
    __syncthreads();
    const uint64_t lo = (uint64_t)blockIdx.x * chunk;
    const uint64_t hi = umin64(n, lo + chunk);
    // warp-uniform trip count: every lane reaches the shuffles in hist_add_warp
    for (uint64_t base = lo; base < hi; base += 4ull * SHARD_HIST_THREADS) {
        uint32_t d[4];
        bool ok[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const uint64_t i = base + (uint64_t)u * SHARD_HIST_THREADS + threadIdx.x;
            ok[u] = i < hi;
            d[u] = ok[u] ? op(ldg_stream(reinterpret_cast<const uint2 *>(in) + i).x) : 0;
        }
        const bool dup = warp_has_dups(d[0], ok[0]);
#pragma unroll
        for (int u = 0; u < 4; u++) hist_add_warp(sh, d[u], ok[u], dup);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < (int)op.n; i += SHARD_HIST_THREADS) hist[(uint64_t)blockIdx.x * op.n + i] = sh[i];
}

// K3: chunk c scatters its rows by shard to cursor[d] = base[d] + pre[c][d],
// base[d] = rows of the shards before d (from the totals).
__global__ void __launch_bounds__(SHARD_THREADS, 2) k_shard_scatter(const Row *__restrict__ in, uint64_t n,
                                                                    uint64_t chunk, Row *__restrict__ out,
                                                                    const uint32_t *__restrict__ pre,
                                                                    const uint32_t *__restrict__ totals, ShardOp op,
                                                                    unsigned *err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto &sm = *reinterpret_cast<PartSmem<SHARD_THREADS> *>(smem_raw);
    __shared__ uint64_t scratch[SHARD_THREADS / 32 + 1];
    const int c = blockIdx.x, tid = threadIdx.x;
    const uint64_t mine = tid < (int)op.n ? totals[tid] : 0;
    uint64_t total;
    const uint64_t base = block_excl_scan<SHARD_THREADS>(mine, &total, scratch);
    if (tid < (int)op.n) sm.cursor[tid] = (uint32_t)base + pre[(uint64_t)c * op.n + tid];
    __syncthreads();
    const uint64_t lo = (uint64_t)c * chunk;
    const uint64_t hi = umin64(n, lo + chunk);
    part_range<SHARD_THREADS>(in, lo, hi, n, out, (uint32_t)n, op, (int)op.n, sm, err);
}

int shard_split(const Row *d_in, uint64_t n, int nshards, Row *d_out, uint64_t *offsets, cudaStream_t st) {
    Workspace *w = workspace_for(st);
    if (!w) return set_error(TBG_ERR_CUDA, "workspace");
    const ShardOp op{(uint32_t)nshards};
    // two partitioning CTAs per SM, four chunks per SM, >= 32K rows per chunk
    const int G = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)w->nsm * 4, (n + 32767) / 32768));
    const uint64_t chunk = ((n + G - 1) / G + 1) & ~1ull;
    cudaError_t e;
    if ((e = w->shard.ensure((size_t)G * nshards * 4 + (size_t)nshards * 4 + 64)) != cudaSuccess ||
        (e = w->ctrl.ensure(sizeof(Ctrl))) != cudaSuccess)
        return cuda_error(e, "cudaMalloc");
    uint32_t *hist = w->shard.as<uint32_t>();
    uint32_t *totals = hist + (size_t)G * nshards;
    Ctrl *ctrl = w->ctrl.as<Ctrl>();
    // pinned read-back area: the totals (<= 256 words), then the error word
    uint32_t *htot = static_cast<uint32_t *>(w->host_small);
    static_assert(SCATTER_FMAX * 4 + 4 <= Workspace::HOST_SMALL_BYTES, "pinned read-back area too small");
    if ((e = cudaMemsetAsync(&ctrl->error, 0, sizeof(unsigned), st)) != cudaSuccess) return cuda_error(e, "memset");
    k_shard_hist<<<G, SHARD_HIST_THREADS, 0, st>>>(d_in, n, chunk, hist, op);
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "shard histogram");
    if ((e = launch_colscan(hist, G, nshards, totals, st)) != cudaSuccess) return cuda_error(e, "shard prefix");
    const size_t smem = sizeof(PartSmem<SHARD_THREADS>);
    if ((e = smem_limit((const void *)k_shard_scatter, smem)) != cudaSuccess) return cuda_error(e, "shard scatter");
    k_shard_scatter<<<G, SHARD_THREADS, smem, st>>>(d_in, n, chunk, d_out, hist, totals, op, &ctrl->error);
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_error(e, "shard scatter");
    // the totals (and the error word) back to the host: the caller sizes its exchange with them
    if ((e = cudaMemcpyAsync(htot, totals, (size_t)nshards * 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(htot + SCATTER_FMAX, &ctrl->error, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_error(e, "shard totals");
    const unsigned err = htot[SCATTER_FMAX];
    uint64_t run = 0;
    for (int d = 0; d < nshards; d++) {
        offsets[d] = run;
        run += htot[d];
    }
    offsets[nshards] = run;
    if (err) return set_error((int)err, "device reported error %u", err);
    if (run != n) return set_error(TBG_ERR_CUDA, "shard split placed %llu of %llu rows", (unsigned long long)run,
                                   (unsigned long long)n);
    return TBG_OK;
}

}  // namespace tbg

using namespace tbg;

extern "C" {

int tbg_shard_split(const struct row_t *d_in, uint64_t n, int nshards, struct row_t *d_out, uint64_t *offsets,
                    void *stream) {
    if (nshards < 1 || nshards > SCATTER_FMAX || !offsets) return set_error(TBG_ERR_ARG, "nshards must be 1..256");
    if (n && (!d_in || !d_out)) return set_error(TBG_ERR_ARG, "null relation with rows");
    if (n > 0xFFFFFFFFull) return set_error(TBG_ERR_ARG, "a split holds at most 2^32 - 1 rows");
    if ((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out)) & 7)
        return set_error(TBG_ERR_ARG, "relations must be 8-byte aligned");
    if (n == 0) {
        for (int d = 0; d <= nshards; d++) offsets[d] = 0;
        return TBG_OK;
    }
    return shard_split(reinterpret_cast<const Row *>(d_in), n, nshards, reinterpret_cast<Row *>(d_out), offsets,
                       (cudaStream_t)stream);
}

uint32_t tbg_shard_of(uint32_t key, int nshards) { return nshards > 0 ? ShardOp{(uint32_t)nshards}(key) : 0u; }

}  // extern "C"
