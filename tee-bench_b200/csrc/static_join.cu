// Join count without device allocation: tbg_join_count_static.
//
// For callers that cannot call cudaMalloc / cudaFree: engines whose device
// memory is owned and budgeted by their own pool allocator (a query engine's
// buffer manager, a framework's caching allocator), and latency-bound
// pipelines that cannot accept the device-wide synchronisation cudaFree
// implies or an out-of-memory failure in the middle of a query.  Every byte
// the join needs besides the caller's inputs and output lives in one
// file-scope device array of fixed size, so every GPU that loads the library
// holds it until the process exits.
//
// The join is the batched persistent kernel (k_batch) run on a plan of one
// join, count only: a direct shared-memory join when |R| fits one table
// (8192 rows), otherwise one radix pass of B = clamp(log2 |R| - 11, 1, 8)
// bits, then build/probe per partition.  A one-block prologue kernel writes
// the plan into the array and clears what must start at zero (progress
// counters, histograms, the caller's count), so no call depends on what the
// previous one left there.  Calls whose executions overlap on the GPU share
// the array and race: serialise them (one stream, or events).
#include <algorithm>
#include <mutex>

#include "batch.h"
#include "tbg_runtime.h"

namespace tbg {
namespace {

constexpr uint64_t STATIC_MAX_ROWS = 1ull << 22;   // |R| + |S|, = TBG_STATIC_MAX_ROWS
constexpr uint32_t STATIC_CHUNK = 32768;
constexpr uint32_t STATIC_CAPS_RADIX = 65536;
constexpr uint32_t STATIC_CAPS_DIRECT = 16384;
constexpr size_t STATIC_META_BYTES = 256u << 10;   // plan, counters, histograms, bases, items
constexpr size_t STATIC_SCRATCH_BYTES = STATIC_META_BYTES + STATIC_MAX_ROWS * sizeof(Row) + 512;

// The scratch.  In host code this name is only a handle for
// cudaGetSymbolAddress, never a device address.
static __device__ __align__(256) unsigned char g_static_scratch[STATIC_SCRATCH_BYTES];

constexpr size_t al(size_t x) { return (x + 255) & ~size_t(255); }

// Byte offsets inside the scratch.
constexpr size_t OFF_CTL = 0;                                  // ticket, error word
constexpr size_t OFF_SYNC = 256;                               // BatchSync[1]
constexpr size_t OFF_JOIN = 512;                               // BatchJoin[1]
constexpr size_t MAX_CHUNKS = STATIC_MAX_ROWS / STATIC_CHUNK + 2;
constexpr size_t OFF_CHUNKS = al(OFF_JOIN + sizeof(BatchJoin));
constexpr size_t OFF_SCANS = al(OFF_CHUNKS + MAX_CHUNKS * sizeof(uint2));
constexpr size_t MAX_JT = STATIC_MAX_ROWS / STATIC_CAPS_DIRECT + 1;
constexpr size_t OFF_JT = al(OFF_SCANS + sizeof(uint32_t));
constexpr size_t OFF_BASE = al(OFF_JT + MAX_JT * sizeof(uint2));
constexpr size_t MAX_ITEMS = BATCH_FMAX + STATIC_MAX_ROWS / STATIC_CAPS_RADIX + 1;
constexpr size_t OFF_ITEMS = al(OFF_BASE + 2 * BATCH_FMAX * sizeof(uint32_t));
constexpr size_t OFF_HIST = al(OFF_ITEMS + MAX_ITEMS * sizeof(Item));
constexpr size_t OFF_ROWS = al(OFF_HIST + MAX_CHUNKS * BATCH_FMAX * sizeof(uint32_t));
static_assert(OFF_ROWS <= STATIC_META_BYTES, "plan region overflows its share of the scratch");
static_assert(OFF_ROWS + STATIC_MAX_ROWS * sizeof(Row) + 256 <= STATIC_SCRATCH_BYTES, "rows overflow the scratch");

struct StaticPlan {
    unsigned char *base;  // device address of the scratch
    const Row *R, *S;
    uint64_t nR, nS;
    uint32_t B, capS, GR, GS, n_jt, item_cap, rp_rows;
    unsigned long long *count;
};

// Writes the one-join plan into the scratch and zeroes the counters, the
// histograms and the caller's count (one block).
__global__ void __launch_bounds__(256) k_static_plan(StaticPlan p) {
    const int tid = threadIdx.x;
    unsigned char *b = p.base;
    const uint32_t P = 1u << p.B;
    if (tid == 0) {
        BatchJoin J{};
        J.R = p.R;
        J.S = p.S;
        J.nR = p.nR;
        J.nS = p.nS;
        J.B = p.B;
        J.P = P;
        J.layout = 0;
        J.capS = p.capS;
        J.chunk = STATIC_CHUNK;
        J.orig = 0;
        if (p.B) {
            J.Rp = reinterpret_cast<Row *>(b + OFF_ROWS);
            J.Sp = reinterpret_cast<Row *>(b + OFF_ROWS) + p.rp_rows;
            J.histR = reinterpret_cast<uint32_t *>(b + OFF_HIST);
            J.histS = J.histR + (size_t)p.GR * P;
            J.baseR = reinterpret_cast<uint32_t *>(b + OFF_BASE);
            J.baseS = J.baseR + BATCH_FMAX;
            J.items = reinterpret_cast<Item *>(b + OFF_ITEMS);
            J.GR = p.GR;
            J.GS = p.GS;
            J.item_cap = p.item_cap;
        }
        *reinterpret_cast<BatchJoin *>(b + OFF_JOIN) = J;
        *reinterpret_cast<uint32_t *>(b + OFF_SCANS) = 0;
        reinterpret_cast<unsigned *>(b + OFF_CTL)[0] = 0;  // ticket
        reinterpret_cast<unsigned *>(b + OFF_CTL)[1] = 0;  // error word
        *reinterpret_cast<BatchSync *>(b + OFF_SYNC) = BatchSync{};
        *p.count = 0;
    }
    uint2 *chunks = reinterpret_cast<uint2 *>(b + OFF_CHUNKS);
    if (p.B) {
        for (uint32_t c = tid; c < p.GR + p.GS; c += 256)
            chunks[c] = c < p.GR ? make_uint2(0, c) : make_uint2(0, 0x80000000u | (c - p.GR));
        uint32_t *hist = reinterpret_cast<uint32_t *>(b + OFF_HIST);
        for (uint64_t i = tid; i < (uint64_t)(p.GR + p.GS) * P; i += 256) hist[i] = 0;
    }
    uint2 *jt = reinterpret_cast<uint2 *>(b + OFF_JT);
    for (uint32_t q = tid; q < p.n_jt; q += 256) jt[q] = make_uint2(0, q);
}

struct StaticDevice {
    bool ok = false;
    unsigned char *scratch = nullptr;
    int grid = 0;
};
std::mutex g_static_mu;
StaticDevice g_static_dev[64];

// With device `dev` current: the scratch's device address (from
// cudaGetSymbolAddress) and the persistent kernel's grid, whose set-up also
// raises k_batch's shared-memory limit on this device.  Only a successful
// set-up is kept; after a failure the next call on the device tries again.
cudaError_t static_device(int dev, StaticDevice *out) {
    std::lock_guard<std::mutex> g(g_static_mu);
    StaticDevice &d = g_static_dev[dev];
    if (!d.ok) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
        if (e != cudaSuccess) return e;
        int nsm = 0, per_sm = 0;
        if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        if ((e = batch_occupancy(&per_sm)) != cudaSuccess) return e;
        d.scratch = static_cast<unsigned char *>(ptr);
        d.grid = nsm * per_sm;
        d.ok = true;
    }
    *out = d;
    return cudaSuccess;
}

}  // namespace
}  // namespace tbg

using namespace tbg;

extern "C" TBG_API int tbg_join_count_static(const row_t *dR, uint64_t nR, const row_t *dS, uint64_t nS,
                                             uint64_t *d_count, uint32_t *d_status, void *stream) {
    if (!d_count) return set_error(TBG_ERR_ARG, "tbg_join_count_static: d_count is NULL");
    if ((nR && !dR) || (nS && !dS))
        return set_error(TBG_ERR_ARG, "tbg_join_count_static: null relation with nonzero size");
    if (nR > STATIC_MAX_ROWS || nS > STATIC_MAX_ROWS || nR + nS > STATIC_MAX_ROWS)
        return set_error(TBG_ERR_ARG,
                         "tbg_join_count_static: |R| + |S| = %llu rows exceeds the static scratch limit of %llu "
                         "rows; use tbg_join_device for larger joins",
                         (unsigned long long)(nR + nS), (unsigned long long)STATIC_MAX_ROWS);
    if ((reinterpret_cast<uintptr_t>(dR) | reinterpret_cast<uintptr_t>(dS) | reinterpret_cast<uintptr_t>(d_count)) &
        7)
        return set_error(TBG_ERR_ARG, "tbg_join_count_static: relations and d_count must be 8-byte aligned");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetDevice");
    if (dev < 0 || dev >= 64) return set_error(TBG_ERR_ARG, "tbg_join_count_static: device index %d out of range", dev);
    StaticDevice sdev;
    if ((e = static_device(dev, &sdev)) != cudaSuccess) {
        cudaGetLastError();
        return cuda_error(e, "tbg_join_count_static: set-up");
    }
    const StaticDevice *sd = &sdev;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char *b = sd->scratch;
    if (nR == 0 || nS == 0) {
        e = cudaMemsetAsync(d_count, 0, sizeof(uint64_t), st);
        if (e == cudaSuccess && d_status) e = cudaMemsetAsync(d_status, 0, sizeof(uint32_t), st);
        return e == cudaSuccess ? TBG_OK : cuda_error(e, "cudaMemsetAsync");
    }
    StaticPlan p{};
    p.base = b;
    p.R = reinterpret_cast<const Row *>(dR);
    p.S = reinterpret_cast<const Row *>(dS);
    p.nR = nR;
    p.nS = nS;
    p.count = reinterpret_cast<unsigned long long *>(d_count);
    if (nR <= (uint64_t)BATCH_CAPR) {
        p.B = 0;
        p.capS = STATIC_CAPS_DIRECT;
        p.n_jt = (uint32_t)((nS + p.capS - 1) / p.capS);
    } else {
        const int lg = 63 - __builtin_clzll(nR);
        p.B = (uint32_t)std::max(1, std::min(lg + 1 - 12, 8));
        p.capS = STATIC_CAPS_RADIX;
        p.GR = (uint32_t)((nR + STATIC_CHUNK - 1) / STATIC_CHUNK);
        p.GS = (uint32_t)((nS + STATIC_CHUNK - 1) / STATIC_CHUNK);
        p.item_cap = (1u << p.B) + (uint32_t)((nS + p.capS - 1) / p.capS);
        p.rp_rows = (uint32_t)((nR + 31) & ~uint64_t(31));  // S copy starts 256-byte aligned
        const uint64_t w = std::max<uint64_t>(1, (nR + nS) >> 18);
        p.n_jt = (uint32_t)std::min<uint64_t>(p.item_cap, w);
    }
    BatchArgs a{};
    a.joins = reinterpret_cast<const BatchJoin *>(b + OFF_JOIN);
    a.chunks = reinterpret_cast<const uint2 *>(b + OFF_CHUNKS);
    a.scans = reinterpret_cast<const uint32_t *>(b + OFF_SCANS);
    a.jt = reinterpret_cast<const uint2 *>(b + OFF_JT);
    a.sync = reinterpret_cast<BatchSync *>(b + OFF_SYNC);
    a.ticket = reinterpret_cast<unsigned *>(b + OFF_CTL);
    a.err = reinterpret_cast<unsigned *>(b + OFF_CTL) + 1;
    a.counts = p.count;
    a.n_chunks = p.B ? p.GR + p.GS : 0;
    a.n_scans = p.B ? 1 : 0;
    a.n_jt = p.n_jt;
    a.capR = BATCH_CAPR;
    k_static_plan<<<1, 256, 0, st>>>(p);
    count_launch();
    e = cudaGetLastError();
    if (e == cudaSuccess) e = launch_batch(a, sd->grid, st);
    if (e == cudaSuccess && d_status) e = cudaMemcpyAsync(d_status, a.err, sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
    return e == cudaSuccess ? TBG_OK : cuda_error(e, "tbg_join_count_static: launch");
}
