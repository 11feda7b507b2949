// Drop-in join entry points with the reference's signature
//     result_t *NAME(struct table_t *relR, struct table_t *relS, int nthreads)
// (Joins/radix_join.h:20-24, Joins/radix_sortmerge_join.h:4,
// Joins/psm/parallel_sortmerge_join.h:61) and the name registry of
// native.cpp:34-46.  A call copies R and S to the GPU, runs the device
// pipeline and returns a malloc'd result_t shaped like the reference's:
// totalresults, nthreads, and per-"thread" result lists under materialisation
// (Joins/radix_join.c:1195-1199), here NULL-terminated contiguous node arrays.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "tbg_internal.h"
#include "tbg_runtime.h"

namespace tbg {

static std::mutex g_dropin_mu;
static cudaStream_t g_stream = nullptr;
static tbg_row_out *g_host_rows = nullptr;  // pinned staging for result rows
static size_t g_host_rows_cap = 0;
static uint64_t g_last_h2d = 0, g_last_d2h = 0;  // bytes the last call moved

extern int dropin_errmode();

// RHO and RHT copy large S in slices on a second stream and join each slice
// as it lands (run_radix_join_sliced), so only the last slice's work follows
// the last copy.
constexpr int MAX_SLICES = 16;
constexpr uint64_t SLICE_ROWS = 1ull << 26;  // 512 MiB of S per slice
static int g_slices = 0;                     // 0: SLICE_ROWS per slice, up to MAX_SLICES
static cudaStream_t g_copy = nullptr;
static cudaEvent_t g_ready[MAX_SLICES + 1];  // [0]: R copied; [1 + k]: slice k copied
static cudaEvent_t g_idle;                   // the join stream reached the copies

static int slice_count(int algo, uint64_t nR, uint64_t nS) {
    if (algo != TBG_RHO && algo != TBG_RHT) return 1;
    if (nR == 0 || nR > 0xFFFFFFFFull || nS > 0xFFFFFFFFull) return 1;
    const uint64_t k = g_slices > 0 ? (uint64_t)g_slices : nS / SLICE_ROWS;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(std::min<uint64_t>(k, MAX_SLICES), nS));
}

static cudaError_t slice_streams() {
    if (g_copy) return cudaSuccess;
    cudaError_t e = cudaStreamCreateWithFlags(&g_copy, cudaStreamNonBlocking);
    for (auto &ev : g_ready)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g_idle, cudaEventDisableTiming);
    return e;
}

static cudaError_t h2d(void *dst, const void *src, size_t bytes, cudaStream_t st) {
    if (!bytes) return cudaSuccess;
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
}

static result_t *fail(int code) {
    if (dropin_errmode() == TBG_ERRMODE_EXIT) {
        fprintf(stderr, "[ERROR] tee-bench-b200: %s (status %d)\n", tbg_last_error_string(), code);
        exit(EXIT_FAILURE);
    }
    return nullptr;
}

static result_t *make_result(uint64_t matches, int nthreads, const tbg_row_out *rows) {
    result_t *res = (result_t *)malloc(sizeof(result_t));
    if (!res) return nullptr;
    res->totalresults = (int64_t)matches;
    res->nthreads = nthreads;
    res->resultlist = (threadresult_t *)calloc((size_t)nthreads, sizeof(threadresult_t));
    if (!res->resultlist) {
        free(res);
        return nullptr;
    }
    for (int t = 0; t < nthreads; t++) {
        uint64_t lo = matches * (uint64_t)t / (uint64_t)nthreads;
        uint64_t hi = matches * (uint64_t)(t + 1) / (uint64_t)nthreads;
        threadresult_t &tr = res->resultlist[t];
        tr.nresults = (int64_t)(hi - lo);
        tr.threadid = (uint32_t)t;
        tr.results = nullptr;
        if (rows && hi > lo) {
            output_list_t *nodes = (output_list_t *)malloc(sizeof(output_list_t) * (hi - lo));
            if (!nodes) {
                tbg_result_free(res);
                return nullptr;
            }
            for (uint64_t i = lo; i < hi; i++) {
                output_list_t &n = nodes[i - lo];
                n.key = rows[i].key;
                n.Rpayload = rows[i].Rpayload;
                n.Spayload = rows[i].Spayload;
                n.next = (i + 1 < hi) ? &nodes[i - lo + 1] : nullptr;
            }
            tr.results = nodes;
        }
    }
    return res;
}

static result_t *dropin(int algo, struct table_t *relR, struct table_t *relS, int nthreads, bool mat) {
    std::lock_guard<std::mutex> g(g_dropin_mu);
    if (nthreads < 1) nthreads = 1;
    if (!relR || !relS || (relR->num_tuples && !relR->tuples) || (relS->num_tuples && !relS->tuples))
        return fail(set_error(TBG_ERR_ARG, "null relation"));
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(set_error(TBG_ERR_NO_DEVICE, "no CUDA device visible"));
    }
    if (!g_stream && cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(cuda_error(cudaGetLastError(), "stream"));
    Workspace *w = workspace_for(g_stream);
    if (!w) return fail(set_error(TBG_ERR_CUDA, "workspace"));
    const uint64_t nR = relR->num_tuples, nS = relS->num_tuples;
    cudaError_t e;
    if ((e = w->inR.ensure(std::max<uint64_t>(nR, 1) * 8)) != cudaSuccess) return fail(cuda_error(e, "cudaMalloc"));
    if ((e = w->inS.ensure(std::max<uint64_t>(nS, 1) * 8)) != cudaSuccess) return fail(cuda_error(e, "cudaMalloc"));
    const int K = slice_count(algo, nR, nS);
    if (K == 1) {
        if ((e = h2d(w->inR.p, relR->tuples, nR * 8, g_stream)) != cudaSuccess) return fail(cuda_error(e, "H2D R"));
        if ((e = h2d(w->inS.p, relS->tuples, nS * 8, g_stream)) != cudaSuccess) return fail(cuda_error(e, "H2D S"));
    } else {
        if ((e = slice_streams()) != cudaSuccess) return fail(cuda_error(e, "copy stream"));
        // the copies overwrite the inputs only after the join stream's earlier work
        if ((e = cudaEventRecord(g_idle, g_stream)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(g_copy, g_idle, 0)) != cudaSuccess)
            return fail(cuda_error(e, "copy stream"));
    }

    g_last_h2d = (nR + nS) * 8;
    g_last_d2h = sizeof(Ctrl);
    tbg_config cfg;
    tbg_config_init(&cfg);
    cfg.algo = algo;
    cfg.materialize = mat ? 1 : 0;
    uint64_t matches = 0;
    uint64_t cap = 0;
    tbg_row_out *d_rows = nullptr;
    const Row *dR = w->inR.as<Row>(), *dS = w->inS.as<Row>();
    bool resident = K == 1;
    for (int attempt = 0; attempt < 2; attempt++) {
        if (mat) {
            cap = attempt == 0 ? std::max<uint64_t>(nS, 1024) : std::max<uint64_t>(matches, 1);
            if ((e = w->rows.ensure(cap * sizeof(tbg_row_out))) != cudaSuccess) return fail(cuda_error(e, "cudaMalloc rows"));
            d_rows = w->rows.as<tbg_row_out>();
        }
        int rc;
        if (resident) {
            rc = tbg_join_device(&cfg, reinterpret_cast<const row_t *>(dR), nR, reinterpret_cast<const row_t *>(dS),
                                 nS, d_rows, cap, &matches, nullptr, g_stream);
        } else {
            uint64_t lo[MAX_SLICES + 1];
            for (int k = 0; k <= K; k++) lo[k] = nS * (uint64_t)k / (uint64_t)K;
            auto issue = [&](int k) -> int {
                const bool isR = k < 0;
                const uint64_t off = isR ? 0 : lo[k] * 8, bytes = isR ? nR * 8 : (lo[k + 1] - lo[k]) * 8;
                const void *src = static_cast<const char *>(isR ? (const void *)relR->tuples : (const void *)relS->tuples) + off;
                void *dst = static_cast<char *>(isR ? w->inR.p : w->inS.p) + off;
                cudaError_t ce = h2d(dst, src, bytes, g_copy);
                if (ce == cudaSuccess) ce = cudaEventRecord(g_ready[isR ? 0 : 1 + k], g_copy);
                return ce == cudaSuccess ? TBG_OK : cuda_error(ce, isR ? "H2D R" : "H2D S slice");
            };
            JoinRun run;
            rc = run_radix_join_sliced(cfg, dR, nR, dS, lo, K, issue, g_ready[0], g_ready + 1, d_rows, cap, *w,
                                       g_stream, &run);
            if (rc == TBG_OK) rc = finish_join(cfg, *w, g_stream, run, nR, nS, cap, &matches, nullptr);
            cudaError_t ce = cudaStreamSynchronize(g_copy);  // no copy outlives the call, even on error
            if (rc == TBG_OK && ce != cudaSuccess) rc = cuda_error(ce, "H2D");
            resident = true;
        }
        if (rc == TBG_OK) break;
        if (!(rc == TBG_ERR_CAPACITY && attempt == 0)) return fail(rc);
    }
    const tbg_row_out *host_rows = nullptr;
    if (mat && matches) {
        size_t bytes = matches * sizeof(tbg_row_out);
        if (bytes > g_host_rows_cap) {
            if (g_host_rows) cudaFreeHost(g_host_rows);
            g_host_rows = nullptr;
            g_host_rows_cap = 0;
            if ((e = cudaMallocHost(&g_host_rows, bytes)) != cudaSuccess) return fail(cuda_error(e, "cudaMallocHost"));
            g_host_rows_cap = bytes;
        }
        if ((e = cudaMemcpyAsync(g_host_rows, d_rows, bytes, cudaMemcpyDeviceToHost, g_stream)) != cudaSuccess)
            return fail(cuda_error(e, "D2H rows"));
        if ((e = cudaStreamSynchronize(g_stream)) != cudaSuccess) return fail(cuda_error(e, "D2H rows"));
        host_rows = g_host_rows;
        g_last_d2h += bytes;
    }
    result_t *res = make_result(matches, nthreads, host_rows);
    if (!res) return fail(set_error(TBG_ERR_OOM, "host allocation of the result"));
    return res;
}

}  // namespace tbg

using namespace tbg;

extern "C" {

result_t *RHO(struct table_t *R, struct table_t *S, int n) { return dropin(TBG_RHO, R, S, n, false); }
result_t *RHT(struct table_t *R, struct table_t *S, int n) { return dropin(TBG_RHT, R, S, n, false); }
result_t *RSM(struct table_t *R, struct table_t *S, int n) { return dropin(TBG_RSM, R, S, n, false); }
result_t *PSM(struct table_t *R, struct table_t *S, int n) { return dropin(TBG_PSM, R, S, n, false); }
result_t *LRN(struct table_t *R, struct table_t *S, int n) { return dropin(TBG_LRN, R, S, n, false); }
result_t *RHO_mat(struct table_t *R, struct table_t *S, int n) { return dropin(TBG_RHO, R, S, n, true); }
result_t *RHT_mat(struct table_t *R, struct table_t *S, int n) { return dropin(TBG_RHT, R, S, n, true); }
result_t *RSM_mat(struct table_t *R, struct table_t *S, int n) { return dropin(TBG_RSM, R, S, n, true); }
result_t *PSM_mat(struct table_t *R, struct table_t *S, int n) { return dropin(TBG_PSM, R, S, n, true); }
result_t *LRN_mat(struct table_t *R, struct table_t *S, int n) { return dropin(TBG_LRN, R, S, n, true); }

const algorithm_t tbg_algorithms[] = {
    {"RHO", RHO},
    {"RHT", RHT},
    {"RSM", RSM},
    {"PSM", PSM},
    {"LRN", LRN},
};
const int tbg_num_algorithms = (int)(sizeof(tbg_algorithms) / sizeof(tbg_algorithms[0]));

const algorithm_t *tbg_find(const char *name) {
    if (!name) return nullptr;
    for (int i = 0; i < tbg_num_algorithms; i++)
        if (strcmp(name, tbg_algorithms[i].name) == 0) return &tbg_algorithms[i];
    set_error(TBG_ERR_UNKNOWN_ALGO, "unknown algorithm '%s'", name);
    return nullptr;
}

int tbg_set_dropin_slices(int k) {
    std::lock_guard<std::mutex> g(g_dropin_mu);
    const int prev = g_slices;
    g_slices = std::max(0, std::min(k, MAX_SLICES));
    return prev;
}

void tbg_last_transfer_bytes(uint64_t *h2d, uint64_t *d2h) {
    if (h2d) *h2d = g_last_h2d;
    if (d2h) *d2h = g_last_d2h;
}

void tbg_result_free(result_t *res) {
    if (!res) return;
    if (res->resultlist) {
        for (int t = 0; t < res->nthreads; t++) free(res->resultlist[t].results);
        free(res->resultlist);
    }
    free(res);
}

}  // extern "C"
