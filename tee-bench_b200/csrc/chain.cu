// Chained joins on device-resident output: the reference's enclave driver
// joins R and S, turns the materialised rows into a relation of (key,
// R payload) tuples (to_relation, Enclave/TrustedJoins/secure_joins.cpp:
// 277-301: it copies the first 8 bytes of each output node) and joins T
// with it (ecall_three_way_join_sealed_tables, :348-399).  Here the rows
// never leave HBM: one kernel converts them and the second join reads the
// result in place.
#include <algorithm>

#include "tbg_internal.h"
#include "tbg_runtime.h"

namespace tbg {

// (key, Rpayload, Spayload) rows -> (key, payload = Rpayload) relation:
// 12 B read and 8 B written per row.
__global__ void __launch_bounds__(256) k_rows_to_relation(const tbg_row_out *__restrict__ rows, uint64_t n,
                                                          uint2 *__restrict__ out) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const tbg_row_out r = rows[i];
        out[i] = make_uint2(r.key, r.Rpayload);
    }
}

cudaError_t launch_rows_to_relation(const tbg_row_out *rows, uint64_t n, Row *out, int nsm, cudaStream_t st) {
    if (!n) return cudaSuccess;
    const unsigned g = (unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)nsm * 16);
    k_rows_to_relation<<<g, 256, 0, st>>>(rows, n, reinterpret_cast<uint2 *>(out));
    count_launch();
    return cudaGetLastError();
}

// Materialised join R x S into w-owned rows, growing the buffer once if the
// first guess (|S| rows) was too small.  Returns the rows and their count.
static int join_rows(const tbg_config &cfg, const Row *dR, uint64_t nR, const Row *dS, uint64_t nS, DevBuf &buf,
                     cudaStream_t st, tbg_row_out **rows, uint64_t *m) {
    tbg_config c = cfg;
    c.materialize = 1;
    uint64_t cap = std::max<uint64_t>(nS, 1);
    for (int attempt = 0; attempt < 2; attempt++) {
        cudaError_t e = buf.ensure(cap * sizeof(tbg_row_out));
        if (e != cudaSuccess) return cuda_error(e, "cudaMalloc (chain rows)");
        const int rc = tbg_join_device(&c, reinterpret_cast<const row_t *>(dR), nR,
                                       reinterpret_cast<const row_t *>(dS), nS, buf.as<tbg_row_out>(), cap, m,
                                       nullptr, st);
        if (rc == TBG_OK) {
            *rows = buf.as<tbg_row_out>();
            return TBG_OK;
        }
        if (rc != TBG_ERR_CAPACITY) return rc;
        cap = std::max<uint64_t>(*m, 1);  // exact count is known now
    }
    return set_error(TBG_ERR_CAPACITY, "chained join: output grew between attempts");
}

}  // namespace tbg

using namespace tbg;

extern "C" {

TBG_API int tbg_rows_to_relation(const tbg_row_out *d_rows, uint64_t n, row_t *d_out, void *stream) {
    if (n && (!d_rows || !d_out)) return set_error(TBG_ERR_ARG, "tbg_rows_to_relation: NULL buffer");
    if (reinterpret_cast<uintptr_t>(d_out) & 7)
        return set_error(TBG_ERR_ARG, "tbg_rows_to_relation: output must be 8-byte aligned");
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = launch_rows_to_relation(d_rows, n, reinterpret_cast<Row *>(d_out), nsm,
                                            static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? TBG_OK : cuda_error(e, "tbg_rows_to_relation");
}

TBG_API int tbg_join_three_way(const tbg_config *cfg, const row_t *dR, uint64_t nR, const row_t *dS, uint64_t nS,
                               const row_t *dT, uint64_t nT, tbg_row_out *d_rows2, uint64_t rows2_cap,
                               uint64_t *matches1, uint64_t *matches2, void *stream) {
    if (!cfg || !matches1 || !matches2) return set_error(TBG_ERR_ARG, "tbg_join_three_way: NULL argument");
    if (nT && !dT) return set_error(TBG_ERR_ARG, "tbg_join_three_way: NULL T");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Workspace *w = workspace_for(st);
    if (!w) return set_error(TBG_ERR_CUDA, "workspace");
    // join 1: R x S, materialised on the device
    tbg_row_out *rows1 = nullptr;
    uint64_t m1 = 0;
    int rc = join_rows(*cfg, reinterpret_cast<const Row *>(dR), nR, reinterpret_cast<const Row *>(dS), nS,
                       w->chain_rows, st, &rows1, &m1);
    if (rc) return rc;
    *matches1 = m1;
    // to_relation: (key, R payload) tuples, in HBM
    cudaError_t e = w->chain_rel.ensure(std::max<uint64_t>(m1, 1) * sizeof(Row));
    if (e != cudaSuccess) return cuda_error(e, "cudaMalloc (chain relation)");
    e = launch_rows_to_relation(rows1, m1, w->chain_rel.as<Row>(), w->nsm, st);
    if (e != cudaSuccess) return cuda_error(e, "to_relation");
    // join 2: T x relation (T on the build side, as the reference calls it)
    tbg_config c2 = *cfg;
    c2.materialize = d_rows2 ? 1 : 0;
    return tbg_join_device(&c2, dT, nT, reinterpret_cast<const row_t *>(w->chain_rel.as<Row>()), m1, d_rows2,
                           d_rows2 ? rows2_cap : 0, matches2, nullptr, stream);
}

}  // extern "C"
