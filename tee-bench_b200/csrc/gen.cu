// On-GPU seeded generators with the semantics of the reference's
// App/Lib/generator.cpp (pk: permutation of 1..n; fk: n / maxid permuted
// copies of 1..maxid followed by a permuted block of 1..(n % maxid)) and
// App/Lib/genzipf.c (Zipf ranks over an alphabet 1..N), plus the order-free
// checksum of materialised rows.  The random source is counter based, so the
// data depend only on (n, seed), not on the launch shape.
#include <cmath>

#include "tbg_device.cuh"

namespace tbg {

// A seeded bijection of [0, 2^k) built from odd multiplications, additions
// and xor-shifts (each invertible mod 2^k); cycle-walking restricts it to a
// permutation of [0, n).
struct Perm {
    uint64_t n, mask, a1, a2, a3, c1, c2;
    int s1, s2;
};

__host__ __device__ inline Perm make_perm(uint64_t n, uint64_t seed) {
    Perm p;
    int k = 0;
    while (k < 63 && (1ull << k) < n) k++;
    p.n = n;
    p.mask = k ? ((1ull << k) - 1) : 0;
    p.a1 = mix64(seed ^ 0x1111) | 1;
    p.a2 = mix64(seed ^ 0x2222) | 1;
    p.a3 = mix64(seed ^ 0x3333) | 1;
    p.c1 = mix64(seed ^ 0x4444);
    p.c2 = mix64(seed ^ 0x5555);
    p.s1 = (k + 1) / 2 > 0 ? (k + 1) / 2 : 1;
    p.s2 = k / 3 + 1;
    return p;
}

__device__ __forceinline__ uint64_t perm_round(const Perm &p, uint64_t x) {
    x = (x ^ p.c1) & p.mask;
    x = (x * p.a1) & p.mask;
    x ^= x >> p.s1;
    x = (x * p.a2) & p.mask;
    x ^= x >> p.s2;
    x = (x * p.a3) & p.mask;
    x ^= x >> p.s1;
    x = (x + p.c2) & p.mask;
    return x;
}

__device__ __forceinline__ uint64_t perm_apply(const Perm &p, uint64_t x) {
    // the cycle of a permutation through x returns below n; expected < 2 steps
    uint64_t y = perm_round(p, x);
    while (y >= p.n) y = perm_round(p, y);
    return y;
}

__global__ void k_gen_pk(Row *d, uint64_t n, uint64_t seed) {
    const Perm p = make_perm(n, seed);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        d[i] = Row{(uint32_t)(perm_apply(p, i) + 1), (uint32_t)i};
}

__global__ void k_gen_fk(Row *d, uint64_t n, uint64_t maxid, uint64_t seed) {
    const uint64_t iters = n / maxid, rem = n % maxid;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = i / maxid, j = i % maxid;
        const uint64_t m = c < iters ? maxid : rem;
        const Perm p = make_perm(m, mix64(seed + 0x9E37ull * (c + 1)));
        d[i] = Row{(uint32_t)(perm_apply(p, j) + 1), (uint32_t)i};
    }
}

// Zipf(z) over ranks 1..N by rejection-inversion (Hormann & Derflinger 1996,
// "Rejection-inversion to generate variates from monotone discrete
// distributions"): invert the integral H of the hat x^-z, round to the
// nearest rank, accept with the squeeze test.  Exact in distribution.
struct ZipfRI {
    double z, hx1, hn, sq;
    __host__ __device__ static double helper1(double t) {  // log1p(t)/t
        return fabs(t) > 1e-8 ? log1p(t) / t : 1.0 - t * (0.5 - t * (1.0 / 3.0 - 0.25 * t));
    }
    __host__ __device__ static double helper2(double t) {  // expm1(t)/t
        return fabs(t) > 1e-8 ? expm1(t) / t : 1.0 + t * 0.5 * (1.0 + t * (1.0 / 3.0) * (1.0 + 0.25 * t));
    }
    __host__ __device__ double H(double x) const {
        double lx = log(x);
        return helper2((1.0 - z) * lx) * lx;
    }
    __host__ __device__ double h(double x) const { return exp(-z * log(x)); }
    __host__ __device__ double Hinv(double u) const {
        double t = u * (1.0 - z);
        if (t < -1.0) t = -1.0;
        return exp(helper1(t) * u);
    }
    __host__ __device__ void init(double z_, double N) {
        z = z_;
        hx1 = H(1.5) - 1.0;
        hn = H(N + 0.5);
        sq = 2.0 - Hinv(H(2.5) - h(2.0));
    }
};

__device__ __forceinline__ double u01(uint64_t seed, uint64_t ctr) {
    return (double)(mix64(seed ^ mix64(ctr)) >> 11) * (1.0 / 9007199254740992.0);
}

__global__ void k_gen_zipf(Row *d, uint64_t n, uint64_t N, double z, int scatter, uint64_t seed,
                           ZipfRI zr) {
    const Perm p = make_perm(N, seed ^ 0xABCDEFull);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t k;
        if (z == 0.0) {
            k = 1 + (uint64_t)(u01(seed, 2 * i) * (double)N);
            if (k > N) k = N;
        } else {
            k = 1;
            for (uint64_t a = 0; a < 64; a++) {  // expected ~1.1 rounds
                double u = zr.hn + u01(seed, i * 64 + a) * (zr.hx1 - zr.hn);
                double x = zr.Hinv(u);
                double kk = floor(x + 0.5);
                if (kk < 1) kk = 1;
                if (kk > (double)N) kk = (double)N;
                k = (uint64_t)kk;
                if (kk - x <= zr.sq || u >= zr.H(kk + 0.5) - zr.h(kk)) break;
            }
        }
        uint32_t key = scatter ? (uint32_t)(perm_apply(p, k - 1) + 1) : (uint32_t)k;
        d[i] = Row{key, (uint32_t)i};
    }
}

static unsigned gen_grid(uint64_t n) {
    uint64_t g = (n + 255) / 256;
    return (unsigned)std::min<uint64_t>(g, 148ull * 32);
}

cudaError_t launch_gen_pk(Row *d, uint64_t n, uint64_t seed, cudaStream_t st) {
    if (!n) return cudaSuccess;
    k_gen_pk<<<gen_grid(n), 256, 0, st>>>(d, n, seed);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_gen_fk(Row *d, uint64_t n, uint64_t maxid, uint64_t seed, cudaStream_t st) {
    if (!n) return cudaSuccess;
    k_gen_fk<<<gen_grid(n), 256, 0, st>>>(d, n, maxid, seed);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_gen_zipf(Row *d, uint64_t n, uint64_t alphabet, double z, int scatter,
                            uint64_t seed, cudaStream_t st) {
    if (!n) return cudaSuccess;
    ZipfRI zr;
    zr.init(z, (double)alphabet);
    k_gen_zipf<<<gen_grid(n), 256, 0, st>>>(d, n, alphabet, z, scatter, seed, zr);
    count_launch();
    return cudaGetLastError();
}

__global__ void k_checksum(const tbg_row_out *rows, uint64_t n, unsigned long long *out) {
    unsigned long long s = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        s += row_hash(rows[i].key, rows[i].Rpayload, rows[i].Spayload);
    s = warp_sum_u64(s);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(out, s);
}

cudaError_t launch_checksum(const tbg_row_out *rows, uint64_t n, unsigned long long *out,
                            cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess || !n) return e;
    k_checksum<<<gen_grid(n), 256, 0, st>>>(rows, n, out);
    count_launch();
    return cudaGetLastError();
}

}  // namespace tbg
