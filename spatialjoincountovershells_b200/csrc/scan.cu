// Device-wide exclusive prefix sum of u32 values (reduce, scan of partials,
// apply).  Used for the radix sort's digit-major tile histograms.
#include "sjcs_internal.cuh"

namespace sjcs {
namespace {

constexpr int SC_THREADS = 1024;
constexpr int SC_ITEMS = 4;
constexpr int SC_CHUNK = SC_THREADS * SC_ITEMS;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the block total in *total.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t ws[SC_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t incl = warp_incl_scan(v, lane);
    if (lane == 31) ws[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = ws[lane];
        const uint32_t wi = warp_incl_scan(w, lane);
        ws[lane] = wi - w;
        if (lane == 31) *total = wi;
    }
    __syncthreads();
    const uint32_t r = incl - v + ws[warp];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(SC_THREADS) k_scan_reduce(const uint32_t* __restrict__ in, uint64_t m,
                                                            uint32_t* __restrict__ partials) {
    const uint64_t base = (uint64_t)blockIdx.x * SC_CHUNK;
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < SC_ITEMS; ++i) {
        const uint64_t idx = base + (uint64_t)i * SC_THREADS + threadIdx.x;
        if (idx < m) s += in[idx];
    }
    __shared__ uint32_t tot;
    (void)block_excl_scan(s, &tot);
    if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

// One block scans all partials (exclusive), carrying the running total.
__global__ void __launch_bounds__(SC_THREADS) k_scan_partials(uint32_t* __restrict__ p, uint32_t np) {
    __shared__ uint32_t tot;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < np; base += SC_THREADS) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < np ? p[i] : 0u;
        const uint32_t e = block_excl_scan(v, &tot);
        if (i < np) p[i] = e + carry;
        carry += tot;
        __syncthreads();
    }
}

// Each thread owns SC_ITEMS consecutive values (blocked layout).
__global__ void __launch_bounds__(SC_THREADS) k_scan_apply(uint32_t* __restrict__ data, uint64_t m,
                                                           const uint32_t* __restrict__ partials) {
    const uint64_t base = (uint64_t)blockIdx.x * SC_CHUNK + (uint64_t)threadIdx.x * SC_ITEMS;
    uint32_t v[SC_ITEMS];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < SC_ITEMS; ++i) {
        v[i] = (base + i < m) ? data[base + i] : 0u;
        s += v[i];
    }
    __shared__ uint32_t tot;
    uint32_t run = block_excl_scan(s, &tot) + partials[blockIdx.x];
#pragma unroll
    for (int i = 0; i < SC_ITEMS; ++i) {
        if (base + i < m) data[base + i] = run;
        run += v[i];
    }
}

}  // namespace

uint64_t scan_partials_needed(uint64_t m) { return (m + SC_CHUNK - 1) / SC_CHUNK; }

int exclusive_scan_u32(uint32_t* d_data, uint64_t m, cudaStream_t s, uint32_t* partials) {
    if (m == 0) return SJCS_OK;
    const uint64_t nb = (m + SC_CHUNK - 1) / SC_CHUNK;
    if (nb > 0xffffffffull) return fail(SJCS_ERR_INVALID, "scan too large (%llu)", (unsigned long long)m);
    StreamScratch scr(s);
    if (!partials) SJCS_CUDA_TRY(scr.alloc(&partials, nb * sizeof(uint32_t)));
    k_scan_reduce<<<(unsigned)nb, SC_THREADS, 0, s>>>(d_data, m, partials);
    SJCS_LAUNCH_CHECK();
    k_scan_partials<<<1, SC_THREADS, 0, s>>>(partials, (uint32_t)nb);
    SJCS_LAUNCH_CHECK();
    k_scan_apply<<<(unsigned)nb, SC_THREADS, 0, s>>>(d_data, m, partials);
    SJCS_LAUNCH_CHECK();
    return SJCS_OK;
}

}  // namespace sjcs
