// Stable LSD radix sort of (u32 key, 16-byte payload) records, 8- or 9-bit
// digits, reduce-then-scan per digit pass:
//   k_radix_upsweep    per-tile digit histogram           -> hist[digit][tile]
//   exclusive_scan_u32 over hist (digit-major)            -> global slot base of (digit, tile)
//   k_radix_downsweep  stable in-tile rank (warp match),   shared-memory exchange of key and
//                      payload so each digit run leaves as consecutive (coalesced) stores
// No block ever waits on another block.  The payload travels with the key
// through every pass, so no pass reads memory at random.
//
// The reference sorts with 8-bit LSD passes too (Build.c:164-201, 407-534:
// per-thread 256-bin histograms, prefix sums, 32-entry local buffers); here a
// tile of 4096 records plays the role of a thread's slice and the shared-memory
// exchange plays the role of its local buffers.
//
// Key and payload producers and the consumer are functors, so the first pass
// computes keys and payload straight from the caller's coordinates and the
// last pass writes the final layout.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

#include "sjcs_internal.cuh"

namespace sjcs {

constexpr int RS_THREADS = 512;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;  // 4096 records per tile
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_BITS = 8;  // default digit width
constexpr int RS_BINS = 1 << RS_BITS;
constexpr int RS_SUBHIST = 4;  // upsweep: warps share RS_SUBHIST histograms
// dynamic shared memory of the downsweep: exchanged keys + payloads, and for
// array payloads the source slot of every ranked record
constexpr size_t RS_DOWN_SMEM = (size_t)RS_TILE * (sizeof(uint32_t) + sizeof(uint4) + sizeof(uint16_t));

// A digit of BITS bits (8 or 9).  The downsweep keeps one counter per warp
// and bin; a tile holds 4096 records, so 16-bit counters suffice and keep the
// 9-bit downsweep's shared memory at two blocks per SM.
template <int BITS>
struct RsDigit {
    static_assert(BITS == 8 || BITS == 9, "digits of 8 or 9 bits");
    static constexpr int BINS = 1 << BITS;
    using Cnt = typename std::conditional<(BITS > 8), uint16_t, uint32_t>::type;
};

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Intermediate record arrays: keys[n] and payload[n] (uint4).
struct KeysFromArray {
    const uint32_t* __restrict__ keys;
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const { return keys[i]; }
};
struct PayFromArray {
    const uint4* __restrict__ pay;
    __device__ __forceinline__ uint4 operator()(uint64_t i) const { return pay[i]; }
};
struct SinkRecords {
    uint32_t* __restrict__ keys;
    uint4* __restrict__ pay;
    __device__ __forceinline__ void operator()(uint32_t g, uint32_t k, const uint4& v) const {
        keys[g] = k;
        pay[g] = v;
    }
};

// Digit histogram of one tile from the keys a thread holds (item i counted
// when bit i of `valid` is set) -> hist[digit][tile].
template <int BITS>
__device__ __forceinline__ void tile_histogram(const uint32_t (&key)[RS_ITEMS], uint32_t valid, int shift,
                                               uint32_t* __restrict__ hist, uint32_t ntiles) {
    constexpr int BINS = RsDigit<BITS>::BINS;
    __shared__ uint32_t sh[RS_SUBHIST][BINS];
    const int tid = threadIdx.x;
    for (int i = tid; i < RS_SUBHIST * BINS; i += RS_THREADS) (&sh[0][0])[i] = 0;
    __syncthreads();
    uint32_t* mine = sh[(tid >> 5) % RS_SUBHIST];
#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i)
        if (valid & (1u << i)) atomicAdd(&mine[(key[i] >> shift) & (BINS - 1)], 1u);
    __syncthreads();
    for (int d = tid; d < BINS; d += RS_THREADS) {
        uint32_t s = 0;
#pragma unroll
        for (int h = 0; h < RS_SUBHIST; ++h) s += sh[h][d];
        hist[(uint64_t)d * ntiles + blockIdx.x] = s;
    }
}

template <int BITS, class KeyOp>
__global__ void __launch_bounds__(RS_THREADS)
k_radix_upsweep(KeyOp kop, uint64_t n, int shift, uint32_t* __restrict__ hist, uint32_t ntiles) {
    const int tid = threadIdx.x;
    const uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
    // keys first: their loads are in flight while the histograms are cleared
    uint32_t key[RS_ITEMS], valid = 0;
#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i) {
        const uint64_t idx = base + (uint64_t)i * RS_THREADS + tid;
        key[i] = idx < n ? kop(idx) : 0u;
        valid |= (idx < n ? 1u : 0u) << i;
    }
    tile_histogram<BITS>(key, valid, shift, hist, ntiles);
}

// 16-byte asynchronous global -> shared copy (cp.async, L2 only); the copies
// of a thread are awaited with cp_async_wait_all before a block barrier.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

template <class PayOp>
struct PayIsArray {
    static constexpr bool value = false;
};
template <>
struct PayIsArray<PayFromArray> {
    static constexpr bool value = true;
};

// Payload of a first pass over a 16-byte-aligned array of (x, y, z) floats:
// the downsweep stages each tile's 48 KB of particles in shared memory with
// cp.async, then takes the keys (KeyOp::key_of(x, y, z)) and the payloads
// (x, y, z, 0) from there instead of reading each particle twice.
struct PayFromXyzStaged {
    const float* __restrict__ xyz;
    __device__ __forceinline__ uint4 operator()(uint64_t i) const {
        return make_uint4(__float_as_uint(xyz[3 * i]), __float_as_uint(xyz[3 * i + 1]),
                          __float_as_uint(xyz[3 * i + 2]), 0u);
    }
};
template <class PayOp>
struct PayIsXyz {
    static constexpr bool value = false;
};
template <>
struct PayIsXyz<PayFromXyzStaged> {
    static constexpr bool value = true;
};

// First-pass histogram over a 16-byte-aligned (x, y, z) float array: thread t
// of a tile takes its 8 consecutive particles as six 16-byte loads (96 bytes,
// 16-byte aligned because a tile starts at a multiple of 4096 particles) and
// computes their keys with KeyOp::key_of.  Which thread counts which particle
// does not matter to a histogram.
template <int BITS, class KeyOp>
__global__ void __launch_bounds__(RS_THREADS)
k_radix_upsweep_xyz(KeyOp kop, const float* __restrict__ xyz, uint64_t n, int shift, uint32_t* __restrict__ hist,
                    uint32_t ntiles) {
    static_assert(RS_ITEMS == 8, "six float4 per thread hold 8 particles");
    const int tid = threadIdx.x;
    const uint64_t p0 = (uint64_t)blockIdx.x * RS_TILE + (uint64_t)tid * RS_ITEMS;
    uint32_t key[RS_ITEMS], valid = 0;
    if (p0 + RS_ITEMS <= n) {
        const float4* v = reinterpret_cast<const float4*>(xyz + 3 * p0);
        float4 a[6];
#pragma unroll
        for (int j = 0; j < 6; ++j) a[j] = __ldg(v + j);
        const float* f = reinterpret_cast<const float*>(a);
#pragma unroll
        for (int i = 0; i < RS_ITEMS; ++i) key[i] = kop.key_of(f[3 * i], f[3 * i + 1], f[3 * i + 2]);
        valid = 0xffu;
    } else {
#pragma unroll
        for (int i = 0; i < RS_ITEMS; ++i) {
            const uint64_t p = p0 + (uint64_t)i;
            key[i] = p < n ? kop.key_of(xyz[3 * p], xyz[3 * p + 1], xyz[3 * p + 2]) : 0u;
            valid |= (p < n ? 1u : 0u) << i;
        }
    }
    tile_histogram<BITS>(key, valid, shift, hist, ntiles);
}

template <int BITS, class KeyOp, class PayOp, class Sink>
__global__ void __launch_bounds__(RS_THREADS)
k_radix_downsweep(KeyOp kop, PayOp pop, uint64_t n, int shift,
                  const uint32_t* __restrict__ offs, uint32_t ntiles, Sink sink) {
    // Array payloads are copied asynchronously into shared memory in load
    // order as the tile starts, so their latency overlaps the ranking; the
    // ranked records then carry their source slot.  Computed payloads are
    // produced at the scatter, in rank order.
    constexpr bool kAsync = PayIsArray<PayOp>::value;
    constexpr bool kXyz = PayIsXyz<PayOp>::value;  // particles staged in xpay
    constexpr int RS_BINS = RsDigit<BITS>::BINS;  // bins of this pass's digit
    static_assert(RS_BINS <= RS_THREADS, "one thread per bin in the digit scan");
    using Cnt = typename RsDigit<BITS>::Cnt;
    __shared__ Cnt warp_cnt[RS_WARPS][RS_BINS];
    __shared__ uint32_t dstart[RS_BINS];
    __shared__ uint32_t gbase[RS_BINS];
    __shared__ uint32_t wsum[RS_BINS / 32];
    extern __shared__ uint4 xdyn[];
    uint4* xpay = xdyn;                                            // [RS_TILE]: rank order, or load order (kAsync)
    uint32_t* xkey = reinterpret_cast<uint32_t*>(xdyn + RS_TILE);  // [RS_TILE], rank order
    uint16_t* xsrc = reinterpret_cast<uint16_t*>(xkey + RS_TILE);  // [RS_TILE], rank order (kAsync, kXyz)
    const float* sxyz = reinterpret_cast<const float*>(xdyn);      // [3 * RS_TILE] in load order (kXyz)

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t tile = blockIdx.x;
    const uint64_t tile_base = (uint64_t)tile * RS_TILE;
    const uint64_t rem = n - tile_base;
    const uint32_t tile_n = rem < (uint64_t)RS_TILE ? (uint32_t)rem : (uint32_t)RS_TILE;
    const uint32_t wbase = (uint32_t)warp * 32u * RS_ITEMS;
    // The tile's global digit bases are needed only after the ranking: load
    // them now so their latency overlaps it.
    const uint32_t my_gbase = tid < RS_BINS ? offs[(uint64_t)tid * ntiles + tile] : 0u;

    if constexpr (kAsync) {
#pragma unroll
        for (int i = 0; i < RS_ITEMS; ++i) {
            const uint32_t loc = wbase + (uint32_t)i * 32u + (uint32_t)lane;
            if (loc < tile_n) cp_async16(&xpay[loc], pop.pay + tile_base + loc);
        }
    }

    for (int d = lane; d < RS_BINS; d += 32) warp_cnt[warp][d] = 0;
    __syncwarp();
    if constexpr (kXyz) {
        // tile_base * 12 bytes is a multiple of 16; a ragged last tile ends
        // with up to three 4-byte words loaded plainly
        const uint32_t words = tile_n * 3u, chunks = words >> 2;
        const float* src = pop.xyz + 3 * tile_base;
        float* dst = reinterpret_cast<float*>(xdyn);
        for (uint32_t c = (uint32_t)tid; c < chunks; c += RS_THREADS) cp_async16(dst + 4 * c, src + 4 * c);
        for (uint32_t w = chunks * 4u + (uint32_t)tid; w < words; w += RS_THREADS) dst[w] = src[w];
        cp_async_wait_all();
        __syncthreads();
    }

    // Warp w owns tile slots [w*32*ITEMS, (w+1)*32*ITEMS); item i of lane l is
    // slot w*32*ITEMS + i*32 + l, so loads are coalesced and the stable order
    // inside the warp is item-major, lane-minor.
    // All keys are loaded first, so their loads are in flight together; the
    // ranking that follows is a dependent chain through the warp's counters.
    uint32_t key[RS_ITEMS], pos[RS_ITEMS];
#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i) {
        const uint32_t loc = wbase + (uint32_t)i * 32u + (uint32_t)lane;
        if constexpr (kXyz)
            key[i] = loc < tile_n ? kop.key_of(sxyz[3 * loc], sxyz[3 * loc + 1], sxyz[3 * loc + 2]) : 0u;
        else
            key[i] = loc < tile_n ? kop(tile_base + loc) : 0u;
    }
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i) {
        const uint32_t loc = wbase + (uint32_t)i * 32u + (uint32_t)lane;
        const bool valid = loc < tile_n;
        const uint32_t k = key[i];
        const uint32_t d = valid ? ((k >> shift) & (RS_BINS - 1)) : (uint32_t)RS_BINS;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = __popc(peers & lt);
        const uint32_t c = valid ? warp_cnt[warp][d] : 0u;
        __syncwarp();
        if (valid && before == 0) warp_cnt[warp][d] = (Cnt)(c + __popc(peers));
        __syncwarp();
        pos[i] = valid ? c + before : 0xffffffffu;
    }
    __syncthreads();

    // Per digit: exclusive prefix over warps (in place), then an exclusive
    // scan over digits of the tile totals gives each digit's start in the tile.
    uint32_t tot = 0, incl = 0;
    if (tid < RS_BINS) {
#pragma unroll
        for (int w = 0; w < RS_WARPS; ++w) {
            const uint32_t t = warp_cnt[w][tid];
            warp_cnt[w][tid] = (Cnt)tot;
            tot += t;
        }
        incl = tot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) wsum[warp] = incl;
    }
    __syncthreads();
    if (tid < RS_BINS) {
        uint32_t add = 0;
        for (int w = 0; w < warp; ++w) add += wsum[w];
        dstart[tid] = incl - tot + add;
        gbase[tid] = my_gbase;
    }
    __syncthreads();

#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i) {
        if (pos[i] != 0xffffffffu) {
            const uint32_t d = (key[i] >> shift) & (RS_BINS - 1);
            pos[i] += dstart[d] + warp_cnt[warp][d];
            const uint32_t loc = wbase + (uint32_t)i * 32u + (uint32_t)lane;
            xkey[pos[i]] = key[i];
            if constexpr (kAsync || kXyz) xsrc[pos[i]] = (uint16_t)loc;
            else xpay[pos[i]] = pop(tile_base + loc);
        }
    }
    if constexpr (kAsync) cp_async_wait_all();
    __syncthreads();
#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k) {
        const uint32_t j = (uint32_t)tid + (uint32_t)k * RS_THREADS;
        if (j < tile_n) {
            const uint32_t kk = xkey[j];
            const uint32_t d = (kk >> shift) & (RS_BINS - 1);
            uint4 v;
            if constexpr (kXyz) {
                const uint32_t src = xsrc[j];
                v = make_uint4(__float_as_uint(sxyz[3 * src]), __float_as_uint(sxyz[3 * src + 1]),
                               __float_as_uint(sxyz[3 * src + 2]), 0u);
            } else {
                v = kAsync ? xpay[xsrc[j]] : xpay[j];
            }
            // in bounds unless the input changed between the histogram and this pass
            const uint32_t gpos = gbase[d] + (j - dstart[d]);
            if (gpos < n) sink(gpos, kk, v);
        }
    }
}

template <int BITS = RS_BITS, class KeyOp, class PayOp, class Sink>
int radix_pass(KeyOp kop, PayOp pop, Sink sink, uint64_t n, int shift, uint32_t* hist, uint32_t ntiles,
               cudaStream_t s, uint32_t* partials) {
    if constexpr (PayIsXyz<PayOp>::value)
        k_radix_upsweep_xyz<BITS><<<ntiles, RS_THREADS, 0, s>>>(kop, pop.xyz, n, shift, hist, ntiles);
    else
        k_radix_upsweep<BITS><<<ntiles, RS_THREADS, 0, s>>>(kop, n, shift, hist, ntiles);
    SJCS_LAUNCH_CHECK();
    int rc = exclusive_scan_u32(hist, (uint64_t)RsDigit<BITS>::BINS * ntiles, s, partials);
    if (rc) return rc;
    auto kern = k_radix_downsweep<BITS, KeyOp, PayOp, Sink>;
    SJCS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RS_DOWN_SMEM));
    kern<<<ntiles, RS_THREADS, RS_DOWN_SMEM, s>>>(kop, pop, n, shift, hist, ntiles, sink);
    SJCS_LAUNCH_CHECK();
    return SJCS_OK;
}

// Sort n records by their low key_bits key bits.  Pass 0 reads (kop0, pop0);
// the last pass hands every record to `final`; passes in between ping-pong
// through (keys_x, pay_x) and (keys_y, pay_y), arranged so that the pass
// before the last one writes the x buffers.  BITS is the digit width (8 or
// 9): hist holds RsDigit<BITS>::BINS * ntiles u32 and partials (optional)
// holds the scan's scan_partials_needed(RsDigit<BITS>::BINS * ntiles).
template <int BITS = RS_BITS, class KeyOp0, class PayOp0, class FinalSink>
int radix_sort_records(uint64_t n, int key_bits, KeyOp0 kop0, PayOp0 pop0, FinalSink final_sink,
                       uint32_t* keys_x, uint4* pay_x, uint32_t* keys_y, uint4* pay_y, uint32_t* hist,
                       cudaStream_t s, uint32_t* partials = nullptr) {
    if (n == 0) return SJCS_OK;
    const uint32_t ntiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
    const int passes = key_bits <= 0 ? 1 : (key_bits + BITS - 1) / BITS;
    for (int p = 0; p < passes; ++p) {
        const int shift = p * BITS;
        const bool first = (p == 0), last = (p == passes - 1);
        // record buffers written by pass p (p < passes-1): x when (passes-2-p) is even
        const bool to_x = ((passes - 2 - p) % 2) == 0;
        uint32_t* kout = to_x ? keys_x : keys_y;
        uint4* vout = to_x ? pay_x : pay_y;
        uint32_t* kin = to_x ? keys_y : keys_x;  // written by pass p-1
        uint4* vin = to_x ? pay_y : pay_x;
        int rc;
        if (first && last)
            rc = radix_pass<BITS>(kop0, pop0, final_sink, n, shift, hist, ntiles, s, partials);
        else if (first)
            rc = radix_pass<BITS>(kop0, pop0, SinkRecords{kout, vout}, n, shift, hist, ntiles, s, partials);
        else if (last)
            rc = radix_pass<BITS>(KeysFromArray{keys_x}, PayFromArray{pay_x}, final_sink, n, shift, hist, ntiles, s,
                            partials);
        else
            rc = radix_pass<BITS>(KeysFromArray{kin}, PayFromArray{vin}, SinkRecords{kout, vout}, n, shift, hist, ntiles,
                            s, partials);
        if (rc) return rc;
    }
    return SJCS_OK;
}

}  // namespace sjcs
