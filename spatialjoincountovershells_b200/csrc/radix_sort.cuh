// Stable LSD radix sort of (u32 key, u32 value) pairs, 8-bit digits,
// reduce-then-scan per digit pass:
//   k_radix_upsweep    per-tile digit histogram           -> hist[digit][tile]
//   exclusive_scan_u32 over hist (digit-major)            -> global slot base of (digit, tile)
//   k_radix_downsweep  stable in-tile rank (warp match),   shared-memory exchange so that
//                      each digit run leaves as consecutive (coalesced) stores
// No block ever waits on another block.
//
// The reference sorts with 8-bit LSD passes too (Build.c:164-201, 407-534:
// per-thread 256-bin histograms, prefix sums, 32-entry local buffers); here a
// tile of 4096 keys plays the role of a thread's slice and the shared-memory
// exchange plays the role of its local buffers.
//
// Key and value producers and the final consumer are functors, so the first
// pass can compute keys straight from particle coordinates and the last pass
// can gather particle coordinates into sorted order instead of writing
// indices.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace sjcs {

constexpr int RS_THREADS = 512;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;  // 4096 keys per tile
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_BITS = 8;
constexpr int RS_BINS = 1 << RS_BITS;
constexpr int RS_SUBHIST = 4;  // upsweep: warps share RS_SUBHIST histograms

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

struct KeysFromArray {
    const uint32_t* __restrict__ keys;
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const { return keys[i]; }
};
struct ValsFromArray {
    const uint32_t* __restrict__ vals;
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const { return vals[i]; }
};
struct ValsIota {
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const { return (uint32_t)i; }
};
struct SinkPairs {
    uint32_t* __restrict__ keys;
    uint32_t* __restrict__ vals;
    __device__ __forceinline__ void operator()(uint32_t g, uint32_t k, uint32_t v) const {
        keys[g] = k;
        vals[g] = v;
    }
};

template <class KeyOp>
__global__ void __launch_bounds__(RS_THREADS)
k_radix_upsweep(KeyOp kop, uint64_t n, int shift, uint32_t* __restrict__ hist, uint32_t ntiles) {
    __shared__ uint32_t sh[RS_SUBHIST][RS_BINS];
    const int tid = threadIdx.x;
    for (int i = tid; i < RS_SUBHIST * RS_BINS; i += RS_THREADS) (&sh[0][0])[i] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * RS_TILE;
    uint32_t* mine = sh[(tid >> 5) % RS_SUBHIST];
#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i) {
        const uint64_t idx = base + (uint64_t)i * RS_THREADS + tid;
        if (idx < n) atomicAdd(&mine[(kop(idx) >> shift) & (RS_BINS - 1)], 1u);
    }
    __syncthreads();
    for (int d = tid; d < RS_BINS; d += RS_THREADS) {
        uint32_t s = 0;
#pragma unroll
        for (int h = 0; h < RS_SUBHIST; ++h) s += sh[h][d];
        hist[(uint64_t)d * ntiles + blockIdx.x] = s;
    }
}

template <class KeyOp, class ValOp, class Sink>
__global__ void __launch_bounds__(RS_THREADS)
k_radix_downsweep(KeyOp kop, ValOp vop, uint64_t n, int shift,
                  const uint32_t* __restrict__ offs, uint32_t ntiles, Sink sink) {
    __shared__ uint32_t warp_cnt[RS_WARPS][RS_BINS];
    __shared__ uint32_t dstart[RS_BINS];
    __shared__ uint32_t gbase[RS_BINS];
    __shared__ uint32_t wsum[RS_BINS / 32];
    __shared__ uint32_t xbuf[RS_TILE];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t tile = blockIdx.x;
    const uint64_t tile_base = (uint64_t)tile * RS_TILE;
    const uint64_t rem = n - tile_base;
    const uint32_t tile_n = rem < (uint64_t)RS_TILE ? (uint32_t)rem : (uint32_t)RS_TILE;

    for (int d = lane; d < RS_BINS; d += 32) warp_cnt[warp][d] = 0;
    __syncwarp();

    // Warp w owns tile slots [w*32*ITEMS, (w+1)*32*ITEMS); item i of lane l is
    // slot w*32*ITEMS + i*32 + l, so loads are coalesced and the stable order
    // inside the warp is item-major, lane-minor.
    uint32_t key[RS_ITEMS], pos[RS_ITEMS];
    const uint32_t wbase = (uint32_t)warp * 32u * RS_ITEMS;
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i) {
        const uint32_t loc = wbase + (uint32_t)i * 32u + (uint32_t)lane;
        const bool valid = loc < tile_n;
        const uint32_t k = valid ? kop(tile_base + loc) : 0u;
        const uint32_t d = valid ? ((k >> shift) & (RS_BINS - 1)) : (uint32_t)RS_BINS;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = __popc(peers & lt);
        const uint32_t c = valid ? warp_cnt[warp][d] : 0u;
        __syncwarp();
        if (valid && before == 0) warp_cnt[warp][d] = c + __popc(peers);
        __syncwarp();
        key[i] = k;
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
            warp_cnt[w][tid] = tot;
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
        gbase[tid] = offs[(uint64_t)tid * ntiles + tile];
    }
    __syncthreads();

#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i) {
        if (pos[i] != 0xffffffffu) {
            const uint32_t d = (key[i] >> shift) & (RS_BINS - 1);
            pos[i] += dstart[d] + warp_cnt[warp][d];
            xbuf[pos[i]] = key[i];
        }
    }
    __syncthreads();

    uint32_t okey[RS_ITEMS], og[RS_ITEMS];
#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k) {
        const uint32_t j = (uint32_t)tid + (uint32_t)k * RS_THREADS;
        if (j < tile_n) {
            const uint32_t kk = xbuf[j];
            const uint32_t d = (kk >> shift) & (RS_BINS - 1);
            okey[k] = kk;
            og[k] = gbase[d] + (j - dstart[d]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < RS_ITEMS; ++i) {
        if (pos[i] != 0xffffffffu) {
            const uint32_t loc = wbase + (uint32_t)i * 32u + (uint32_t)lane;
            xbuf[pos[i]] = vop(tile_base + loc);
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < RS_ITEMS; ++k) {
        const uint32_t j = (uint32_t)tid + (uint32_t)k * RS_THREADS;
        if (j < tile_n) sink(og[k], okey[k], xbuf[j]);
    }
}

}  // namespace sjcs
