// Grid index build in two passes over the particles: partition by bucket,
// then a counting sort of each bucket -- by a cluster of 8 blocks sharing
// their cell counters through distributed shared memory -- that writes the
// particles in cell order and the bucket's cell offsets.
//
// Replaces the STR bulk load of the reference (MakeTreeWithSameThreadPoolArraySTR,
// src/objects/ArraySTR/Build.c:845-963).  Counts do not depend on the tree
// shape, and none depends on the order of the particles inside a cell, so
// the index only has to group particles by cell and record where each cell
// starts.  Cells are numbered x-fastest; a bucket is 2^L consecutive cell ids
// (L = 16: ~70 rows of x cells of one z layer at the automatic grid, ~2000
// buckets at 2^27 cells).
//
//   k_bucket_hist     chunk c of the AoS input (one chunk per SM): per-bucket
//                     particle counts -> hist[bucket][chunk]
//   scan              exclusive scan of hist (bucket-major): the slot where
//                     chunk c's particles of bucket b go; hist[b][0] is the
//                     start of bucket b
//   k_bucket_scatter  chunk c again: each particle takes the next slot of its
//                     bucket (shared-memory cursor; the order inside a bucket
//                     is free) and is written as (x, y, z, cell id)
//   k_bucket_sort     one cluster of 8 blocks per bucket, block r owning the
//                     bucket's cells [r 2^L/8, (r+1) 2^L/8): each block reads
//                     an eighth of the bucket's records (kept in its shared
//                     memory) and counts them in the owning block's counters
//                     (distributed shared memory atomics); each block scans
//                     its counters into cell_start entries, offset by the
//                     totals of the blocks before it; then every particle
//                     takes the next slot of its cell from the owner's
//                     counter and is written as a float4 into pts
//
// Why these sizes: the scatter's writes of a (chunk, bucket) slice trickle in
// and are merged into whole lines in L2; with one chunk per SM and ~2000
// buckets the slices' open lines (148 x 2044 x 128 B = 39 MB) stay resident
// until they are complete, so every DRAM write is a full sector.  (With
// ~16000 buckets of 2^13 cells they did not: sectors were evicted half
// written and read back to merge, and 32-byte records that fill a sector
// each were written at random DRAM rows -- 3.1-3.9 ms per 1e8 particles.)
// A bucket of 2^16 cells holds ~49k particles at the README scale; split
// over a cluster's 8 SMs that is ~6k records, 98 KB, per block.
//
// Per particle: 12 B read twice, 16 B written and read once, 16 B written;
// per cell 4 B.  No block waits on another block outside its own cluster.
#include <cooperative_groups.h>

#include <algorithm>

#include "sjcs_internal.cuh"

namespace cg = cooperative_groups;

namespace sjcs {
namespace {

constexpr int kBucketBits = 16;          // cells per bucket: 2^16
constexpr uint32_t kMaxBuckets = 16384;  // shared-memory cursors of the scatter (64 KB): grids up to 2^30 cells
constexpr int kClusterBlocks = 8;        // blocks per bucket in the sort
constexpr int BB_THREADS = 512;          // histogram and scatter blocks
constexpr int BS_THREADS = 1024;         // bucket sort blocks
constexpr uint32_t kStageCap = 7168;     // records of a block's share kept in shared memory (112 KB)
constexpr int BB_ITEMS = 8;              // particles per thread per iteration (six float4 loads)
constexpr uint64_t kChunkQuantum = 4096;

struct BucketGeom {
    GridGeom g;
    uint64_t n;
    uint64_t S;     // particles per chunk (multiple of kChunkQuantum)
    uint32_t C;     // chunks
    uint32_t nb;    // buckets
    int L;          // cell bits per bucket
    int lper;       // log2 of the cells each block of the sort owns (max(L - 3, 0))
};

// The keys of the 8 particles p0 .. p0+7 of [p0, end): six 16-byte loads when
// all 8 are present and the array is 16-byte aligned, else scalar loads.
template <bool VEC>
__device__ __forceinline__ uint32_t load8(const float* __restrict__ xyz, uint64_t p0, uint64_t end,
                                          const GridGeom& g, float (&f)[3 * BB_ITEMS], uint32_t (&key)[BB_ITEMS]) {
    uint32_t valid = 0;
    if (VEC && p0 + BB_ITEMS <= end) {
        const float4* v = reinterpret_cast<const float4*>(xyz + 3 * p0);
        float4 a[6];
#pragma unroll
        for (int j = 0; j < 6; ++j) a[j] = __ldcs(v + j);  // read once: stream past L1 and L2
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            f[4 * j] = a[j].x;
            f[4 * j + 1] = a[j].y;
            f[4 * j + 2] = a[j].z;
            f[4 * j + 3] = a[j].w;
        }
        valid = 0xffu;
    } else {
#pragma unroll
        for (int i = 0; i < BB_ITEMS; ++i) {
            const uint64_t p = p0 + (uint64_t)i;
            const bool ok = p < end;
            f[3 * i] = ok ? xyz[3 * p] : 0.0f;
            f[3 * i + 1] = ok ? xyz[3 * p + 1] : 0.0f;
            f[3 * i + 2] = ok ? xyz[3 * p + 2] : 0.0f;
            valid |= (ok ? 1u : 0u) << i;
        }
    }
#pragma unroll
    for (int i = 0; i < BB_ITEMS; ++i) key[i] = cell_key(g, f[3 * i], f[3 * i + 1], f[3 * i + 2]);
    return valid;
}

template <bool VEC>
__global__ void __launch_bounds__(BB_THREADS) k_bucket_hist(const float* __restrict__ xyz, BucketGeom bg,
                                                            uint32_t* __restrict__ hist) {
    extern __shared__ uint32_t cnt[];  // [nb]
    for (uint32_t b = threadIdx.x; b < bg.nb; b += BB_THREADS) cnt[b] = 0u;
    __syncthreads();
    const uint64_t c0 = (uint64_t)blockIdx.x * bg.S;
    const uint64_t c1 = min(bg.n, c0 + bg.S);
    for (uint64_t p0 = c0 + (uint64_t)threadIdx.x * BB_ITEMS; p0 < c1; p0 += (uint64_t)BB_THREADS * BB_ITEMS) {
        float f[3 * BB_ITEMS];
        uint32_t key[BB_ITEMS];
        const uint32_t valid = load8<VEC>(xyz, p0, c1, bg.g, f, key);
#pragma unroll
        for (int i = 0; i < BB_ITEMS; ++i)
            if (valid & (1u << i)) atomicAdd(&cnt[key[i] >> bg.L], 1u);
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < bg.nb; b += BB_THREADS) hist[(uint64_t)b * bg.C + blockIdx.x] = cnt[b];
}

template <bool VEC>
__global__ void __launch_bounds__(BB_THREADS) k_bucket_scatter(const float* __restrict__ xyz, BucketGeom bg,
                                                               const uint32_t* __restrict__ offs,
                                                               uint4* __restrict__ part) {
    extern __shared__ uint32_t cur[];  // [nb]: next slot of each bucket for this chunk
    for (uint32_t b = threadIdx.x; b < bg.nb; b += BB_THREADS) cur[b] = offs[(uint64_t)b * bg.C + blockIdx.x];
    __syncthreads();
    const uint64_t c0 = (uint64_t)blockIdx.x * bg.S;
    const uint64_t c1 = min(bg.n, c0 + bg.S);
    for (uint64_t p0 = c0 + (uint64_t)threadIdx.x * BB_ITEMS; p0 < c1; p0 += (uint64_t)BB_THREADS * BB_ITEMS) {
        float f[3 * BB_ITEMS];
        uint32_t key[BB_ITEMS];
        const uint32_t valid = load8<VEC>(xyz, p0, c1, bg.g, f, key);
#pragma unroll
        for (int i = 0; i < BB_ITEMS; ++i) {
            if (valid & (1u << i)) {
                const uint32_t slot = atomicAdd(&cur[key[i] >> bg.L], 1u);
                part[slot] = make_uint4(__float_as_uint(f[3 * i]), __float_as_uint(f[3 * i + 1]),
                                        __float_as_uint(f[3 * i + 2]), key[i]);
            }
        }
    }
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// In-place exclusive scan of a[0 .. m) (m a power of two) in shared memory
// by the whole block (a multiple of 32 threads, at most 1024): warp w scans
// its segment of m / warps entries (lanes read consecutive words, no bank
// conflicts), then adds the totals of the segments before it.  wsum holds
// one word per warp.  Returns the sum of all entries.
__device__ uint32_t block_excl_scan(uint32_t* a, uint32_t m, uint32_t* wsum) {
    const uint32_t NW = blockDim.x >> 5;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t seg = m / NW;  // >= 32 unless m is small: then warp 0 alone
    uint32_t total = 0;
    if (seg >= 32) {
        uint32_t carry = 0;
        for (uint32_t k = 0; k < seg; k += 32) {
            uint32_t* e = a + (uint32_t)warp * seg + k + (uint32_t)lane;
            const uint32_t v = *e;
            const uint32_t incl = warp_incl_scan(v, lane);
            *e = carry + incl - v;
            carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) wsum[warp] = carry;
        __syncthreads();
        uint32_t add = 0;
        for (uint32_t w = 0; w < NW; ++w) {
            if (w < (uint32_t)warp) add += wsum[w];
            total += wsum[w];
        }
        for (uint32_t k = lane; k < seg; k += 32) a[(uint32_t)warp * seg + k] += add;
        __syncthreads();
    } else {
        if (warp == 0) {
            uint32_t carry = 0;
            for (uint32_t k = 0; k < m; k += 32) {
                const uint32_t i = k + (uint32_t)lane;
                const uint32_t v = i < m ? a[i] : 0u;
                const uint32_t incl = warp_incl_scan(v, lane);
                if (i < m) a[i] = carry + incl - v;
                carry += __shfl_sync(0xffffffffu, incl, 31);
            }
            if (lane == 0) wsum[0] = carry;
        }
        __syncthreads();
        total = wsum[0];
        __syncthreads();
    }
    return total;
}

__global__ void __cluster_dims__(kClusterBlocks, 1, 1) __launch_bounds__(BS_THREADS, 1)
    k_bucket_sort(const uint4* __restrict__ part, BucketGeom bg, const uint32_t* __restrict__ offs,
                  float4* __restrict__ pts, uint32_t* __restrict__ cs) {
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ uint32_t wsum[BS_THREADS / 32];
    __shared__ uint32_t block_total;
    cg::cluster_group cluster = cg::this_cluster();
    const uint32_t rank = cluster.block_rank();
    const uint32_t b = blockIdx.x / kClusterBlocks;  // the cluster's bucket
    const uint32_t per = 1u << bg.lper;              // cells owned by each block of the cluster
    const uint32_t per_words = per < 4u ? 4u : per;  // keeps the stage 16-byte aligned
    uint32_t* cnt = smem;
    uint4* stage = reinterpret_cast<uint4*>(smem + per_words);
    const uint32_t tid = threadIdx.x, T = blockDim.x;
    const uint32_t bucket_cells = 1u << bg.L;
    const uint64_t cell0 = (uint64_t)b << bg.L;
    const uint32_t bs = offs[(uint64_t)b * bg.C];
    const uint32_t be = (b + 1 < bg.nb) ? offs[(uint64_t)(b + 1) * bg.C] : (uint32_t)bg.n;
    const uint32_t m = be - bs;
    // this block's share of the bucket's records
    const uint32_t lo = bs + (uint32_t)((uint64_t)m * rank / kClusterBlocks);
    const uint32_t hi = bs + (uint32_t)((uint64_t)m * (rank + 1) / kClusterBlocks);
    const uint32_t ms = hi - lo;
    const bool staged = ms <= kStageCap;
    for (uint32_t c = tid; c < per_words; c += T) cnt[c] = 0u;
    cluster.sync();
    for (uint32_t i = tid; i < ms; i += T) {
        const uint4 r = part[lo + i];
        if (staged) stage[i] = r;
        const uint32_t local = r.w - (uint32_t)cell0;
        atomicAdd(cluster.map_shared_rank(cnt, (int)(local >> bg.lper)) + (local & (per - 1u)), 1u);
    }
    cluster.sync();
    const uint32_t tot = block_excl_scan(cnt, per, wsum);
    if (tid == 0) block_total = tot;
    cluster.sync();
    uint32_t base = bs;
    for (uint32_t r = 0; r < rank; ++r) base += *cluster.map_shared_rank(&block_total, (int)r);
    for (uint32_t c = tid; c < per; c += T) {
        const uint32_t local = rank * per + c;
        const uint64_t cell = cell0 + local;
        if (local < bucket_cells && cell < bg.g.ncells) cs[cell] = base + cnt[c];
        cnt[c] += base;
    }
    if (b == 0 && rank == 0 && tid == 0) cs[bg.g.ncells] = (uint32_t)bg.n;
    cluster.sync();
    for (uint32_t i = tid; i < ms; i += T) {
        const uint4 r = staged ? stage[i] : part[lo + i];
        const uint32_t local = r.w - (uint32_t)cell0;
        const uint32_t slot = atomicAdd(cluster.map_shared_rank(cnt, (int)(local >> bg.lper)) + (local & (per - 1u)), 1u);
        pts[slot] = make_float4(__uint_as_float(r.x), __uint_as_float(r.y), __uint_as_float(r.z), 0.0f);
    }
    cluster.sync();  // no block leaves while others still use its counters
}

BucketGeom bucket_geom(const GridGeom& g, uint64_t n, int num_sms) {
    BucketGeom bg{};
    bg.g = g;
    bg.n = n;
    const int kb = grid_key_bits(g);
    bg.L = std::min(kb, kBucketBits);
    bg.lper = std::max(bg.L - 3, 0);
    bg.nb = (uint32_t)((g.ncells + (1ull << bg.L) - 1) >> bg.L);
    // one chunk per SM, a whole number of 4096-particle quanta
    const uint64_t want = (n + (uint64_t)num_sms - 1) / (uint64_t)num_sms;
    bg.S = std::max(kChunkQuantum, (want + kChunkQuantum - 1) / kChunkQuantum * kChunkQuantum);
    bg.C = (uint32_t)((n + bg.S - 1) / bg.S);
    return bg;
}

}  // namespace

bool bucket_build_eligible(const GridGeom& g, uint64_t n) {
    if (n == 0 || n >= 0xffffffffull) return false;
    const int kb = grid_key_bits(g);
    const int L = std::min(kb, kBucketBits);
    const uint64_t nb = (g.ncells + (1ull << L) - 1) >> L;
    return nb <= kMaxBuckets;
}

BucketBuildSizes bucket_build_sizes(const GridGeom& g, uint64_t n, int num_sms) {
    const BucketGeom bg = bucket_geom(g, n, num_sms);
    BucketBuildSizes z{};
    z.part = n;
    z.hist = (uint64_t)bg.nb * bg.C;
    z.partials = scan_partials_needed(z.hist);
    return z;
}

int build_grid_bucketed(const float* d_xyz, uint64_t n, const GridGeom& g, int num_sms, const BucketBuildBuffers& b,
                        cudaStream_t s) {
    const BucketGeom bg = bucket_geom(g, n, num_sms);
    const bool vec = (reinterpret_cast<uintptr_t>(d_xyz) & 15u) == 0;  // S * 12 bytes keeps chunks 16-byte aligned
    const size_t smem_b = (size_t)bg.nb * sizeof(uint32_t);
    if (vec) {
        SJCS_CUDA_TRY(cudaFuncSetAttribute(k_bucket_hist<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_b));
        k_bucket_hist<true><<<bg.C, BB_THREADS, smem_b, s>>>(d_xyz, bg, b.hist);
    } else {
        SJCS_CUDA_TRY(cudaFuncSetAttribute(k_bucket_hist<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_b));
        k_bucket_hist<false><<<bg.C, BB_THREADS, smem_b, s>>>(d_xyz, bg, b.hist);
    }
    SJCS_LAUNCH_CHECK();
    int rc = exclusive_scan_u32(b.hist, (uint64_t)bg.nb * bg.C, s, b.partials);
    if (rc) return rc;
    if (vec) {
        SJCS_CUDA_TRY(cudaFuncSetAttribute(k_bucket_scatter<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_b));
        k_bucket_scatter<true><<<bg.C, BB_THREADS, smem_b, s>>>(d_xyz, bg, b.hist, b.part);
    } else {
        SJCS_CUDA_TRY(cudaFuncSetAttribute(k_bucket_scatter<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_b));
        k_bucket_scatter<false><<<bg.C, BB_THREADS, smem_b, s>>>(d_xyz, bg, b.hist, b.part);
    }
    SJCS_LAUNCH_CHECK();
    const uint32_t per = 1u << bg.lper;
    const size_t smem_s = (size_t)std::max(per, 4u) * sizeof(uint32_t) + (size_t)kStageCap * sizeof(uint4);
    SJCS_CUDA_TRY(cudaFuncSetAttribute(k_bucket_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s));
    k_bucket_sort<<<bg.nb * kClusterBlocks, BS_THREADS, smem_s, s>>>(b.part, bg, b.hist, b.pts, b.cell_start);
    SJCS_LAUNCH_CHECK();
    return SJCS_OK;
}

}  // namespace sjcs
