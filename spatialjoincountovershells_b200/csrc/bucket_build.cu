// Grid index build in two passes over the particles: partition by bucket,
// then a counting sort of each bucket that writes its cells' offsets.
//
// Replaces the STR bulk load of the reference (MakeTreeWithSameThreadPoolArraySTR,
// src/objects/ArraySTR/Build.c:845-963).  Counts do not depend on the tree
// shape, and none depends on the order of the particles inside a cell, so
// the index only has to group particles by cell and record where each cell
// starts.  Cells are numbered x-fastest; a bucket is 2^L consecutive cell ids
// (L = 13: ~8.7 rows of x cells of one z layer at the automatic grid).
//
//   k_bucket_hist     chunk c of the AoS input (S particles): per-bucket
//                     particle counts -> hist[bucket][chunk]
//   scan              exclusive scan of hist (bucket-major): the slot where
//                     chunk c's particles of bucket b go; hist[b][0] is the
//                     start of bucket b
//   k_bucket_scatter  chunk c again: each particle takes the next slot of its
//                     bucket (shared-memory cursor; the order inside a bucket
//                     is free) and is written as one 32-byte record
//                     (x, y, z, cell id, padding) with a single 256-bit store
//   k_bucket_sort     persistent, one block per SM walking the buckets: per
//                     bucket, counts per cell in shared memory (the records
//                     kept in shared memory too), their exclusive scan gives
//                     the bucket's cell_start entries, then every particle
//                     takes the next slot of its cell and is written as a
//                     float4 into pts
//   k_heavy_*         buckets of more than kHeavy particles (clustered data)
//                     are left by k_bucket_sort to three grid-wide kernels
//                     that do the same with global-memory counters, so no
//                     bucket holds one block for long
//
// Why 32-byte records: the scatter sends every particle to one of ~16k
// buckets, so consecutive records of a bucket slice arrive far apart in time.
// A 16-byte record leaves its 32-byte DRAM sector half written; when L2
// evicts it before the other half arrives, the memory controller reads the
// sector back to merge it.  A record that fills its sector is written whole.
// The sort kernel keeps few buckets in flight (one per SM), so its scattered
// 16-byte writes complete their lines in L2.
//
// Per particle: 12 B read twice, 32 B written and read once, 16 B written;
// per cell 4 B.  No block waits on another block.
#include <algorithm>

#include "sjcs_internal.cuh"

namespace sjcs {
namespace {

constexpr int kLocalBits = 13;           // cells per bucket: 2^13
constexpr uint32_t kMaxBuckets = 16384;  // shared-memory cursors of the scatter (64 KB)
constexpr uint64_t kHeavy = 1u << 18;    // particles above which a bucket takes the grid-wide path
constexpr int BB_THREADS = 512;          // histogram, scatter and heavy-scan blocks
constexpr int BS_THREADS = 1024;         // bucket sort blocks (one per SM)
constexpr uint32_t kStageCap = 11264;    // records of one bucket kept in shared memory (176 KB)
constexpr int BB_ITEMS = 8;              // particles per thread per iteration (six float4 loads)
constexpr uint64_t kChunkQuantum = 4096;

struct alignas(32) PartRec {
    uint32_t x, y, z, cell;
    uint32_t pad[4];
};
static_assert(sizeof(PartRec) == 32, "partition records fill one 32-byte sector");

struct BucketGeom {
    GridGeom g;
    uint64_t n;
    uint64_t S;     // particles per chunk (multiple of kChunkQuantum)
    uint32_t C;     // chunks
    uint32_t nb;    // buckets
    int L;          // cell bits per bucket
};

struct HeavyList {
    uint32_t* count;    // number of heavy buckets
    uint32_t* ids;      // their bucket ids
    uint32_t* cursors;  // [max heavy][2^L] running slot of every cell
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

// One 32-byte record (one 256-bit store: the sector is written whole).
__device__ __forceinline__ void store_rec(PartRec* dst, float x, float y, float z, uint32_t cell) {
    asm volatile("st.global.v8.b32 [%0], {%1, %2, %3, %4, %5, %5, %5, %5};" ::"l"(dst), "r"(__float_as_uint(x)),
                 "r"(__float_as_uint(y)), "r"(__float_as_uint(z)), "r"(cell), "r"(0u)
                 : "memory");
}

// The first 16 bytes of a record: (x, y, z, cell).
__device__ __forceinline__ uint4 load_rec(const PartRec* src) { return __ldg(reinterpret_cast<const uint4*>(src)); }

template <bool VEC>
__global__ void __launch_bounds__(BB_THREADS) k_bucket_scatter(const float* __restrict__ xyz, BucketGeom bg,
                                                               const uint32_t* __restrict__ offs,
                                                               PartRec* __restrict__ part) {
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
                store_rec(part + slot, f[3 * i], f[3 * i + 1], f[3 * i + 2], key[i]);
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

// In-place exclusive scan of a[0 .. 2^L) in shared memory by the whole block
// (a multiple of 32 threads, at most 1024): warp w scans its segment of
// 2^L / warps entries (lanes read consecutive words, no bank conflicts), then
// adds the totals of the segments before it.  wsum holds one word per warp.
__device__ void block_excl_scan_cells(uint32_t* a, uint32_t ncells_pow2, uint32_t* wsum) {
    const uint32_t NW = blockDim.x >> 5;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t seg = ncells_pow2 / NW;  // >= 32 unless 2^L is small: then warp 0 alone
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
        for (int w = 0; w < warp; ++w) add += wsum[w];
        for (uint32_t k = lane; k < seg; k += 32) a[(uint32_t)warp * seg + k] += add;
        __syncthreads();
    } else {
        if (warp == 0) {
            uint32_t carry = 0;
            for (uint32_t k = 0; k < ncells_pow2; k += 32) {
                const uint32_t i = k + (uint32_t)lane;
                const uint32_t v = i < ncells_pow2 ? a[i] : 0u;
                const uint32_t incl = warp_incl_scan(v, lane);
                if (i < ncells_pow2) a[i] = carry + incl - v;
                carry += __shfl_sync(0xffffffffu, incl, 31);
            }
        }
        __syncthreads();
    }
}

__device__ __forceinline__ void bucket_range(const BucketGeom& bg, const uint32_t* __restrict__ offs, uint32_t b,
                                             uint32_t* bs, uint32_t* be) {
    *bs = offs[(uint64_t)b * bg.C];
    *be = (b + 1 < bg.nb) ? offs[(uint64_t)(b + 1) * bg.C] : (uint32_t)bg.n;
}

__global__ void __launch_bounds__(BS_THREADS, 1) k_bucket_sort(const PartRec* __restrict__ part, BucketGeom bg,
                                                               const uint32_t* __restrict__ offs,
                                                               float4* __restrict__ pts, uint32_t* __restrict__ cs,
                                                               HeavyList hl) {
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ uint32_t wsum[BS_THREADS / 32];
    const uint32_t ncl_pow2 = 1u << bg.L;
    uint32_t* cnt = smem;                                       // [2^L]
    uint4* stage = reinterpret_cast<uint4*>(smem + ncl_pow2);   // [kStageCap]
    const uint32_t tid = threadIdx.x, T = blockDim.x;
    const uint32_t mask = ncl_pow2 - 1u;
    if (blockIdx.x == 0 && tid == 0) cs[bg.g.ncells] = (uint32_t)bg.n;
    for (uint32_t b = blockIdx.x; b < bg.nb; b += gridDim.x) {
        const uint64_t cell0 = (uint64_t)b << bg.L;
        const uint32_t ncl = (uint32_t)min((uint64_t)ncl_pow2, bg.g.ncells - cell0);
        uint32_t bs, be;
        bucket_range(bg, offs, b, &bs, &be);
        const uint32_t m = be - bs;
        if ((uint64_t)m > kHeavy) {
            // the grid-wide kernels count this bucket in the cell table itself
            for (uint32_t c = tid; c < ncl; c += T) cs[cell0 + c] = 0u;
            if (tid == 0) hl.ids[atomicAdd(hl.count, 1u)] = b;
            continue;
        }
        const bool staged = m <= kStageCap;
        for (uint32_t c = tid; c < ncl_pow2; c += T) cnt[c] = 0u;
        __syncthreads();
        for (uint32_t i = tid; i < m; i += T) {
            const uint4 r = load_rec(part + bs + i);
            if (staged) stage[i] = r;
            atomicAdd(&cnt[r.w & mask], 1u);
        }
        __syncthreads();
        block_excl_scan_cells(cnt, ncl_pow2, wsum);
        for (uint32_t c = tid; c < ncl; c += T) cs[cell0 + c] = bs + cnt[c];
        __syncthreads();
        for (uint32_t i = tid; i < m; i += T) {
            const uint4 r = staged ? stage[i] : load_rec(part + bs + i);
            const uint32_t slot = bs + atomicAdd(&cnt[r.w & mask], 1u);
            pts[slot] = make_float4(__uint_as_float(r.x), __uint_as_float(r.y), __uint_as_float(r.z), 0.0f);
        }
        __syncthreads();  // cnt and stage are reused by the next bucket
    }
}

// ---- heavy buckets: the same counting sort with global-memory counters -----

// Lanes of a warp holding the same cell add once (clustered buckets crowd
// into few cells); returns the running value before this lane's own add.
__device__ __forceinline__ uint32_t aggregated_add(uint32_t* ctr, uint32_t cell, bool live) {
    const uint32_t key = live ? cell : 0xffffffffu;
    const uint32_t peers = __match_any_sync(0xffffffffu, key);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (live && lane == leader) base = atomicAdd(ctr, (uint32_t)__popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
}

__global__ void k_heavy_count(const PartRec* __restrict__ part, BucketGeom bg, const uint32_t* __restrict__ offs,
                              uint32_t* __restrict__ cs, HeavyList hl) {
    const uint32_t nh = *hl.count;
    const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t k = 0; k < nh; ++k) {
        uint32_t bs, be;
        bucket_range(bg, offs, hl.ids[k], &bs, &be);
        // warp-uniform trip count: every lane takes part in the aggregation
        for (uint64_t base = bs + (t0 & ~31ull); base < be; base += T) {
            const uint64_t i = base + (t0 & 31);
            const bool live = i < be;
            const uint32_t cell = live ? load_rec(part + i).w : 0u;
            (void)aggregated_add(cs + cell, cell, live);
        }
    }
}

__global__ void __launch_bounds__(BB_THREADS) k_heavy_scan(BucketGeom bg, const uint32_t* __restrict__ offs,
                                                           uint32_t* __restrict__ cs, HeavyList hl) {
    extern __shared__ uint32_t a[];  // [2^L]
    __shared__ uint32_t wsum[BB_THREADS / 32];
    const uint32_t nh = *hl.count;
    const uint32_t ncl_pow2 = 1u << bg.L;
    for (uint32_t k = blockIdx.x; k < nh; k += gridDim.x) {
        const uint32_t b = hl.ids[k];
        const uint64_t cell0 = (uint64_t)b << bg.L;
        const uint32_t ncl = (uint32_t)min((uint64_t)ncl_pow2, bg.g.ncells - cell0);
        uint32_t bs, be;
        bucket_range(bg, offs, b, &bs, &be);
        for (uint32_t c = threadIdx.x; c < ncl_pow2; c += BB_THREADS) a[c] = c < ncl ? cs[cell0 + c] : 0u;
        __syncthreads();
        block_excl_scan_cells(a, ncl_pow2, wsum);
        for (uint32_t c = threadIdx.x; c < ncl; c += BB_THREADS) {
            cs[cell0 + c] = bs + a[c];
            hl.cursors[(uint64_t)k * ncl_pow2 + c] = bs + a[c];
        }
        __syncthreads();
    }
}

__global__ void k_heavy_scatter(const PartRec* __restrict__ part, BucketGeom bg, const uint32_t* __restrict__ offs,
                                float4* __restrict__ pts, HeavyList hl) {
    const uint32_t nh = *hl.count;
    const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t mask = (1u << bg.L) - 1u;
    for (uint32_t k = 0; k < nh; ++k) {
        uint32_t bs, be;
        bucket_range(bg, offs, hl.ids[k], &bs, &be);
        uint32_t* cur = hl.cursors + ((uint64_t)k << bg.L);
        for (uint64_t base = bs + (t0 & ~31ull); base < be; base += T) {
            const uint64_t i = base + (t0 & 31);
            const bool live = i < be;
            const uint4 r = live ? load_rec(part + i) : make_uint4(0u, 0u, 0u, 0u);
            const uint32_t local = r.w & mask;
            const uint32_t slot = aggregated_add(cur + local, local, live);
            if (live) pts[slot] = make_float4(__uint_as_float(r.x), __uint_as_float(r.y), __uint_as_float(r.z), 0.0f);
        }
    }
}

__global__ void k_zero_u32(uint32_t* p) { *p = 0u; }

BucketGeom bucket_geom(const GridGeom& g, uint64_t n, int num_sms) {
    BucketGeom bg{};
    bg.g = g;
    bg.n = n;
    const int kb = grid_key_bits(g);
    bg.L = std::min(kb, kLocalBits);
    bg.nb = (uint32_t)((g.ncells + (1ull << bg.L) - 1) >> bg.L);
    // about four chunks per SM, each a whole number of 4096-particle quanta
    const uint64_t want = (n + (uint64_t)num_sms * 4 - 1) / ((uint64_t)num_sms * 4);
    bg.S = std::max(kChunkQuantum, (want + kChunkQuantum - 1) / kChunkQuantum * kChunkQuantum);
    bg.C = (uint32_t)((n + bg.S - 1) / bg.S);
    return bg;
}

}  // namespace

bool bucket_build_eligible(const GridGeom& g, uint64_t n) {
    if (n == 0 || n >= 0xffffffffull) return false;
    const int kb = grid_key_bits(g);
    const int L = std::min(kb, kLocalBits);
    const uint64_t nb = (g.ncells + (1ull << L) - 1) >> L;
    return nb <= kMaxBuckets;
}

BucketBuildSizes bucket_build_sizes(const GridGeom& g, uint64_t n, int num_sms) {
    const BucketGeom bg = bucket_geom(g, n, num_sms);
    BucketBuildSizes z{};
    z.part = n;
    z.hist = (uint64_t)bg.nb * bg.C;
    z.partials = scan_partials_needed(z.hist);
    z.max_heavy = n / kHeavy + 1;
    z.cursors = z.max_heavy << bg.L;
    return z;
}

size_t bucket_record_bytes() { return sizeof(PartRec); }

int build_grid_bucketed(const float* d_xyz, uint64_t n, const GridGeom& g, int num_sms, const BucketBuildBuffers& b,
                        cudaStream_t s) {
    const BucketGeom bg = bucket_geom(g, n, num_sms);
    const bool vec = (reinterpret_cast<uintptr_t>(d_xyz) & 15u) == 0;  // S * 12 bytes keeps chunks 16-byte aligned
    if ((reinterpret_cast<uintptr_t>(b.part) & 31u) != 0)
        return fail(SJCS_ERR_INVALID, "bucket build: the record buffer must be 32-byte aligned");
    PartRec* part = static_cast<PartRec*>(b.part);
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
        k_bucket_scatter<true><<<bg.C, BB_THREADS, smem_b, s>>>(d_xyz, bg, b.hist, part);
    } else {
        SJCS_CUDA_TRY(cudaFuncSetAttribute(k_bucket_scatter<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_b));
        k_bucket_scatter<false><<<bg.C, BB_THREADS, smem_b, s>>>(d_xyz, bg, b.hist, part);
    }
    SJCS_LAUNCH_CHECK();
    k_zero_u32<<<1, 1, 0, s>>>(b.heavy_count);
    SJCS_LAUNCH_CHECK();
    const HeavyList hl{b.heavy_count, b.heavy_ids, b.cursors};
    const size_t smem_c = ((size_t)1 << bg.L) * sizeof(uint32_t);
    const size_t smem_s = smem_c + (size_t)kStageCap * sizeof(uint4);
    SJCS_CUDA_TRY(cudaFuncSetAttribute(k_bucket_sort, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_s));
    const unsigned sort_grid = std::min<unsigned>(bg.nb, (unsigned)num_sms);
    k_bucket_sort<<<sort_grid, BS_THREADS, smem_s, s>>>(part, bg, b.hist, b.pts, b.cell_start, hl);
    SJCS_LAUNCH_CHECK();
    // buckets of more than kHeavy particles (none on uniform data): the three
    // kernels below find an empty list and return at once
    k_heavy_count<<<num_sms * 4, 256, 0, s>>>(part, bg, b.hist, b.cell_start, hl);
    SJCS_LAUNCH_CHECK();
    SJCS_CUDA_TRY(cudaFuncSetAttribute(k_heavy_scan, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_c));
    k_heavy_scan<<<num_sms, BB_THREADS, smem_c, s>>>(bg, b.hist, b.cell_start, hl);
    SJCS_LAUNCH_CHECK();
    k_heavy_scatter<<<num_sms * 4, 256, 0, s>>>(part, bg, b.hist, b.pts, hl);
    SJCS_LAUNCH_CHECK();
    return SJCS_OK;
}

}  // namespace sjcs
