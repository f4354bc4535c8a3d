// Morton index build (plain Morton offset table and learned rank model).
//
// Like the grid index this replaces the reference's STR bulk load
// (MakeTreeWithSameThreadPoolArraySTR, src/objects/ArraySTR/Build.c:845-963):
// the counts do not depend on the index's shape, only on which particles lie
// in each query box, so any layout that hands the count kernel a superset of
// the in-box particles gives the reference's counts.
//
// Build of one particle file:
//   sort     stable LSD radix sort by the 63-bit Morton key, 8 passes of 8
//            bits.  The key is carried as two u32 halves: passes 0-3 sort on
//            the low half with the high half riding in the payload's 4th word,
//            pass 4 swaps them, passes 4-7 sort on the high half.  The last
//            pass writes the particles as float4 (4th word = the key's level-10
//            prefix), the level-L cell of every particle and (learned kind)
//            the full keys
//   table    table[c] = first slot of level-L cell c (the plain offset table)
//   train    (learned kind) root from kmin/kmax, exact leaf rank ranges,
//            anchor + fp32 slope per leaf, per-leaf max error over all keys
//   judge    (learned kind, on request) the corrected model rank of every
//            level-L cell boundary is compared with the table; any mismatch
//            switches the count kernel to the table for this index
#include <algorithm>
#include <cmath>

#include "morton.cuh"
#include "radix_sort.cuh"
#include "sjcs_internal.cuh"

namespace sjcs {
namespace {

struct MortonLoKey {
    const float* __restrict__ xyz;
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const {
        return (uint32_t)morton63(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    }
};
struct MortonPay {  // (x, y, z, high half of the key)
    const float* __restrict__ xyz;
    __device__ __forceinline__ uint4 operator()(uint64_t i) const {
        const float x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        return make_uint4(__float_as_uint(x), __float_as_uint(y), __float_as_uint(z),
                          (uint32_t)(morton63(x, y, z) >> 32));
    }
};
struct KeyFromPayW {
    const uint4* __restrict__ pay;
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const { return pay[i].w; }
};
struct PaySwapKey {  // payload's 4th word becomes the low half carried so far
    const uint32_t* __restrict__ keys;
    const uint4* __restrict__ pay;
    __device__ __forceinline__ uint4 operator()(uint64_t i) const {
        const uint4 v = pay[i];
        return make_uint4(v.x, v.y, v.z, keys[i]);
    }
};
// Last pass: key = high half, payload.w = low half.
struct SinkMorton {
    uint4* __restrict__ pts;
    uint32_t* __restrict__ cells;                  // level-L cell of every slot
    unsigned long long* __restrict__ keys;         // full keys (learned kind) or null
    int cell_shift;                                // 31 - 3L: high half -> level-L cell
    __device__ __forceinline__ void operator()(uint32_t g, uint32_t hi, const uint4& v) const {
        pts[g] = make_uint4(v.x, v.y, v.z, hi >> 1);  // level-10 prefix = key >> 33
        cells[g] = hi >> cell_shift;
        if (keys) keys[g] = ((unsigned long long)hi << 32) | v.w;
    }
};

// ---- training --------------------------------------------------------------

__global__ void k_root(const unsigned long long* __restrict__ keys, uint64_t n, LearnedRoot* rt) {
    LearnedRoot r{};
    r.kmin = keys[0];
    r.kmax = keys[n - 1];
    uint32_t sh = 0;
    while (((r.kmax - r.kmin) >> sh) >= kLeaves) ++sh;
    r.shift = sh;
    r.n = (uint32_t)n;
    *rt = r;
}

// first[j] = first rank whose key lies in leaf j or later (first[4096] = n).
__global__ void k_leaf_bounds(const unsigned long long* __restrict__ keys, uint64_t n,
                              const LearnedRoot* __restrict__ rt, uint32_t* __restrict__ first) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    const LearnedRoot r = *rt;
    const int64_t jp = (i == 0) ? -1 : (int64_t)leaf_of(r, keys[i - 1]);
    const int64_t jc = (i == n) ? (int64_t)kLeaves : (int64_t)leaf_of(r, keys[i]);
    for (int64_t j = jp + 1; j <= jc; ++j) first[j] = (uint32_t)i;
}

__global__ void k_leaf_fit(const unsigned long long* __restrict__ keys, const uint32_t* __restrict__ first,
                           LearnedLeaf* __restrict__ leaves) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= kLeaves) return;
    LearnedLeaf lf{};
    lf.r0 = first[j];
    lf.r1 = first[j + 1];
    if (lf.r1 > lf.r0) {
        lf.anchor = keys[lf.r0];
        const unsigned long long last = keys[lf.r1 - 1];
        if (lf.r1 - lf.r0 >= 2 && last > lf.anchor)
            lf.slope = (float)(lf.r1 - lf.r0 - 1) / __ull2float_rn(last - lf.anchor);
    }
    leaves[j] = lf;
}

// err[leaf] = max |P(k_i) - i|, one warp-aggregated atomic per leaf run.
__global__ void k_leaf_err(const unsigned long long* __restrict__ keys, uint64_t n,
                           const LearnedRoot* __restrict__ rt, LearnedLeaf* __restrict__ leaves) {
    const LearnedRoot r = *rt;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const uint64_t i = base + threadIdx.x;
        const bool valid = i < n;
        uint32_t j = 0xffffffffu, e = 0;
        if (valid) {
            const unsigned long long k = keys[i];
            j = leaf_of(r, k);
            const uint32_t P = leaf_predict(leaves[j], k);
            e = P > (uint32_t)i ? P - (uint32_t)i : (uint32_t)i - P;
        }
        const uint32_t peers = __match_any_sync(0xffffffffu, j);
        const uint32_t m = __reduce_max_sync(peers, e);
        if (valid && (threadIdx.x & 31) == (uint32_t)(__ffs(peers) - 1) && m) atomicMax(&leaves[j].err, m);
    }
}

__global__ void k_leaf_stats(const LearnedLeaf* __restrict__ leaves, LearnedRoot* rt) {
    __shared__ unsigned long long s_sum[32];
    __shared__ uint32_t s_max[32], s_ne[32];
    unsigned long long sum = 0;
    uint32_t mx = 0, ne = 0;
    for (uint32_t j = threadIdx.x; j < kLeaves; j += blockDim.x) {
        const LearnedLeaf lf = leaves[j];
        if (lf.r1 > lf.r0) {
            sum += lf.err;
            mx = max(mx, lf.err);
            ++ne;
        }
    }
    for (int o = 16; o; o >>= 1) {
        sum += __shfl_down_sync(0xffffffffu, sum, o);
        mx = max(mx, __shfl_down_sync(0xffffffffu, mx, o));
        ne += __shfl_down_sync(0xffffffffu, ne, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        s_sum[w] = sum;
        s_max[w] = mx;
        s_ne[w] = ne;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
            sum += s_sum[k];
            mx = max(mx, s_max[k]);
            ne += s_ne[k];
        }
        rt->sum_err = sum;
        rt->max_err = mx;
        rt->nonempty = ne;
        rt->checked = 0;
        rt->mismatches = 0;
    }
}

// The judge: corrected model rank of every level-L cell boundary vs the table.
__global__ void k_judge(const LearnedLeaf* __restrict__ leaves, LearnedRoot* rt, const uint32_t* __restrict__ wpref,
                        const uint32_t* __restrict__ table, uint64_t ncells, int key_shift) {
    const LearnedRoot r = *rt;
    unsigned long long bad = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += stride) {
        const uint32_t t = learned_rank(r, leaves, wpref, (unsigned long long)c << key_shift);
        bad += (t != table[c]) ? 1ull : 0ull;
    }
    for (int o = 16; o; o >>= 1) bad += __shfl_down_sync(0xffffffffu, bad, o);
    if ((threadIdx.x & 31) == 0 && bad) atomicAdd(&rt->mismatches, bad);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&rt->checked, (unsigned long long)ncells);
}

}  // namespace

int morton_auto_level(uint64_t n, float radius_hint) {
    // about 4 or more particles per cell on average ...
    int L = 1;
    while (L < 9 && (1ull << (3 * (L + 1))) * 4ull <= n) ++L;
    // ... and cells no smaller than 0.7 R, so a query box spans <= 4 cells per axis
    if (radius_hint > 0.0f)
        while (L > 1 && 1000.0 / (double)(1u << L) < 0.7 * (double)radius_hint) --L;
    return L;
}

int build_morton_index(sjcs_ctx* ctx, const float* d_xyz, uint64_t n, int level, bool learned, bool verify,
                       sjcs_index* idx, cudaStream_t s) {
    (void)ctx;
    idx->level = level;
    idx->verify = learned && verify;
    for (int a = 0; a < 3; ++a) {
        idx->geom.G[a] = 1 << level;
        idx->geom.inv_h[a] = (float)(1 << level) / 1000.0f;
    }
    const uint64_t ncells = 1ull << (3 * level);
    idx->geom.ncells = ncells;
    const uint64_t nalloc = n ? n : 1;
    SJCS_CUDA_TRY(cudaMallocAsync(&idx->pts, nalloc * sizeof(float4), s));
    SJCS_CUDA_TRY(cudaMallocAsync(&idx->cell_start, (ncells + 1) * sizeof(uint32_t), s));
    if (learned) {
        SJCS_CUDA_TRY(cudaMallocAsync(&idx->leaves, kLeaves * sizeof(LearnedLeaf), s));
        SJCS_CUDA_TRY(cudaMallocAsync(&idx->root, sizeof(LearnedRoot), s));
        SJCS_CUDA_TRY(cudaMemsetAsync(idx->root, 0, sizeof(LearnedRoot), s));
        SJCS_CUDA_TRY(cudaMemsetAsync(idx->leaves, 0, kLeaves * sizeof(LearnedLeaf), s));
    }
    if (n == 0) {
        SJCS_CUDA_TRY(cudaMemsetAsync(idx->cell_start, 0, (ncells + 1) * sizeof(uint32_t), s));
        cudaEventRecord(idx->ev_train0, s);
        return SJCS_OK;
    }

    const uint32_t ntiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
    StreamScratch scr(s);
    uint32_t *kx, *ky, *hist, *partials, *cells, *ngaps, *first = nullptr;
    uint4 *px, *py;
    unsigned long long* keys = nullptr;
    void* gaps;
    SJCS_CUDA_TRY(scr.alloc(&kx, n * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&ky, n * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&px, n * sizeof(uint4)));
    SJCS_CUDA_TRY(scr.alloc(&py, n * sizeof(uint4)));
    SJCS_CUDA_TRY(scr.alloc(&cells, n * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&hist, (uint64_t)RS_BINS * ntiles * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&partials, scan_partials_needed((uint64_t)RS_BINS * ntiles) * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&gaps, (size_t)kGridGaps * 12));
    SJCS_CUDA_TRY(scr.alloc(&ngaps, sizeof(uint32_t)));
    if (learned) {
        SJCS_CUDA_TRY(scr.alloc(&keys, n * sizeof(unsigned long long)));
        SJCS_CUDA_TRY(scr.alloc(&first, (kLeaves + 1) * sizeof(uint32_t)));
    }

    // passes 0-3: low half (A = x buffers after even passes, B = y after odd)
    int rc = radix_pass(MortonLoKey{d_xyz}, MortonPay{d_xyz}, SinkRecords{kx, px}, n, 0, hist, ntiles, s, partials);
    for (int p = 1; p < 4 && !rc; ++p) {
        const bool to_x = (p % 2) == 0;
        rc = radix_pass(KeysFromArray{to_x ? ky : kx}, PayFromArray{to_x ? py : px},
                        SinkRecords{to_x ? kx : ky, to_x ? px : py}, n, 8 * p, hist, ntiles, s, partials);
    }
    // pass 4: key = high half from the payload, payload carries the low half
    if (!rc)
        rc = radix_pass(KeyFromPayW{py}, PaySwapKey{ky, py}, SinkRecords{kx, px}, n, 0, hist, ntiles, s, partials);
    for (int p = 5; p < 7 && !rc; ++p) {
        const bool to_x = (p % 2) == 0;
        rc = radix_pass(KeysFromArray{to_x ? ky : kx}, PayFromArray{to_x ? py : px},
                        SinkRecords{to_x ? kx : ky, to_x ? px : py}, n, 8 * (p - 4), hist, ntiles, s, partials);
    }
    if (!rc)
        rc = radix_pass(KeysFromArray{kx}, PayFromArray{px},
                        SinkMorton{reinterpret_cast<uint4*>(idx->pts), cells, keys, 31 - 3 * level}, n, 24, hist,
                        ntiles, s, partials);
    if (rc) return rc;
    rc = fill_cell_table(cells, n, ncells, idx->cell_start, gaps, ngaps, s);
    if (rc) return rc;
    cudaEventRecord(idx->ev_train0, s);
    if (!learned) return SJCS_OK;

    k_root<<<1, 1, 0, s>>>(keys, n, idx->root);
    SJCS_LAUNCH_CHECK();
    k_leaf_bounds<<<(unsigned)((n + 1 + 255) / 256), 256, 0, s>>>(keys, n, idx->root, first);
    SJCS_LAUNCH_CHECK();
    k_leaf_fit<<<kLeaves / 256, 256, 0, s>>>(keys, first, idx->leaves);
    SJCS_LAUNCH_CHECK();
    const unsigned eblocks = (unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
    k_leaf_err<<<eblocks, 256, 0, s>>>(keys, n, idx->root, idx->leaves);
    SJCS_LAUNCH_CHECK();
    k_leaf_stats<<<1, 1024, 0, s>>>(idx->leaves, idx->root);
    SJCS_LAUNCH_CHECK();
    if (verify) {
        const unsigned jblocks = (unsigned)std::min<uint64_t>((ncells + 255) / 256, 148ull * 16);
        k_judge<<<jblocks, 256, 0, s>>>(idx->leaves, idx->root, reinterpret_cast<const uint32_t*>(idx->pts) + 3,
                                        idx->cell_start, ncells + 1, 63 - 3 * level);
        SJCS_LAUNCH_CHECK();
    }
    return SJCS_OK;
}

}  // namespace sjcs
