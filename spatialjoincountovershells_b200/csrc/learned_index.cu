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
//   train    (learned kind) equal-population leaf rank ranges, a fitted
//            fp32 slope and bias per leaf and its exact max error, the
//            root's directory over the leaves' anchors
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
    while (((r.kmax - r.kmin) >> sh) >= (1ull << kDirBits)) ++sh;
    r.shift = sh;
    r.n = (uint32_t)n;
    *rt = r;
}

// first[j] = first rank of leaf j: the first occurrence of the key at rank
// j*n/4096 (first[4096] = n), so every leaf holds about n/4096 keys and
// equal keys share a leaf.
__global__ void k_leaf_first(const unsigned long long* __restrict__ keys, uint64_t n, uint32_t* __restrict__ first) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j > kLeaves) return;
    const uint64_t r = (uint64_t)j * n / kLeaves;
    if (r >= n) {
        first[j] = (uint32_t)n;
        return;
    }
    const unsigned long long k = keys[r];
    uint64_t lo = 0, hi = r;  // lower bound of k in keys[0, r]
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (keys[mid] < k) lo = mid + 1;
        else hi = mid;
    }
    first[j] = (uint32_t)lo;
}

template <class T>
__device__ __forceinline__ T block_reduce(T v, T (*op)(T, T), T* sh) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o; o >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();  // sh is free (an earlier reduction may still be reading it)
    if (lane == 0) sh[w] = v;
    __syncthreads();
    v = sh[0];
    for (int k = 1; k < nw; ++k) v = op(v, sh[k]);
    return v;
}
__device__ double dadd(double a, double b) { return a + b; }
__device__ double dmin(double a, double b) { return fmin(a, b); }
__device__ double dmax(double a, double b) { return fmax(a, b); }
__device__ uint32_t umax(uint32_t a, uint32_t b) { return max(a, b); }

// One block per leaf: least-squares slope of rank over key offset (double),
// the bias that centres the extreme residuals of the fp32 prediction, and
// the exact error bound of the final fp32 predictor.
__global__ void __launch_bounds__(256) k_leaf_fit(const unsigned long long* __restrict__ keys, uint64_t n,
                                                  const uint32_t* __restrict__ first,
                                                  LearnedLeaf* __restrict__ leaves) {
    __shared__ double shd[8];
    __shared__ uint32_t shu[8];
    const uint32_t j = blockIdx.x;
    LearnedLeaf lf{};
    lf.r0 = first[j];
    lf.r1 = first[j + 1];
    lf.anchor = lf.r0 < n ? keys[lf.r0] : ~0ull;
    const uint32_t m = lf.r1 - lf.r0;
    if (m >= 2) {
        double sx = 0, sy = 0, sxx = 0, sxy = 0;
        for (uint32_t i = lf.r0 + threadIdx.x; i < lf.r1; i += blockDim.x) {
            const double x = (double)(keys[i] - lf.anchor), y = (double)(i - lf.r0);
            sx += x;
            sy += y;
            sxx += x * x;
            sxy += x * y;
        }
        sx = block_reduce(sx, dadd, shd);
        sy = block_reduce(sy, dadd, shd);
        sxx = block_reduce(sxx, dadd, shd);
        sxy = block_reduce(sxy, dadd, shd);
        const double var = sxx - sx * sx / m, cov = sxy - sx * sy / m;
        double b = var > 0 ? cov / var : 0.0;
        if (!(b >= 0) || !isfinite(b)) b = 0.0;
        lf.slope = (float)b;
        double lo = 1e300, hi = -1e300;
        for (uint32_t i = lf.r0 + threadIdx.x; i < lf.r1; i += blockDim.x) {
            const float x = __ull2float_rn(keys[i] - lf.anchor);
            const double d = (double)(i - lf.r0) - (double)__fmul_rn(x, lf.slope);
            lo = fmin(lo, d);
            hi = fmax(hi, d);
        }
        lo = block_reduce(lo, dmin, shd);
        hi = block_reduce(hi, dmax, shd);
        lf.bias = (float)(0.5 * (lo + hi) + 0.5);  // + 0.5: truncation then rounds to nearest
        uint32_t e = 0;
        for (uint32_t i = lf.r0 + threadIdx.x; i < lf.r1; i += blockDim.x) {
            const uint32_t P = leaf_predict(lf, keys[i]);
            e = max(e, P > i ? P - i : i - P);
        }
        lf.err = block_reduce(e, umax, shu);
    }
    if (threadIdx.x == 0) leaves[j] = lf;
}

// dir[b] = number of leaves whose anchor is <= kmin + (b << shift), b <= 2^16.
__global__ void k_leaf_dir(const LearnedLeaf* __restrict__ leaves, const LearnedRoot* __restrict__ rt,
                           uint16_t* __restrict__ dir) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= kDirEntries) return;
    const LearnedRoot r = *rt;
    // kmax - kmin < 2^63 keeps shift <= 47, so b << shift (b <= 2^16) fits
    const uint64_t off = (uint64_t)b << r.shift;
    const unsigned long long q = off > r.kmax - r.kmin ? ~0ull : r.kmin + off;
    uint32_t lo = 0, hi = kLeaves;  // upper bound of q among the anchors
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (leaves[mid].anchor <= q) lo = mid + 1;
        else hi = mid;
    }
    dir[b] = (uint16_t)min(lo, (uint32_t)kLeaves);
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
        SJCS_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&idx->leaves), kModelBytes, s));
        SJCS_CUDA_TRY(cudaMallocAsync(&idx->root, sizeof(LearnedRoot), s));
        SJCS_CUDA_TRY(cudaMemsetAsync(idx->root, 0, sizeof(LearnedRoot), s));
        SJCS_CUDA_TRY(cudaMemsetAsync(idx->leaves, 0, kModelBytes, s));
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
    k_leaf_first<<<(kLeaves + 1 + 255) / 256, 256, 0, s>>>(keys, n, first);
    SJCS_LAUNCH_CHECK();
    k_leaf_fit<<<kLeaves, 256, 0, s>>>(keys, n, first, idx->leaves);
    SJCS_LAUNCH_CHECK();
    k_leaf_dir<<<(kDirEntries + 255) / 256, 256, 0, s>>>(idx->leaves, idx->root,
                                                          reinterpret_cast<uint16_t*>(idx->leaves + kLeaves));
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
