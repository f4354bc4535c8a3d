// Morton-ordered index: key layout, the two-level piecewise-linear rank model
// and its exact corrected lookup.  Shared by the build (learned_index.cu) and
// the count kernel (morton_count.cu).
//
// Key: 21 bits per axis, q = clamp(floor(v * 2^21/1000), 0, 2^21 - 1) (the
// same monotone cell function as the grid, so NaN -> 0 and out-of-box values
// clamp into the edge cells), interleaved x-lowest into a 63-bit code.  The
// level-L cell of a particle is the key's top 3L bits (L <= 21); cells of one
// level are contiguous key ranges, so a level-L cell is the slot range
// [lower_bound(c << (63-3L)), lower_bound((c+1) << (63-3L))).
//
// HBM layout of a Morton index over n particles:
//   pts[n]              float4 (x, y, z, level-10 prefix bits), sorted by key
//   table[8^L + 1]      u32 plain offset table of the index's cell level L
//   leaves[4096]        LearnedLeaf, then the root's directory (2^16 + 1 u16),
//   root                one LearnedRoot                         (learned kind)
//
// Rank model (learned kind), in the manner of a radix spline: 4096 leaves of
// equal population -- leaf j holds the ranks [r0_j, r1_j) with r0_j the first
// rank of the key at rank j*n/4096 (so equal keys never straddle two leaves)
// and covers the keys [anchor_j, anchor_{j+1}), anchor_j = key[r0_j].  The
// root finds a key's leaf: a 2^16-entry directory over (key - kmin) >> shift
// gives the few leaves whose anchors can precede the key, and a short binary
// search over those anchors picks the last one <= key.  Leaf j predicts
//     P(q) = r0 + min(trunc(clamp(fp32(fp32(q - anchor) * slope) + bias)), r1 - r0),
// slope and bias fitted to the leaf's keys (least squares, then the bias
// centred on the extreme residuals); P is monotone in q.  Training records
// err = max over the leaf's keys k_i of |P(k_i) - i|.  For a query key q in
// leaf j the true lower bound t satisfies
//     t < r1  =>  P(q) <= P(k_t) <= t + err
//     t > r0  =>  t - 1 - err <= P(k_{t-1}) <= P(q)
// so t lies in [max(r0, P - err), min(r1, P + err + 1)], and a binary search
// over that window (the bounded exact correction) returns t exactly.
#pragma once

#include "sjcs_internal.cuh"

namespace sjcs {

constexpr int kMortonBits = 21;
constexpr float kMortonScale = 2097.152f;  // 2^21 / 1000
constexpr int kLeafBits = 12;
constexpr uint32_t kLeaves = 1u << kLeafBits;  // 4096 leaves
constexpr int kPrefixLevel = 10;               // pts[i].w holds the key's top 30 bits
constexpr int kMaxMortonLevel = 10;

constexpr int kDirBits = 16;
constexpr uint32_t kDirEntries = (1u << kDirBits) + 1u;

struct LearnedLeaf {
    unsigned long long anchor;  // first key of the leaf (~0 for an empty leaf at the end)
    uint32_t r0, r1;            // exact rank range of the leaf's keys
    float slope;                // ranks per key unit
    float bias;                 // ranks added before truncation
    uint32_t err;               // max |P(k_i) - i| over the leaf's keys
    uint32_t pad_;
};
static_assert(sizeof(LearnedLeaf) == 32, "leaf records are 32 bytes");
// bytes of the leaves and the root's directory (one allocation)
constexpr size_t kModelBytes = kLeaves * sizeof(LearnedLeaf) + kDirEntries * sizeof(uint16_t);

struct LearnedRoot {
    unsigned long long kmin, kmax;
    uint32_t shift;  // directory bucket of a key: (key - kmin) >> shift (< 2^16)
    uint32_t n;
    unsigned long long checked;     // cell boundaries compared with the table
    unsigned long long mismatches;  // lookups that disagreed (then the table is used)
    unsigned long long sum_err;     // sum of the leaves' err (non-empty leaves)
    uint32_t max_err;
    uint32_t nonempty;
};

__device__ __forceinline__ uint64_t spread3_21(uint32_t v) {
    uint64_t x = v & 0x1fffffu;
    x = (x | (x << 32)) & 0x001f00000000ffffull;
    x = (x | (x << 16)) & 0x001f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

__device__ __forceinline__ uint32_t morton_q(float v) { return (uint32_t)cell_of(v, kMortonScale, 1 << kMortonBits); }

__device__ __forceinline__ uint64_t morton63(float x, float y, float z) {
    return spread3_21(morton_q(x)) | (spread3_21(morton_q(y)) << 1) | (spread3_21(morton_q(z)) << 2);
}

// Code of cell (x, y, z) at a level <= 10 (30 bits).
__device__ __forceinline__ uint32_t morton_cell(uint32_t x, uint32_t y, uint32_t z) {
    return spread3_10(x) | (spread3_10(y) << 1) | (spread3_10(z) << 2);
}

__device__ __forceinline__ const uint16_t* model_dir(const LearnedLeaf* leaves) {
    return reinterpret_cast<const uint16_t*>(leaves + kLeaves);
}

// Leaf of a key in [kmin, kmax]: the last leaf whose anchor is <= key.
__device__ __forceinline__ uint32_t leaf_of(const LearnedRoot& rt, const LearnedLeaf* __restrict__ leaves,
                                            uint64_t key) {
    const uint16_t* dir = model_dir(leaves);
    const uint32_t b = (uint32_t)((key - rt.kmin) >> rt.shift);
    uint32_t lo = __ldg(dir + b), hi = __ldg(dir + b + 1);  // counts of anchors <= the bucket's ends
    lo = lo ? lo - 1u : 0u;
    hi = hi ? hi - 1u : 0u;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1u) >> 1;
        if (__ldg(&leaves[mid].anchor) <= key) lo = mid;
        else hi = mid - 1u;
    }
    return lo;
}

__device__ __forceinline__ uint32_t leaf_predict(const LearnedLeaf& lf, uint64_t q) {
    const float x = __ull2float_rn(q - lf.anchor);  // q >= anchor
    const float off = fminf(fmaxf(__fadd_rn(__fmul_rn(x, lf.slope), lf.bias), 0.0f), 4.0e9f);
    const uint32_t d = (uint32_t)off;  // off >= 0: truncation is floor
    const uint32_t span = lf.r1 - lf.r0;
    return lf.r0 + (d < span ? d : span);
}

// Exact lower bound of q (a cell boundary: q's low 33 bits are zero) among
// the sorted keys, from the model and a bounded binary search over the
// level-10 prefixes in pts[].w.
__device__ __forceinline__ uint32_t learned_rank(const LearnedRoot& rt, const LearnedLeaf* __restrict__ leaves,
                                                 const uint32_t* __restrict__ wpref, uint64_t q) {
    if (q <= rt.kmin) return 0u;
    if (q > rt.kmax) return rt.n;
    const LearnedLeaf lf = leaves[leaf_of(rt, leaves, q)];
    const uint32_t P = leaf_predict(lf, q);
    uint32_t lo = (P - lf.r0 > lf.err) ? P - lf.err : lf.r0;
    const uint64_t hi64 = (uint64_t)P + lf.err + 1ull;
    uint32_t hi = hi64 < (uint64_t)lf.r1 ? (uint32_t)hi64 : lf.r1;
    const uint32_t qp = (uint32_t)(q >> 33);
    while (lo < hi) {
        const uint32_t mid = lo + ((hi - lo) >> 1);
        if (__ldg(wpref + 4ull * mid) < qp) lo = mid + 1u;
        else hi = mid;
    }
    return lo;
}

// N exact lower bounds at once (as learned_rank), the N bounded binary
// searches advanced together so their probes are independent loads in flight
// at the same time.  act[j] == false: out[j] = 0 and no memory is read.
template <int N>
__device__ __forceinline__ void learned_rank_n(const LearnedRoot& rt, const LearnedLeaf* __restrict__ leaves,
                                               const uint32_t* __restrict__ wpref, const uint64_t (&q)[N],
                                               const bool (&act)[N], uint32_t (&out)[N]) {
    uint32_t lo[N], hi[N], qp[N];
#pragma unroll
    for (int j = 0; j < N; ++j) {
        lo[j] = 0u;
        hi[j] = 0u;
        qp[j] = (uint32_t)(q[j] >> 33);
        if (!act[j]) continue;
        if (q[j] <= rt.kmin) continue;  // rank 0
        if (q[j] > rt.kmax) {
            lo[j] = hi[j] = rt.n;
            continue;
        }
        const LearnedLeaf lf = leaves[leaf_of(rt, leaves, q[j])];
        const uint32_t P = leaf_predict(lf, q[j]);
        lo[j] = (P - lf.r0 > lf.err) ? P - lf.err : lf.r0;
        const uint64_t h64 = (uint64_t)P + lf.err + 1ull;
        hi[j] = h64 < (uint64_t)lf.r1 ? (uint32_t)h64 : lf.r1;
    }
    for (;;) {
        bool any = false;
#pragma unroll
        for (int j = 0; j < N; ++j) any |= lo[j] < hi[j];
        if (!any) break;
        uint32_t v[N], mid[N];
#pragma unroll
        for (int j = 0; j < N; ++j) {
            mid[j] = lo[j] + ((hi[j] - lo[j]) >> 1);
            v[j] = lo[j] < hi[j] ? __ldg(wpref + 4ull * mid[j]) : 0u;
        }
#pragma unroll
        for (int j = 0; j < N; ++j) {
            if (lo[j] < hi[j]) {
                if (v[j] < qp[j]) lo[j] = mid[j] + 1u;
                else hi[j] = mid[j];
            }
        }
    }
#pragma unroll
    for (int j = 0; j < N; ++j) out[j] = lo[j];
}

}  // namespace sjcs
