// Persistent work-queue schedule, shared by the grid and Morton count kernels.
//
// A count kernel's estimate kernel gives every halo (Morton order) a size
// bucket (est_bucket of its estimated candidates) and a histogram of the
// buckets; order_and_plan then
//   sorts    one 8-bit radix pass by descending bucket (stable: Morton order
//            within a bucket) -> ord[i] = Morton index
//   plans    k_plan_items, per bucket (lower bound e of its estimates): halos
//            with e >= piece are split into min(max_pieces, ceil(e/piece))
//            pieces that separate warps count (every candidate set split
//            evenly); halos with e >= single are items of their own; lighter
//            halos go min(32, piece/e) to an item.  The buckets' item counts
//            are prefix-summed into a 256-entry table.
// and persistent warps claim items with one atomicAdd each (claim_item: no
// claim ever fails or retries), largest buckets first, so the longest items
// start early and the light ones fill the tail.
#pragma once

#include "count_common.cuh"
#include "radix_sort.cuh"

namespace sjcs {
namespace {

struct BucketPlan {
    uint32_t start;   // first position of the bucket in ord
    uint32_t count;   // halos in the bucket
    uint32_t per;     // halos per item (batch) or 0 when halos are split
    uint32_t pieces;  // pieces per halo when split
    uint32_t item0;   // first item of the bucket
};
constexpr int kBuckets = 256;

struct QueueParams {
    const uint32_t* __restrict__ ord;     // Morton index, descending size buckets
    const BucketPlan* __restrict__ plan;  // [kBuckets] in position order (key 0 = largest)
    uint32_t* __restrict__ ctl;           // [0] item counter, [1] total items
};

__device__ __forceinline__ uint32_t bucket_low(uint32_t b) {
    if (b == 0) return 0u;
    const uint32_t lg = (b - 1u) >> 3, mant = (b - 1u) & 7u;
    return lg >= 3 ? (8u + mant) << (lg - 3) : (8u + mant) >> (3 - lg);
}

// One block of kBuckets threads: bucket starts, item sizes and item prefix.
__global__ void k_plan_items(const uint32_t* __restrict__ hist, uint32_t piece, uint32_t max_pieces,
                             uint32_t single, BucketPlan* __restrict__ plan, uint32_t* __restrict__ ctl) {
    __shared__ uint32_t s_cnt[kBuckets], s_items[kBuckets];
    const int k = threadIdx.x;  // position order: key k holds bucket 255 - k
    const uint32_t cnt = hist[k];
    const uint32_t lo = bucket_low(255u - (uint32_t)k);
    uint32_t per = 0, pieces = 1, items;
    if (lo >= piece) {
        pieces = min(max_pieces, (lo + piece - 1u) / piece);
        items = cnt * pieces;  // <= 2^32 for the sizes accepted (nhalos * max_pieces is checked on the host)
    } else {
        per = lo >= single ? 1u : min(32u, max(1u, piece / max(lo, 1u)));
        items = (cnt + per - 1u) / per;
    }
    s_cnt[k] = cnt;
    s_items[k] = items;
    __syncthreads();
    if (k == 0) {
        uint32_t pos = 0, it = 0;
        for (int j = 0; j < kBuckets; ++j) {
            const uint32_t c = s_cnt[j], n = s_items[j];
            s_cnt[j] = pos;
            s_items[j] = it;
            pos += c;
            it += n;
        }
        ctl[0] = 0;
        ctl[1] = it;
    }
    __syncthreads();
    plan[k] = BucketPlan{s_cnt[k], cnt, per, pieces, s_items[k]};
}

struct KeyFromEst {
    const uint32_t* __restrict__ key;
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const { return key[i]; }
};
struct PayIndex {
    __device__ __forceinline__ uint4 operator()(uint64_t i) const { return make_uint4((uint32_t)i, 0u, 0u, 0u); }
};
struct SinkOrd {
    uint32_t* __restrict__ ord;
    __device__ __forceinline__ void operator()(uint32_t g, uint32_t, const uint4& v) const { ord[g] = v.x; }
};

// Sort halos by descending size bucket and plan the queue's items.
inline int order_and_plan(uint64_t n, const uint32_t* key, const uint32_t* hist, const Schedule& sc, uint32_t* ord,
                          BucketPlan* plan, uint32_t* ctl, uint32_t* rhist, cudaStream_t s) {
    int rc = radix_sort_records(n, 8, KeyFromEst{key}, PayIndex{}, SinkOrd{ord}, nullptr, nullptr, nullptr, nullptr,
                                rhist, s);
    if (rc) return rc;
    k_plan_items<<<1, kBuckets, 0, s>>>(hist, sc.piece, sc.max_pieces, sc.single, plan, ctl);
    SJCS_LAUNCH_CHECK();
    return SJCS_OK;
}

// Claim the next item (lane 0 takes it, the warp learns it).  Returns false
// when the queue is empty; otherwise *bp is the item's bucket and *r its
// index inside the bucket.
__device__ __forceinline__ bool claim_item(const QueueParams& q, uint32_t nitems, int lane, int* bk, BucketPlan* bp,
                                           uint32_t* r) {
    uint32_t g = 0;
    if (lane == 0) g = atomicAdd(q.ctl, 1u);
    g = __shfl_sync(0xffffffffu, g, 0);
    if (g >= nitems) return false;
    while (*bk + 1 < kBuckets && __ldg(&q.plan[*bk + 1].item0) <= g) ++*bk;
    *bp = q.plan[*bk];
    *r = g - bp->item0;
    return true;
}

}  // namespace
}  // namespace sjcs
