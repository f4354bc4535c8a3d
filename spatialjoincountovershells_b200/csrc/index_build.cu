// Plain (grid) index build for one particle file.
//
// Replaces the STR bulk load of the reference (MakeTreeWithSameThreadPoolArraySTR,
// src/objects/ArraySTR/Build.c:845-963: per level, LSD radix sorts on the
// y, x, z centres, gather, pack 10 children per parent MBR).  The counts the
// reference produces do not depend on the tree shape -- a leaf is reached iff
// its point lies inside the query box, because every parent MBR is the exact
// hull of its children (adjustMbrArraySTRNode, src/objects/ArraySTR/Node.c:10-58)
// -- so any index that returns a superset of the in-box points gives the same
// counts.  Here the index is a uniform cell grid:
//   pass 0   key = cell of (x,y,z) and payload = (x,y,z), read from the AoS input
//            (staged in shared memory a tile at a time when 16-byte aligned)
//   passes   stable LSD radix sort of (key, payload), 8 bits per pass (9 for
//            25-27-bit cell keys: three passes instead of four)
//   last     writes the sorted particles as float4 and the sorted keys
//   offsets  cell_start[c] = first sorted slot of cell c (boundary fill)
#include <algorithm>
#include <cmath>

#include "radix_sort.cuh"
#include "sjcs_internal.cuh"

namespace sjcs {
namespace {

struct KeysFromParticles {
    const float* __restrict__ xyz;
    GridGeom g;
    __device__ __forceinline__ uint32_t key_of(float x, float y, float z) const { return cell_key(g, x, y, z); }
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const {
        return key_of(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    }
};
struct PayFromParticles {
    const float* __restrict__ xyz;
    __device__ __forceinline__ uint4 operator()(uint64_t i) const {
        return make_uint4(__float_as_uint(xyz[3 * i]), __float_as_uint(xyz[3 * i + 1]),
                          __float_as_uint(xyz[3 * i + 2]), 0u);
    }
};
// Last pass: sorted key (for the offsets) and the particle as float4.
struct SinkParticles {
    uint32_t* __restrict__ keys;
    uint4* __restrict__ pts;
    __device__ __forceinline__ void operator()(uint32_t g, uint32_t k, const uint4& v) const {
        keys[g] = k;
        pts[g] = v;
    }
};

struct Gap {
    uint32_t lo, hi, val;  // cells [lo, hi] start at slot val
};
constexpr uint32_t kGapInline = 64;

// cell_start[c] = i for every cell c in [lo, hi] (lo > hi: nothing); runs
// longer than kGapInline go to the gap list.
__device__ __forceinline__ void fill_cells(uint64_t lo, uint64_t hi, uint32_t i, uint32_t* __restrict__ cs,
                                           Gap* __restrict__ gaps, uint32_t* __restrict__ ngaps,
                                           uint32_t max_gaps) {
    if (lo > hi) return;
    const uint64_t cnt = hi - lo + 1;
    const uint64_t inl = cnt < kGapInline ? cnt : kGapInline;
    for (uint64_t c = 0; c < inl; ++c) cs[lo + c] = i;
    if (cnt > kGapInline) {
        const uint32_t slot = atomicAdd(ngaps, 1u);
        if (slot < max_gaps) {
            gaps[slot] = Gap{(uint32_t)(lo + kGapInline), (uint32_t)hi, i};
        } else {
            for (uint64_t c = lo + kGapInline; c <= hi; ++c) cs[c] = i;
        }
    }
}

// cell_start[c] = i for every cell c in (key[i-1], key[i]] (key[-1] = -1,
// key[n] = ncells), so empty cells point at the next occupied slot and
// cell_start[ncells] = n.  Thread t takes boundaries i = 4t .. 4t+3, reading
// their keys with one 16-byte load when the key array is 16-byte aligned.
// Long runs of empty cells go to a gap list that a second kernel fills
// cooperatively.
__global__ void k_cell_start(const uint32_t* __restrict__ keys, uint64_t n, uint64_t ncells,
                             uint32_t* __restrict__ cs, Gap* __restrict__ gaps,
                             uint32_t* __restrict__ ngaps, uint32_t max_gaps, int vec) {
    const uint64_t i0 = 4 * ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x);
    if (i0 > n) return;
    uint64_t cur[4];
    if (vec && i0 + 4 <= n) {
        const uint4 v = *reinterpret_cast<const uint4*>(keys + i0);
        cur[0] = v.x;
        cur[1] = v.y;
        cur[2] = v.z;
        cur[3] = v.w;
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) cur[j] = (i0 + j < n) ? (uint64_t)keys[i0 + j] : ncells;
    }
    uint64_t lo = (i0 == 0) ? 0ull : (uint64_t)keys[i0 - 1] + 1ull;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const uint64_t i = i0 + (uint64_t)j;
        if (i > n) break;
        fill_cells(lo, cur[j], (uint32_t)i, cs, gaps, ngaps, max_gaps);
        lo = cur[j] + 1ull;
    }
}

__global__ void k_fill_gaps(const Gap* __restrict__ gaps, const uint32_t* __restrict__ ngaps,
                            uint32_t max_gaps, uint32_t* __restrict__ cs) {
    const uint32_t ng = min(*ngaps, max_gaps);
    for (uint32_t gi = blockIdx.x; gi < ng; gi += gridDim.x) {
        const Gap gp = gaps[gi];
        for (uint64_t c = (uint64_t)gp.lo + threadIdx.x; c <= gp.hi; c += blockDim.x) cs[c] = gp.val;
    }
}

}  // namespace

GridGeom auto_grid(uint64_t n, float radius_hint, const uint32_t* grid_req) {
    GridGeom g{};
    int G[3];
    if (grid_req && grid_req[0] && grid_req[1] && grid_req[2]) {
        for (int a = 0; a < 3; ++a) G[a] = (int)grid_req[a];
    } else {
        // Rows of cells run along x and are looked up with two offsets, so x
        // can be finer than y/z for free: cells are 2.5x longer in y and z.
        // Target about 1.6 cells per particle, at most 2^27 cells (a 27-bit
        // cell key sorts in three 9-bit radix passes), and keep y/z cells
        // >= R/4: a query box then spans at most 9x9 rows (boxes of more
        // than 25 rows are counted without the per-batch row plan).
        constexpr double kMaxCells = 134217728.0;  // 2^27
        const double target = std::min(std::max(1.6 * (double)n, 4096.0), kMaxCells);
        double hyz = std::cbrt(2.5e9 / target);
        if (radius_hint > 0.0f) hyz = std::max(hyz, 0.25 * (double)radius_hint);
        for (;;) {
            const double hx = hyz / 2.5;
            G[0] = (int)std::min(std::max(std::ceil(1000.0 / hx), 1.0), 4096.0);
            G[1] = (int)std::min(std::max(std::ceil(1000.0 / hyz), 1.0), 4096.0);
            G[2] = G[1];
            if ((double)G[0] * G[1] * G[2] <= kMaxCells) break;
            hyz *= 1.002;  // rounding up per axis overshot the cap
        }
    }
    for (int a = 0; a < 3; ++a) {
        g.G[a] = G[a];
        g.inv_h[a] = (float)G[a] / 1000.0f;
    }
    g.ncells = (uint64_t)G[0] * G[1] * G[2];
    return g;
}

int grid_key_bits(const GridGeom& g) {
    int key_bits = 1;
    while (key_bits < 32 && (1ull << key_bits) < g.ncells) ++key_bits;
    return key_bits;
}

int grid_digit_bits(const GridGeom& g) {
    const int kb = grid_key_bits(g);
    return (kb > 24 && kb <= 27) ? 9 : 8;  // three passes instead of four
}

template <int BITS, class PayOp0>
int sort_particles(const float* d_xyz, uint64_t n, const GridGeom& g, const GridBuildBuffers& b, PayOp0 pop0,
                   cudaStream_t s) {
    return radix_sort_records<BITS>(n, grid_key_bits(g), KeysFromParticles{d_xyz, g}, pop0,
                                    SinkParticles{b.kfinal, reinterpret_cast<uint4*>(b.pts)}, b.kx, b.px, b.ky,
                                    b.py, b.hist, s, b.partials);
}

int build_grid_into(const float* d_xyz, uint64_t n, const GridGeom& g, const GridBuildBuffers& b, cudaStream_t s) {
    static_assert(sizeof(Gap) == 12, "gap records are 12 bytes");
    // A 16-byte-aligned particle array is staged tile by tile in the first
    // pass; any other alignment is read particle by particle.
    const bool staged = (reinterpret_cast<uintptr_t>(d_xyz) & 15u) == 0;
    int rc;
    if (b.digit_bits == 9)
        rc = staged ? sort_particles<9>(d_xyz, n, g, b, PayFromXyzStaged{d_xyz}, s)
                    : sort_particles<9>(d_xyz, n, g, b, PayFromParticles{d_xyz}, s);
    else
        rc = staged ? sort_particles<8>(d_xyz, n, g, b, PayFromXyzStaged{d_xyz}, s)
                    : sort_particles<8>(d_xyz, n, g, b, PayFromParticles{d_xyz}, s);
    if (rc) return rc;
    return fill_cell_table(b.kfinal, n, g.ncells, b.cell_start, b.gaps, b.ngaps, s);
}

int fill_cell_table(const uint32_t* sorted_cells, uint64_t n, uint64_t ncells, uint32_t* cell_start, void* gaps,
                    uint32_t* ngaps, cudaStream_t s) {
    SJCS_CUDA_TRY(cudaMemsetAsync(ngaps, 0, sizeof(uint32_t), s));
    const uint64_t threads = n / 4 + 1;  // boundaries 0..n, four per thread
    const unsigned blocks = (unsigned)((threads + 255) / 256);
    const int vec = (reinterpret_cast<uintptr_t>(sorted_cells) & 15u) == 0;
    k_cell_start<<<blocks, 256, 0, s>>>(sorted_cells, n, ncells, cell_start, static_cast<Gap*>(gaps), ngaps,
                                        kGridGaps, vec);
    SJCS_LAUNCH_CHECK();
    k_fill_gaps<<<1024, 256, 0, s>>>(static_cast<Gap*>(gaps), ngaps, kGridGaps, cell_start);
    SJCS_LAUNCH_CHECK();
    return SJCS_OK;
}

int build_grid_index(sjcs_ctx* ctx, const float* d_xyz, uint64_t n, const GridGeom& g,
                     sjcs_index* idx, cudaStream_t s) {
    (void)ctx;
    idx->geom = g;
    const uint64_t nalloc = n ? n : 1;
    SJCS_CUDA_TRY(cudaMallocAsync(&idx->pts, nalloc * sizeof(float4), s));
    SJCS_CUDA_TRY(cudaMallocAsync(&idx->cell_start, (g.ncells + 1) * sizeof(uint32_t), s));

    GridBuildBuffers b{};
    b.pts = idx->pts;
    b.cell_start = idx->cell_start;
    const uint64_t ntiles = (n + RS_TILE - 1) / RS_TILE;
    b.digit_bits = grid_digit_bits(g);
    const int passes = (grid_key_bits(g) + b.digit_bits - 1) / b.digit_bits;
    StreamScratch scr(s);  // freed (stream-ordered) on every return path
    SJCS_CUDA_TRY(scr.alloc(&b.kfinal, nalloc * sizeof(uint32_t)));
    if (passes > 1) {
        SJCS_CUDA_TRY(scr.alloc(&b.kx, nalloc * sizeof(uint32_t)));
        SJCS_CUDA_TRY(scr.alloc(&b.px, nalloc * sizeof(uint4)));
    }
    if (passes > 2) {
        SJCS_CUDA_TRY(scr.alloc(&b.ky, nalloc * sizeof(uint32_t)));
        SJCS_CUDA_TRY(scr.alloc(&b.py, nalloc * sizeof(uint4)));
    }
    SJCS_CUDA_TRY(scr.alloc(&b.hist, ((uint64_t)(1u << b.digit_bits) * (ntiles ? ntiles : 1)) * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&b.gaps, kGridGaps * sizeof(Gap)));
    SJCS_CUDA_TRY(scr.alloc(&b.ngaps, sizeof(uint32_t)));
    return build_grid_into(d_xyz, n, g, b, s);
}

}  // namespace sjcs
