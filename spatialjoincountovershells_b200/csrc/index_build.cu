// Plain (grid) index build for one particle file.
//
// Replaces the STR bulk load of the reference (MakeTreeWithSameThreadPoolArraySTR,
// src/objects/ArraySTR/Build.c:845-963: per level, LSD radix sorts on the
// y, x, z centres, gather, pack 10 children per parent MBR).  The counts the
// reference produces do not depend on the tree shape -- a leaf is reached iff
// its point lies inside the query box, because every parent MBR is the exact
// hull of its children (adjustMbrArraySTRNode, src/objects/ArraySTR/Node.c:10-58)
// -- so any index that returns a superset of the in-box points gives the same
// counts.  Here the index is a uniform cell grid.  Cell keys of up to 30 bits
// (every automatic grid) are built by the partition build further down; wider
// keys, and the fixed-buffer build, by a stable LSD radix sort:
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

// ---------------------------------------------------------------------------
// Partition build, for cell keys of at most 30 bits.
//
// The counts need each cell's particles together and the cells in key order;
// the order inside a cell is free (a count is a sum).  So the records are
// partitioned most significant digit first, without stable ranking: a block
// places each record of its tile with one shared-memory atomic and reserves
// room per digit with one global cursor atomic, and the last pass
// counting-sorts groups of 4096 cells in shared memory and writes their
// cell-table entries itself:
//   top     counts of the key's top digit (<= 9 bits) over x,y,z, in shared
//           memory; their prefix starts the top buckets
//   pass A  x,y,z -> (x, y, z, key) records by the top digit, and beside them
//           the next digit (16 bits per record)
//   mid     per tile of a top bucket: counts of the next digit in shared
//           memory, added to the segment counts (a segment is 2^sb cells,
//           sb = max(9, key bits - 18) <= 12); their prefix starts the segments
//   pass B  records by the next digit (<= 9 bits) inside each top bucket
//           (keys of more than sb + 9 bits; else the top digit is the segment)
//   cells   per group of 4096 cells (whole segments): cell counts, cell_start
//           of its cells, records written in cell order
// Records are 16 bytes with the cell key in .w, which the count kernel does
// not read.  (12-byte records, keys computed again in every pass, were
// measured slower: a record then leaves as three scattered 4-byte stores.)
constexpr int PB_THREADS = 512;
constexpr int PB_ITEMS = 8;
constexpr uint32_t PB_TILE = PB_THREADS * PB_ITEMS;  // records per block in a partition pass
constexpr int PB_MIN_SEG_BITS = 9;
constexpr int PB_GROUP_BITS = 12;
constexpr uint32_t PB_GROUP_CELLS = 1u << PB_GROUP_BITS;  // cells per block in the last pass
constexpr size_t PB_SMEM = (size_t)PB_TILE * sizeof(float4);  // exchange (pass A: staged x,y,z first)
constexpr size_t PB_STAGE_SMEM = (size_t)PB_TILE * 3 * sizeof(float);  // a tile's x,y,z
constexpr int PB_MAX_KEY_BITS = PB_GROUP_BITS + 18;  // segment + two digits of <= 9 bits

struct PbTile {
    uint32_t bucket, start, len;  // records [start, start + len) of top bucket `bucket`
};

// Exclusive scan over the block (PB_THREADS threads) of one value per thread;
// *total gets the sum.  ws holds PB_THREADS / 32 + 1 words; one call per kernel.
__device__ __forceinline__ uint32_t pb_block_scan(uint32_t v, uint32_t* ws, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) ws[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        constexpr int W = PB_THREADS / 32;
        const uint32_t w = lane < W ? ws[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < W) ws[lane] = wi - w;
        if (lane == W - 1) ws[W] = wi;
    }
    __syncthreads();
    *total = ws[PB_THREADS / 32];
    return incl - v + ws[warp];
}

__device__ __forceinline__ uint32_t pb_key(const float4& r) { return __float_as_uint(r.w); }

// top_hist[cell >> shift] += 1 for every particle (at most PB_THREADS bins,
// counted in shared memory first).  Block b takes tiles PB_TOP_TILES*b ..
// (one reduction per bin for all of them); each tile's x,y,z are staged in
// shared memory with coalesced 16-byte copies (cp.async when the array is
// 16-byte aligned) and the keys taken from there.
constexpr uint32_t PB_TOP_TILES = 4;
__global__ void __launch_bounds__(PB_THREADS)
k_pb_top_hist(const float* __restrict__ xyz, int aligned, uint64_t n, GridGeom g, int shift,
              uint32_t* __restrict__ top_hist) {
    __shared__ uint32_t sh[PB_THREADS];
    extern __shared__ float4 stage4[];
    float* sx = reinterpret_cast<float*>(stage4);
    const int tid = threadIdx.x;
    sh[tid] = 0u;
    for (uint32_t t = 0; t < PB_TOP_TILES; ++t) {
        const uint64_t start = ((uint64_t)blockIdx.x * PB_TOP_TILES + t) * PB_TILE;
        if (start >= n) break;  // uniform across the block
        const uint64_t rem = n - start;
        const uint32_t len = rem < PB_TILE ? (uint32_t)rem : PB_TILE;
        const float* src = xyz + 3 * start;
        const uint32_t words = 3u * len;
        uint32_t w0 = 0;
        __syncthreads();  // the previous tile's staged words have been read
        if (aligned) {
            const uint32_t chunks = words >> 2;
            for (uint32_t c = (uint32_t)tid; c < chunks; c += PB_THREADS) cp_async16(sx + 4 * c, src + 4 * c);
            w0 = chunks * 4u;
        }
        for (uint32_t w = w0 + (uint32_t)tid; w < words; w += PB_THREADS) sx[w] = src[w];
        cp_async_wait_all();
        __syncthreads();
#pragma unroll
        for (int i = 0; i < PB_ITEMS; ++i) {
            const uint32_t loc = (uint32_t)i * PB_THREADS + (uint32_t)tid;
            if (loc < len) atomicAdd(&sh[cell_key(g, sx[3 * loc], sx[3 * loc + 1], sx[3 * loc + 2]) >> shift], 1u);
        }
    }
    __syncthreads();
    const uint32_t c = sh[tid];
    if (c) atomicAdd(&top_hist[tid], c);
}

// Tiles of the middle pass: each top bucket's records [top_start[t],
// top_start[t+1]) cut into tiles of at most PB_TILE, so a tile never mixes
// buckets.  Every block computes the buckets' tile offsets (ntop <=
// PB_THREADS) and writes tiles blockIdx.x * PB_THREADS + threadIdx.x.
__global__ void __launch_bounds__(PB_THREADS)
k_pb_tiles(const uint32_t* __restrict__ top_start, uint32_t ntop, PbTile* __restrict__ tiles,
           uint32_t* __restrict__ ntiles) {
    __shared__ uint32_t ws[PB_THREADS / 32 + 1];
    __shared__ uint32_t tend[PB_THREADS];  // inclusive tile prefix: tiles of buckets <= t
    const uint32_t t = threadIdx.x;
    const uint32_t lo = t < ntop ? top_start[t] : 0u, hi = t < ntop ? top_start[t + 1] : 0u;
    const uint32_t nt = (hi - lo + PB_TILE - 1) / PB_TILE;
    uint32_t total;
    const uint32_t base = pb_block_scan(nt, ws, &total);
    tend[t] = base + nt;
    __syncthreads();
    if (blockIdx.x == 0 && t == 0) *ntiles = total;
    const uint32_t i = blockIdx.x * PB_THREADS + t;
    if (i >= total) return;
    // bucket of tile i: the first b with tend[b] > i (it has tiles)
    uint32_t b = 0;
#pragma unroll
    for (uint32_t step = PB_THREADS / 2; step > 0; step >>= 1)
        if (tend[b + step - 1] <= i) b += step;
    const uint32_t b_lo = top_start[b], b_len = top_start[b + 1] - b_lo;
    const uint32_t off = (i - (tend[b] - (b_len + PB_TILE - 1) / PB_TILE)) * PB_TILE;
    tiles[i] = PbTile{b, b_lo + off, min(PB_TILE, b_len - off)};
}

// Segment counts for the middle pass: block i counts the middle digits of
// tiles 8i .. 8i+7 (mid[] as written by pass A) in shared memory and adds
// them to seg_hist[(bucket << bits_mid) + digit] whenever the bucket changes
// and at the end -- a reduction per (bucket run, digit) rather than per
// record.
constexpr uint32_t PB_MID_TILES = 8;
__global__ void __launch_bounds__(PB_THREADS)
k_pb_mid_hist(const uint16_t* __restrict__ mid, const PbTile* __restrict__ tiles,
              const uint32_t* __restrict__ ntiles, int bits_mid, uint64_t nseg, uint32_t* __restrict__ seg_hist) {
    __shared__ uint32_t sh[PB_THREADS];
    const uint32_t nt = *ntiles, t0 = blockIdx.x * PB_MID_TILES;
    if (t0 >= nt) return;
    const uint32_t t1 = min(t0 + PB_MID_TILES, nt);
    // masked: a slot that pass A left unwritten (only if the input changed
    // after the histogram) cannot index out of range
    const uint32_t mask = (1u << bits_mid) - 1u;
    sh[threadIdx.x] = 0u;
    uint32_t bucket = tiles[t0].bucket;
    __syncthreads();
    for (uint32_t t = t0; t < t1; ++t) {
        const PbTile tl = tiles[t];
        if (tl.bucket != bucket) {  // uniform across the block
            __syncthreads();
            const uint32_t c = sh[threadIdx.x];
            const uint64_t sg = ((uint64_t)bucket << bits_mid) + threadIdx.x;
            if (c && sg < nseg) atomicAdd(&seg_hist[sg], c);
            sh[threadIdx.x] = 0u;
            bucket = tl.bucket;
            __syncthreads();
        }
        for (uint32_t j = threadIdx.x; j < tl.len; j += PB_THREADS) atomicAdd(&sh[mid[tl.start + j] & mask], 1u);
    }
    __syncthreads();
    const uint32_t c = sh[threadIdx.x];
    const uint64_t sg = ((uint64_t)bucket << bits_mid) + threadIdx.x;
    if (c && sg < nseg) atomicAdd(&seg_hist[sg], c);
}

// Stage floats [w_src, w_src + words) of `base` (total_words long) in shared
// memory at sx[off ..], off = w_src mod 4: 16-byte cp.async chunks from the
// aligned word at or below w_src when `base` is 16-byte aligned (the chunks
// stay inside the array; words past the last whole chunk load plainly), else
// plain loads (off = 0).  sx holds at least words + 6 floats.  The copies are
// awaited by the caller (cp_async_wait_all, then a block barrier).
__device__ __forceinline__ uint32_t pb_stage(const float* __restrict__ base, int aligned, uint64_t w_src,
                                             uint32_t words, uint64_t total_words, float* sx) {
    const uint32_t tid = threadIdx.x;
    if (!aligned) {
        for (uint32_t w = tid; w < words; w += PB_THREADS) sx[w] = base[w_src + w];
        return 0u;
    }
    const uint64_t a0 = w_src & ~3ull, wend = w_src + words;
    const uint64_t cend = min((wend + 3ull) & ~3ull, total_words & ~3ull);
    const uint32_t chunks = cend > a0 ? (uint32_t)((cend - a0) >> 2) : 0u;
    for (uint32_t c = tid; c < chunks; c += PB_THREADS) cp_async16(sx + 4 * c, base + a0 + 4 * c);
    for (uint64_t w = a0 + 4ull * chunks + tid; w < wend; w += PB_THREADS) sx[w - a0] = base[w];
    return (uint32_t)(w_src - a0);
}

// One partition pass.  kTiles == false: tile blockIdx.x of the caller's
// x,y,z (the first pass; staged in shared memory, keys computed here);
// otherwise tile blockIdx.x of `tiles` over 16-byte (x, y, z, key) records.
// A record's digit is (key >> shift) & (2^bits - 1) and its room is reserved
// from cursors[(bucket << cur_shift) + digit].  With `mid` given, the pass
// also writes mid[slot] = (key >> sb) & mid_mask beside every record.
template <bool kTiles>
__global__ void __launch_bounds__(PB_THREADS, 2)
k_pb_partition(const float* __restrict__ xyz, int xyz_aligned, const float4* __restrict__ in,
               const PbTile* __restrict__ tiles, const uint32_t* __restrict__ ntiles, uint64_t n, GridGeom g,
               int shift, int bits, int cur_shift, uint32_t* __restrict__ cursors, float4* __restrict__ out,
               uint16_t* __restrict__ mid, int sb, uint32_t mid_mask) {
    __shared__ uint32_t cnt[PB_THREADS];  // one bin per thread (digits of <= 9 bits)
    __shared__ uint32_t dstart[PB_THREADS];
    __shared__ uint32_t delta[PB_THREADS];
    __shared__ uint32_t ws[PB_THREADS / 32 + 1];
    extern __shared__ float4 xch[];
    const int tid = threadIdx.x;
    const uint32_t mask = (1u << bits) - 1u;
    uint64_t start;
    uint32_t len, bucket;
    if constexpr (!kTiles) {
        start = (uint64_t)blockIdx.x * PB_TILE;
        const uint64_t rem = n - start;
        len = rem < PB_TILE ? (uint32_t)rem : PB_TILE;
        bucket = 0;
    } else {
        if (blockIdx.x >= *ntiles) return;
        const PbTile tl = tiles[blockIdx.x];
        start = tl.start;
        len = tl.len;
        bucket = tl.bucket;
    }
    cnt[tid] = 0;
    float4 v[PB_ITEMS];
    if constexpr (!kTiles) {
        float* sx = reinterpret_cast<float*>(xch);
        const uint32_t off = pb_stage(xyz, xyz_aligned, 3 * start, 3u * len, 3 * n, sx);
        cp_async_wait_all();
        __syncthreads();
#pragma unroll
        for (int i = 0; i < PB_ITEMS; ++i) {
            const uint32_t loc = (uint32_t)i * PB_THREADS + (uint32_t)tid;
            if (loc < len) {
                const float x = sx[off + 3 * loc], y = sx[off + 3 * loc + 1], z = sx[off + 3 * loc + 2];
                v[i] = make_float4(x, y, z, __uint_as_float(cell_key(g, x, y, z)));
            }
        }
    } else {
#pragma unroll
        for (int i = 0; i < PB_ITEMS; ++i) {
            const uint32_t loc = (uint32_t)i * PB_THREADS + (uint32_t)tid;
            if (loc < len) v[i] = in[start + loc];
        }
        __syncthreads();
    }
    uint32_t r[PB_ITEMS];
#pragma unroll
    for (int i = 0; i < PB_ITEMS; ++i) {
        const uint32_t loc = (uint32_t)i * PB_THREADS + (uint32_t)tid;
        if (loc < len) r[i] = atomicAdd(&cnt[(pb_key(v[i]) >> shift) & mask], 1u);
    }
    __syncthreads();  // ranks done; the staged x,y,z are no longer read
    const uint32_t c = cnt[tid];
    uint32_t gb = 0, total;
    if (c) gb = atomicAdd(&cursors[((uint64_t)bucket << cur_shift) + (uint64_t)tid], c);
    const uint32_t ds = pb_block_scan(c, ws, &total);
    dstart[tid] = ds;
    delta[tid] = gb - ds;  // slot of the record at tile position j of this digit: delta + j
    __syncthreads();
#pragma unroll
    for (int i = 0; i < PB_ITEMS; ++i) {
        const uint32_t loc = (uint32_t)i * PB_THREADS + (uint32_t)tid;
        if (loc < len) xch[dstart[(pb_key(v[i]) >> shift) & mask] + r[i]] = v[i];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < PB_ITEMS; ++k) {
        const uint32_t j = (uint32_t)k * PB_THREADS + (uint32_t)tid;
        if (j < len) {
            const float4 w = xch[j];
            const uint32_t o = delta[(pb_key(w) >> shift) & mask] + j;
            if (o < n) {  // in range unless the input changed after the histogram
                out[o] = w;
                if (mid) mid[o] = (uint16_t)((pb_key(w) >> sb) & mid_mask);
            }
        }
    }
}

// Last pass: block b counting-sorts the records of cells [4096 b, 4096 b +
// 4096) (whole segments of 2^sb cells, contiguous after the partition passes)
// and writes cell_start for those of its cells that are <= ncells.  A group
// of at most PB_TILE records goes through shared memory; a larger one is read
// twice (counts, then placement) and written in place.
__global__ void __launch_bounds__(PB_THREADS, 2)
k_pb_cells(const float4* __restrict__ in, const uint32_t* __restrict__ seg_start, uint64_t nseg, int sb,
           uint64_t ncells, uint32_t* __restrict__ cs, float4* __restrict__ out) {
    __shared__ __align__(16) uint32_t hist[PB_GROUP_CELLS];
    __shared__ uint32_t ws[PB_THREADS / 32 + 1];
    extern __shared__ float4 xch[];
    static_assert(PB_GROUP_CELLS == 8 * PB_THREADS, "a thread scans 8 cells");
    const int tid = threadIdx.x;
    const uint64_t cell0 = (uint64_t)blockIdx.x * PB_GROUP_CELLS;
    const uint64_t seg0 = cell0 >> sb;
    const uint64_t seg1 = min(seg0 + (PB_GROUP_CELLS >> sb), nseg);
    const uint32_t lo = seg_start[seg0], cnt = seg_start[seg1] - lo;
    const uint32_t c0 = (uint32_t)cell0;
    uint4* h4 = reinterpret_cast<uint4*>(hist);
    h4[2 * tid] = make_uint4(0u, 0u, 0u, 0u);
    h4[2 * tid + 1] = make_uint4(0u, 0u, 0u, 0u);
    const bool fits = cnt <= PB_TILE;
    float4 v[PB_ITEMS];
    uint32_t r[PB_ITEMS];
    if (fits) {
#pragma unroll
        for (int i = 0; i < PB_ITEMS; ++i) {
            const uint32_t j = (uint32_t)i * PB_THREADS + (uint32_t)tid;
            if (j < cnt) v[i] = in[lo + j];
        }
    }
    __syncthreads();
    if (fits) {
#pragma unroll
        for (int i = 0; i < PB_ITEMS; ++i) {
            const uint32_t j = (uint32_t)i * PB_THREADS + (uint32_t)tid;
            r[i] = 0xffffffffu;
            if (j < cnt) {
                // a key outside the group (only if the input changed after the
                // histogram) is dropped rather than counted out of range
                const uint32_t lk = pb_key(v[i]) - c0;
                if (lk < PB_GROUP_CELLS) r[i] = atomicAdd(&hist[lk], 1u);
            }
        }
    } else {
        for (uint32_t j = (uint32_t)tid; j < cnt; j += PB_THREADS) {
            const uint32_t lk = pb_key(in[lo + j]) - c0;
            if (lk < PB_GROUP_CELLS) atomicAdd(&hist[lk], 1u);
        }
    }
    __syncthreads();
    // exclusive scan of the 4096 cell counts; thread t owns cells 8t .. 8t+7
    const uint4 a = h4[2 * tid], b = h4[2 * tid + 1];
    uint32_t e[8];
    e[0] = 0u;
    e[1] = a.x;
    e[2] = e[1] + a.y;
    e[3] = e[2] + a.z;
    e[4] = e[3] + a.w;
    e[5] = e[4] + b.x;
    e[6] = e[5] + b.y;
    e[7] = e[6] + b.z;
    uint32_t total;
    const uint32_t base = pb_block_scan(e[7] + b.w, ws, &total);
#pragma unroll
    for (int k = 0; k < 8; ++k) e[k] += base;
    h4[2 * tid] = make_uint4(e[0], e[1], e[2], e[3]);
    h4[2 * tid + 1] = make_uint4(e[4], e[5], e[6], e[7]);
    const uint64_t c8 = cell0 + 8u * (uint64_t)tid;
    if (c8 + 7 <= ncells) {
        uint4* dst = reinterpret_cast<uint4*>(cs + c8);
        dst[0] = make_uint4(lo + e[0], lo + e[1], lo + e[2], lo + e[3]);
        dst[1] = make_uint4(lo + e[4], lo + e[5], lo + e[6], lo + e[7]);
    } else {
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (c8 + k <= ncells) cs[c8 + k] = lo + e[k];
    }
    __syncthreads();
    if (fits) {
#pragma unroll
        for (int i = 0; i < PB_ITEMS; ++i) {
            if (r[i] != 0xffffffffu) xch[hist[pb_key(v[i]) - c0] + r[i]] = v[i];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < PB_ITEMS; ++k) {
            const uint32_t j = (uint32_t)k * PB_THREADS + (uint32_t)tid;
            if (j < cnt) out[lo + j] = xch[j];
        }
    } else {
        for (uint32_t j = (uint32_t)tid; j < cnt; j += PB_THREADS) {
            const float4 w = in[lo + j];
            const uint32_t lk = pb_key(w) - c0;
            if (lk < PB_GROUP_CELLS) out[lo + atomicAdd(&hist[lk], 1u)] = w;
        }
    }
}

// The partition build into pts (n records) and cs (ncells + 1 entries).
int build_grid_partitioned(const float* d_xyz, uint64_t n, const GridGeom& g, float4* pts, uint32_t* cs,
                           cudaStream_t s) {
    if (n == 0) {
        SJCS_CUDA_TRY(cudaMemsetAsync(cs, 0, (g.ncells + 1) * sizeof(uint32_t), s));
        return SJCS_OK;
    }
    const int kb = grid_key_bits(g);
    const int sb = kb > PB_MIN_SEG_BITS + 18 ? kb - 18 : PB_MIN_SEG_BITS;  // segment bits, <= PB_GROUP_BITS
    const int upper = kb > sb ? kb - sb : 0;  // bits above the segment
    const int bits_mid = upper > 9 ? upper - 9 : 0;
    const int bits_top = upper - bits_mid;
    const uint64_t nseg = (g.ncells + (1ull << sb) - 1) >> sb;
    const uint32_t ntop = (uint32_t)((nseg + (1ull << bits_mid) - 1) >> bits_mid);
    const uint64_t ntiles_in = (n + PB_TILE - 1) / PB_TILE;
    const uint64_t ntiles_mid = ntiles_in + ntop;  // bound on the middle pass's tiles
    const uint64_t ngroups = g.ncells / PB_GROUP_CELLS + 1;  // the last one holds cell_start[ncells]
    const int aligned = (reinterpret_cast<uintptr_t>(d_xyz) & 15u) == 0;

    StreamScratch scr(s);
    uint32_t *top = nullptr, *cur_top = nullptr, *seg = nullptr, *cur_seg = nullptr, *ntiles = nullptr;
    float4* tmp = nullptr;
    PbTile* tiles = nullptr;
    uint16_t* mid = nullptr;
    // top digit counts and starts (ntop + 1 entries); without a middle pass
    // the top digit is the segment and these are the segment starts too
    SJCS_CUDA_TRY(scr.alloc(&top, ((uint64_t)ntop + 1) * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&cur_top, (uint64_t)ntop * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&tmp, n * sizeof(float4)));
    if (bits_mid) {
        SJCS_CUDA_TRY(scr.alloc(&seg, (nseg + 1) * sizeof(uint32_t)));
        SJCS_CUDA_TRY(scr.alloc(&cur_seg, nseg * sizeof(uint32_t)));
        SJCS_CUDA_TRY(scr.alloc(&tiles, ntiles_mid * sizeof(PbTile)));
        SJCS_CUDA_TRY(scr.alloc(&ntiles, sizeof(uint32_t)));
        SJCS_CUDA_TRY(scr.alloc(&mid, n * sizeof(uint16_t)));
        SJCS_CUDA_TRY(cudaMemsetAsync(seg, 0, (nseg + 1) * sizeof(uint32_t), s));
    } else {
        seg = top;
    }
    const int top_shift = sb + bits_mid;
    SJCS_CUDA_TRY(cudaFuncSetAttribute(k_pb_top_hist, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)PB_STAGE_SMEM));
    SJCS_CUDA_TRY(cudaMemsetAsync(top, 0, ((uint64_t)ntop + 1) * sizeof(uint32_t), s));
    k_pb_top_hist<<<(unsigned)((ntiles_in + PB_TOP_TILES - 1) / PB_TOP_TILES), PB_THREADS, PB_STAGE_SMEM, s>>>(
        d_xyz, aligned, n, g, top_shift, top);
    SJCS_LAUNCH_CHECK();
    int rc = exclusive_scan_u32(top, (uint64_t)ntop + 1, s);
    if (rc) return rc;
    SJCS_CUDA_TRY(cudaMemcpyAsync(cur_top, top, (uint64_t)ntop * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    SJCS_CUDA_TRY(cudaFuncSetAttribute(k_pb_partition<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)PB_SMEM));
    SJCS_CUDA_TRY(cudaFuncSetAttribute(k_pb_partition<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)PB_SMEM));
    SJCS_CUDA_TRY(cudaFuncSetAttribute(k_pb_cells, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PB_SMEM));
    // pass A writes pts when a middle pass follows (pts is free until the
    // last pass), else tmp; with a middle pass it also writes the middle digits
    float4* a_out = bits_mid ? pts : tmp;
    const uint32_t mid_mask = (1u << bits_mid) - 1u;
    k_pb_partition<false><<<(unsigned)ntiles_in, PB_THREADS, PB_SMEM, s>>>(
        d_xyz, aligned, nullptr, nullptr, nullptr, n, g, top_shift, bits_top, 0, cur_top, a_out, mid, sb, mid_mask);
    SJCS_LAUNCH_CHECK();
    if (bits_mid) {
        const unsigned tile_blocks = (unsigned)((ntiles_mid + PB_THREADS - 1) / PB_THREADS);
        k_pb_tiles<<<tile_blocks, PB_THREADS, 0, s>>>(top, ntop, tiles, ntiles);
        SJCS_LAUNCH_CHECK();
        k_pb_mid_hist<<<(unsigned)((ntiles_mid + PB_MID_TILES - 1) / PB_MID_TILES), PB_THREADS, 0, s>>>(
            mid, tiles, ntiles, bits_mid, nseg, seg);
        SJCS_LAUNCH_CHECK();
        rc = exclusive_scan_u32(seg, nseg + 1, s);
        if (rc) return rc;
        SJCS_CUDA_TRY(cudaMemcpyAsync(cur_seg, seg, nseg * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
        k_pb_partition<true><<<(unsigned)ntiles_mid, PB_THREADS, PB_SMEM, s>>>(
            nullptr, 0, pts, tiles, ntiles, n, g, sb, bits_mid, bits_mid, cur_seg, tmp, nullptr, sb, 0u);
        SJCS_LAUNCH_CHECK();
    }
    k_pb_cells<<<(unsigned)ngroups, PB_THREADS, PB_SMEM, s>>>(tmp, seg, nseg, sb, g.ncells, cs, pts);
    SJCS_LAUNCH_CHECK();
    return SJCS_OK;
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
        // Target about 1.6 cells per particle, at most 2^28 cells (a 1 GB
        // cell table; keys of up to 30 bits take the partition build), and
        // keep y/z cells >= R/4: a query box then spans at most 9x9 rows.
        // A box spans at most 5x5 rows -- the per-batch row plan -- when
        // y/z cells are >= R/2, so cells go below R/2 only as far as the
        // 2^27-cell size would (the 5x5 plan counts far faster than 6x6
        // boxes without it, for the small gain of finer cells).
        constexpr double kMaxCells = 268435456.0;  // 2^28
        const double want = std::max(1.6 * (double)n, 4096.0);
        double hyz = std::cbrt(2.5e9 / std::min(want, kMaxCells));
        if (radius_hint > 0.0f) {
            const double h27 = std::cbrt(2.5e9 / std::min(want, 134217728.0));
            hyz = std::max(hyz, std::min(0.5 * (double)radius_hint, h27));
            hyz = std::max(hyz, 0.25 * (double)radius_hint);
        }
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
    if (grid_key_bits(g) <= PB_MAX_KEY_BITS)
        return build_grid_partitioned(d_xyz, n, g, reinterpret_cast<float4*>(idx->pts), idx->cell_start, s);

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
