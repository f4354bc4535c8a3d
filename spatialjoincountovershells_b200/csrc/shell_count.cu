// Warp-cooperative periodic multi-shell count (plain grid index).
//
// One warp owns one halo at a time.  For every periodic image of the halo the
// warp turns the query box into rows of cells (one row = one contiguous slot
// range of the sorted particles), clips each row's x-extent to the sphere of
// radius R with conservative floating-point margins (a row whose cells cannot
// hold a particle within R is skipped), flattens the rows into one candidate
// sequence and lets lane l test candidates l, l+32, ... so every particle load
// is a coalesced 128-bit load.  Accepted candidates are binned through a
// lookup table on the float bit pattern of the squared distance (one compare
// refines the slot) and counted in per-warp shared-memory counters; the warp
// adds its counters to the halo's row once per halo with fire-and-forget
// reductions.
//
// Arithmetic follows the reference exactly (fp32, round-to-nearest, no FMA,
// no flush-to-zero):
//   R     = (float)sqrt((double)r2[n-1])               MultiRangeCount.c:19 (host side)
//   box   lo = c - R, hi = c + R                        setQueryMbr, Mbr.c:207-239
//   test  !(p < lo) && !(hi < p) on x, y, z             checkOverlapMbr, Mbr.c:167-205
//   dist  (dx*dx + dy*dy) + dz*dz, d = p - c            CalcDistance, Distance.h:5-25 (_mm_dp_ps 0x77)
//   shell first i with dist < r2[i]                     MultiRangeCountRecursive, MultiRangeCount.c:103-113
//   images: flags from the un-shifted box, lo < 0 -> c += 1000, else hi > 1000
//           -> c -= 1000, every non-empty subset of the flagged axes
//                                                       MultiRangeCount.c:31-71, Mbr.c:284-313
// For a non-decreasing, NaN-free table "first i with dist < r2[i]" equals
// #{i : r2[i] <= dist} and a particle is counted iff dist < r2[n-1]; other
// tables use the literal first-match scan (and no sphere clipping).
//
// Why the sphere clipping never drops a counted particle: a counted particle
// has fp32 dist < r2max, and fp32 rounding of the 3 differences and 5
// products/sums lowers the exact squared distance by at most a factor
// (1 - 2^-24)^5, so its exact squared distance is < r2max * (1 + 1e-5) = r2p.
// Its y lies inside its cell's y-extent, so (py - cy)^2 >= gy^2 where gy is a
// lower bound of the halo's distance to that extent (cell edges widened by
// 1e-3 + 2e-6*|edge|, far above the rounding of k*h and of the cell function);
// likewise z.  Hence (px - cx)^2 < r2p - gy^2 - gz^2, and the fp32 evaluation
// of that bound is off by at most 4 ulps of r2p < 1e-5*r2p, which is added
// back before the square root; the x cell range then uses cx -+ (xr + 1e-3 +
// 1e-6*(|cx| + xr)).
#include "count_common.cuh"
#include "queue_common.cuh"
#include "radix_sort.cuh"
#include "sjcs_internal.cuh"

namespace sjcs {
namespace {

using namespace count;

constexpr int CT_WARPS = 4;
constexpr int CT_THREADS = CT_WARPS * 32;
constexpr int kMaxSmemTable = 8192;  // r2 entries held in shared memory
constexpr int kMaxSmemRads = 1024;   // per-warp shared counters up to this many shells

// Row r of the image (r < nrows) -> (y cell, z cell); exact for all r < 2^31.
__device__ __forceinline__ void row_yz(const Image& im, uint32_t r, int* yy, int* zz) {
    uint32_t q;
    if (im.nrows <= (1u << 20)) {
        // float quotient estimate: relative error < 4e-7, so for r < 2^20 it is
        // off by at most one; corrected exactly below
        q = (uint32_t)__fmul_rz((float)r, __frcp_rn((float)im.ny));
        if (q * (uint32_t)im.ny > r) --q;
        else if ((q + 1u) * (uint32_t)im.ny <= r) ++q;
    } else {
        q = r / (uint32_t)im.ny;
    }
    *yy = im.y0 + (int)(r - q * (uint32_t)im.ny);
    *zz = im.z0 + (int)q;
}

// Lane `lane` takes row rb + lane of the image: clip its x cells to the
// sphere and fetch the row's first and one-past-last slots.  Returns the
// slot range through *start / *end (empty: start == end).  gy_l / gz_l are
// the lane-distributed gap tables of the image (valid when ny, nz <= 32).
__device__ __forceinline__ void row_issue(const CountParams& p, const Image& im, uint32_t rb, int lane,
                                          float gy_l, float gz_l, uint32_t* start, uint32_t* end) {
    const uint32_t r = rb + (uint32_t)lane;
    int yy = 0, zz = 0;
    const bool live = r < im.nrows;
    if (live) row_yz(im, r, &yy, &zz);
    int xa = im.x0, xb = im.x1;
    if (p.prune) {
        const bool small = im.ny <= 32 && im.nz <= 32;
        float gy = __shfl_sync(0xffffffffu, gy_l, (yy - im.y0) & 31);
        float gz = __shfl_sync(0xffffffffu, gz_l, (zz - im.z0) & 31);
        if (!small) {
            gy = cell_gap(im.cy, yy, p.h[1], p.g.G[1]);
            gz = cell_gap(im.cz, zz, p.h[2], p.g.G[2]);
        }
        const float rem =
            __fadd_rn(__fsub_rn(__fsub_rn(p.r2p, __fmul_rn(gy, gy)), __fmul_rn(gz, gz)), p.r2slack);
        if (rem < 0.0f) {
            xb = xa - 1;  // no particle of this row can be within R
        } else {
            // approximate square root: its error (< 1e-6 relative) is far inside the margin
            float xr = rem > 0.0f ? __fmul_rn(rem, rsqrtf(rem)) : 0.0f;
            xr = __fadd_rn(xr, 1e-3f + 1e-6f * (fabsf(im.cx) + xr));
            const float xl = __fsub_rn(im.cx, xr), xh = __fadd_rn(im.cx, xr);
            xa = max(xa, cell_of(xl, p.g.inv_h[0], p.g.G[0]));
            if (xh == xh) xb = min(xb, cell_of(xh, p.g.inv_h[0], p.g.G[0]));
        }
    }
    uint32_t s0 = 0, s1 = 0;
    if (live && xa <= xb) {
        const uint64_t rowcell = ((uint64_t)zz * (uint64_t)p.g.G[1] + (uint64_t)yy) * (uint64_t)p.g.G[0];
        s0 = __ldg(p.cs + rowcell + xa);
        s1 = __ldg(p.cs + rowcell + xb + 1);
    }
    *start = s0;
    *end = s1;
}

// Lane-distributed gap tables: lane j holds the gap of y cell y0 + j (and z).
__device__ __forceinline__ void gap_tables(const CountParams& p, const Image& im, int lane, float* gy, float* gz) {
    *gy = 0.0f;
    *gz = 0.0f;
    if (p.prune) {
        if (lane < im.ny) *gy = cell_gap(im.cy, im.y0 + lane, p.h[1], p.g.G[1]);
        if (lane < im.nz) *gz = cell_gap(im.cz, im.z0 + lane, p.h[2], p.g.G[2]);
    }
}

// Every row chunk of an image from chunk `first_chunk` on, synchronously.
template <int BIN, bool BIG>
__device__ __forceinline__ void count_image(const CountParams& p, const Image& im, uint32_t first_chunk,
                                            uint32_t* __restrict__ sink, const float* __restrict__ tab,
                                            const uint32_t* __restrict__ lut, int lane) {
    float gy, gz;
    gap_tables(p, im, lane, &gy, &gz);
    for (uint32_t rb = first_chunk * 32u; rb < im.nrows; rb += 32u) {
        uint32_t s0, s1;
        row_issue(p, im, rb, lane, gy, gz, &s0, &s1);
        run_rows<BIN, BIG>(p, im, s0, s1, sink, tab, lut, lane);
    }
}

// Piece `part` of `nparts` of every row chunk of an image (heavy halos
// shared by several warps).
template <int BIN, bool BIG>
__device__ __forceinline__ void count_image_part(const CountParams& p, const Image& im,
                                                 uint32_t* __restrict__ sink, const float* __restrict__ tab,
                                                 const uint32_t* __restrict__ lut, int lane, uint32_t part,
                                                 uint32_t nparts) {
    float gy, gz;
    gap_tables(p, im, lane, &gy, &gz);
    for (uint32_t rb = 0; rb < im.nrows; rb += 32u) {
        uint32_t s0, s1;
        row_issue(p, im, rb, lane, gy, gz, &s0, &s1);
        run_rows_part<BIN, BIG>(p, im, s0, s1, sink, tab, lut, lane, part, nparts);
    }
}

// Periodic images other than the un-shifted one: every non-empty subset S of
// the flagged axes (MultiRangeCount.c:31-71).  nparts > 1: this warp's piece
// of each image only.
template <int BIN, bool BIG>
__device__ __forceinline__ void count_shifted_images(const CountParams& p, const float4 c,
                                                     uint32_t* __restrict__ sink, const float* __restrict__ tab,
                                                     const uint32_t* __restrict__ lut, int lane,
                                                     uint32_t part = 0, uint32_t nparts = 1) {
    const float lox = __fsub_rn(c.x, p.half), hix = __fadd_rn(c.x, p.half);
    const float loy = __fsub_rn(c.y, p.half), hiy = __fadd_rn(c.y, p.half);
    const float loz = __fsub_rn(c.z, p.half), hiz = __fadd_rn(c.z, p.half);
    const unsigned F = ((lox < kBoxLow) | (hix > kBoxUpp) ? 1u : 0u) |
                       ((loy < kBoxLow) | (hiy > kBoxUpp) ? 2u : 0u) |
                       ((loz < kBoxLow) | (hiz > kBoxUpp) ? 4u : 0u);
    if (F == 0) return;
    // min_oob takes precedence over max_oob on an axis (MultiRangeCount.c:38-43)
    const float sx = (lox < kBoxLow) ? __fadd_rn(c.x, kBoxUpp) : __fsub_rn(c.x, kBoxUpp);
    const float sy = (loy < kBoxLow) ? __fadd_rn(c.y, kBoxUpp) : __fsub_rn(c.y, kBoxUpp);
    const float sz = (loz < kBoxLow) ? __fadd_rn(c.z, kBoxUpp) : __fsub_rn(c.z, kBoxUpp);
    for (unsigned S = F; S != 0; S = (S - 1u) & F) {
        const Image im = make_image(p, (S & 1u) ? sx : c.x, (S & 2u) ? sy : c.y, (S & 4u) ? sz : c.z);
        if (nparts > 1) count_image_part<BIN, BIG>(p, im, sink, tab, lut, lane, part, nparts);
        else count_image<BIN, BIG>(p, im, 0, sink, tab, lut, lane);
    }
}

// Per-halo plan written by the planning phase (one lane per halo).
struct HaloPlan {
    float cx, cy, cz;  // the box is c -+ half, recomputed (same fp32 ops) when the halo is counted
    uint32_t row;    // the halo's row in the count array
    uint32_t nrows;  // rows stored in the row list; kSlowPlan: count in place
    uint32_t flags;  // periodic axes whose box crosses a face (bit a = axis a)
};
constexpr uint32_t kSlowPlan = 0xffffffffu;
constexpr int kBatch = 32;    // halos per warp batch (one per lane while planning)
constexpr int kMaxRows = 25;  // rows kept per halo (5x5 rows: boxes up to 2R <= 4 y/z cells)

// Shared memory of one warp: plans and row lists of its current batch (24 B
// plans and 25-row lists keep a block at ~25 KB, so 8 blocks fit an SM).
struct WarpPlans {
    HaloPlan plan[kBatch];
    uint32_t row_cell[kBatch][kMaxRows];  // cell-table index of the row's first cell
    uint16_t row_len[kBatch][kMaxRows];   // number of cells of the row
};

// Planning (lane = halo): the un-shifted image's box, and every row of cells
// the sphere can reach, clipped in x, as a cell-table index range.
__device__ __forceinline__ void plan_halo(const CountParams& p, float4 c, bool valid, HaloPlan* pl,
                                          uint32_t* row_cell, uint16_t* row_len) {
    const Image im = make_image(p, c.x, c.y, c.z);
    pl->cx = im.cx;
    pl->cy = im.cy;
    pl->cz = im.cz;
    pl->row = __float_as_uint(c.w);
    uint32_t F = 0;
    if (p.periodic)
        F = ((im.lox < kBoxLow) | (im.hix > kBoxUpp) ? 1u : 0u) | ((im.loy < kBoxLow) | (im.hiy > kBoxUpp) ? 2u : 0u) |
            ((im.loz < kBoxLow) | (im.hiz > kBoxUpp) ? 4u : 0u);
    pl->flags = F;
    if (!valid) {
        pl->nrows = 0;
        return;
    }
    if (im.nrows > (uint32_t)kMaxRows) {
        pl->nrows = kSlowPlan;
        return;
    }
    uint32_t k = 0;
    for (int zz = im.z0; zz <= im.z1; ++zz) {
        const float gz = p.prune ? cell_gap(im.cz, zz, p.h[2], p.g.G[2]) : 0.0f;
        const float rz = __fsub_rn(p.r2p, __fmul_rn(gz, gz));
        for (int yy = im.y0; yy <= im.y1; ++yy) {
            int xa = im.x0, xb = im.x1;
            if (p.prune) {
                const float gy = cell_gap(im.cy, yy, p.h[1], p.g.G[1]);
                const float rem = __fadd_rn(__fsub_rn(rz, __fmul_rn(gy, gy)), p.r2slack);
                if (rem < 0.0f) continue;  // no particle of this row can be within R
                // approximate square root: its error (< 1e-6 relative) is far inside the margin
                float xr = rem > 0.0f ? __fmul_rn(rem, rsqrtf(rem)) : 0.0f;
                xr = __fadd_rn(xr, 1e-3f + 1e-6f * (fabsf(im.cx) + xr));
                const float xl = __fsub_rn(im.cx, xr), xh = __fadd_rn(im.cx, xr);
                xa = max(xa, cell_of(xl, p.g.inv_h[0], p.g.G[0]));
                if (xh == xh) xb = min(xb, cell_of(xh, p.g.inv_h[0], p.g.G[0]));
            }
            if (xa > xb) continue;
            const uint32_t rowcell = ((uint32_t)zz * (uint32_t)p.g.G[1] + (uint32_t)yy) * (uint32_t)p.g.G[0];
            row_cell[k] = rowcell + (uint32_t)xa;
            row_len[k] = (uint16_t)(xb - xa + 1);
            ++k;
        }
    }
    pl->nrows = k;
}

// Lane r fetches the slot range of row r of planned halo k.
__device__ __forceinline__ void fetch_rows(const CountParams& p, const WarpPlans* wp, uint32_t k, uint32_t nrows,
                                           int lane, uint32_t* s0, uint32_t* s1) {
    uint32_t a = 0, b = 0;
    if ((uint32_t)lane < nrows) {
        const uint32_t c0 = wp->row_cell[k][lane];
        a = __ldg(p.cs + c0);
        b = __ldg(p.cs + c0 + wp->row_len[k][lane]);
    }
    *s0 = a;
    *s1 = b;
}

// Flush a warp's shared counters into the halo's count row (fire-and-forget
// reductions) and clear them.
__device__ __forceinline__ void flush_counts(const CountParams& p, uint32_t* __restrict__ wcnt,
                                             uint32_t* __restrict__ row, int lane) {
    __syncwarp();
    for (int sh = lane; sh < p.nrads; sh += 32) {
        const uint32_t v = wcnt[sh];
        if (v) {
            wcnt[sh] = 0u;
            atomicAdd(row + sh, v);  // result unused: compiles to a reduction
        }
    }
    __syncwarp();
}

// One batch of nb <= 32 halos (halo k = c_lane of lane k).  Planning runs one
// lane per halo; execution runs the whole warp on one halo at a time over its
// planned rows, while the cell-table loads of the next halo of the batch are
// in flight.  Halos with more than 28 rows and the shifted periodic images
// (about 3% of halos at the workload's sizes) are counted in place.
template <int BIN, bool BIG>
__device__ __forceinline__ void count_batch(const CountParams& p, WarpPlans* wp, uint32_t nb, float4 c_lane,
                                            uint32_t* __restrict__ wcnt, const float* __restrict__ tab,
                                            const uint32_t* __restrict__ lut, int lane) {
    {
        const bool valid = (uint32_t)lane < nb;
        plan_halo(p, c_lane, valid, &wp->plan[lane], wp->row_cell[lane], wp->row_len[lane]);
    }
    __syncwarp();
    uint32_t s0, s1;
    {
        const uint32_t n0 = wp->plan[0].nrows;
        fetch_rows(p, wp, 0, n0 == kSlowPlan ? 0u : n0, lane, &s0, &s1);
    }
    for (uint32_t k = 0; k < nb; ++k) {
        const HaloPlan pl = wp->plan[k];
        // the next halo's row loads overlap this halo's tests
        uint32_t t0 = 0, t1 = 0;
        if (k + 1 < nb) {
            const uint32_t nn = wp->plan[k + 1].nrows;
            fetch_rows(p, wp, k + 1, nn == kSlowPlan ? 0u : nn, lane, &t0, &t1);
        }
        uint32_t* row = p.counts + (uint64_t)pl.row * (uint64_t)p.nrads;
        uint32_t* sink = BIG ? row : wcnt;
        Image im;
        im.cx = pl.cx;
        im.cy = pl.cy;
        im.cz = pl.cz;
        im.lox = __fsub_rn(pl.cx, p.half);
        im.hix = __fadd_rn(pl.cx, p.half);
        im.loy = __fsub_rn(pl.cy, p.half);
        im.hiy = __fadd_rn(pl.cy, p.half);
        im.loz = __fsub_rn(pl.cz, p.half);
        im.hiz = __fadd_rn(pl.cz, p.half);
        if (pl.nrows == kSlowPlan) {
            count_image<BIN, BIG>(p, make_image(p, pl.cx, pl.cy, pl.cz), 0, sink, tab, lut, lane);
        } else {
            run_rows<BIN, BIG>(p, im, s0, s1, sink, tab, lut, lane);
        }
        if (pl.flags) count_shifted_images<BIN, BIG>(p, make_float4(pl.cx, pl.cy, pl.cz, 0.f), sink, tab, lut, lane);
        if (!BIG) flush_counts(p, wcnt, row, lane);
        s0 = t0;
        s1 = t1;
    }
    __syncwarp();  // the batch's plans are read before the next batch overwrites them
}

// count_batch over several indexes of one grid (p.nidx of them): a halo is
// planned once, and its rows are fetched from every index in turn -- the
// next (halo, index) pair's row loads in flight during the current pair's
// tests -- before its counters are flushed once.  Each index is counted
// through a copy of the parameters that points at it, so the row and
// candidate code is the single-index code.
template <int BIN, bool BIG>
__device__ __forceinline__ void count_batch_multi(const CountParams& p, WarpPlans* wp, uint32_t nb, float4 c_lane,
                                                  uint32_t* __restrict__ wcnt, const float* __restrict__ tab,
                                                  const uint32_t* __restrict__ lut, int lane) {
    {
        const bool valid = (uint32_t)lane < nb;
        plan_halo(p, c_lane, valid, &wp->plan[lane], wp->row_cell[lane], wp->row_len[lane]);
    }
    __syncwarp();
    const int nf = p.nidx;
    uint32_t s0, s1;
    {
        CountParams p0 = p;
        p0.cs = p.mcs[0];
        const uint32_t n0 = wp->plan[0].nrows;
        fetch_rows(p0, wp, 0, n0 == kSlowPlan ? 0u : n0, lane, &s0, &s1);
    }
    for (uint32_t k = 0; k < nb; ++k) {
        for (int f = 0; f < nf; ++f) {
            const bool last = f + 1 == nf;
            const uint32_t kn = last ? k + 1 : k;
            uint32_t t0 = 0, t1 = 0;
            if (kn < nb) {
                CountParams pn = p;
                pn.cs = p.mcs[last ? 0 : f + 1];
                const uint32_t nn = wp->plan[kn].nrows;
                fetch_rows(pn, wp, kn, nn == kSlowPlan ? 0u : nn, lane, &t0, &t1);
            }
            CountParams pf = p;
            pf.pts = p.mpts[f];
            pf.cs = p.mcs[f];
            // the plan and box are read again per index: fewer registers live
            // across the index loop
            const HaloPlan pl = wp->plan[k];
            uint32_t* sink = BIG ? p.counts + (uint64_t)pl.row * (uint64_t)p.nrads : wcnt;
            if (pl.nrows == kSlowPlan) {
                count_image<BIN, BIG>(pf, make_image(pf, pl.cx, pl.cy, pl.cz), 0, sink, tab, lut, lane);
            } else {
                Image im;
                im.cx = pl.cx;
                im.cy = pl.cy;
                im.cz = pl.cz;
                im.lox = __fsub_rn(pl.cx, p.half);
                im.hix = __fadd_rn(pl.cx, p.half);
                im.loy = __fsub_rn(pl.cy, p.half);
                im.hiy = __fadd_rn(pl.cy, p.half);
                im.loz = __fsub_rn(pl.cz, p.half);
                im.hiz = __fadd_rn(pl.cz, p.half);
                run_rows<BIN, BIG>(pf, im, s0, s1, sink, tab, lut, lane);
            }
            if (pl.flags) count_shifted_images<BIN, BIG>(pf, make_float4(pl.cx, pl.cy, pl.cz, 0.f), sink, tab, lut, lane);
            s0 = t0;
            s1 = t1;
        }
        if (!BIG) flush_counts(p, wcnt, p.counts + (uint64_t)wp->plan[k].row * (uint64_t)p.nrads, lane);
    }
    __syncwarp();
}

// Shared-memory set-up common to both schedules: per-warp plans, the r2
// table, the shell lookup table and per-warp counters.
struct SmemView {
    WarpPlans* wp;
    const float* tab;
    const uint32_t* lut;
    uint32_t* wcnt;
};

template <bool BIG>
__device__ __forceinline__ SmemView setup_smem(const CountParams& p, uint32_t* smem, int tid, int warp) {
    SmemView v;
    v.wp = reinterpret_cast<WarpPlans*>(smem) + warp;
    float* r2s = reinterpret_cast<float*>(reinterpret_cast<WarpPlans*>(smem) + CT_WARPS);
    uint32_t* luts = reinterpret_cast<uint32_t*>(r2s + p.pad);
    v.wcnt = luts + p.nlut + warp * p.nrads;
    if (!BIG) {
        for (int i = tid; i < p.pad; i += CT_THREADS) r2s[i] = p.r2[i];
        for (int i = tid; i < p.nlut; i += CT_THREADS) luts[i] = p.lut[i];
        for (int i = tid; i < CT_WARPS * p.nrads; i += CT_THREADS) luts[p.nlut + i] = 0u;
    }
    v.tab = BIG ? p.r2 : r2s;
    v.lut = BIG ? p.lut : luts;
    return v;
}

// Static schedule: warp gw of W takes halos gw, gw + W, gw + 2W, ... in
// batches of 32, so at any moment the resident warps work on one contiguous
// window of the Morton order and share particle lines in L1/L2.
template <int BIN, bool BIG>
__global__ void __launch_bounds__(CT_THREADS, 8) k_shell_count(CountParams p) {
    extern __shared__ uint32_t smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const SmemView v = setup_smem<BIG>(p, smem, tid, warp);
    __syncthreads();
    const uint64_t W = (uint64_t)gridDim.x * CT_WARPS;
    const uint64_t gw = (uint64_t)blockIdx.x * CT_WARPS + warp;
    const uint64_t mine = p.nhalos > gw ? (p.nhalos - gw + W - 1) / W : 0;  // halos of this warp
    for (uint64_t b0 = 0; b0 < mine; b0 += kBatch) {
        const uint32_t nb = (uint32_t)min((uint64_t)kBatch, mine - b0);
        const float4 c = (uint32_t)lane < nb ? p.halos[(b0 + lane) * W + gw] : make_float4(0.f, 0.f, 0.f, 0.f);
        count_batch<BIN, BIG>(p, v.wp, nb, c, v.wcnt, v.tab, v.lut, lane);
    }
}

// Static schedule over p.nidx indexes of one grid (count_batch_multi).
template <int BIN, bool BIG>
__global__ void __launch_bounds__(CT_THREADS, 8) k_shell_count_multi(CountParams p) {
    extern __shared__ uint32_t smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const SmemView v = setup_smem<BIG>(p, smem, tid, warp);
    __syncthreads();
    const uint64_t W = (uint64_t)gridDim.x * CT_WARPS;
    const uint64_t gw = (uint64_t)blockIdx.x * CT_WARPS + warp;
    const uint64_t mine = p.nhalos > gw ? (p.nhalos - gw + W - 1) / W : 0;
    for (uint64_t b0 = 0; b0 < mine; b0 += kBatch) {
        const uint32_t nb = (uint32_t)min((uint64_t)kBatch, mine - b0);
        const float4 c = (uint32_t)lane < nb ? p.halos[(b0 + lane) * W + gw] : make_float4(0.f, 0.f, 0.f, 0.f);
        count_batch_multi<BIN, BIG>(p, v.wp, nb, c, v.wcnt, v.tab, v.lut, lane);
    }
}

// ---- persistent work-queue schedule -----------------------------------------
//
// k_estimate    per halo (Morton order): the number of candidates of its
//               clipped rows (times 2^k for k flagged periodic axes) and its
//               size bucket (est_bucket, 8 bits); a histogram of the buckets
// sort          one 8-bit radix pass by descending bucket (stable: Morton
//               order within a bucket) -> ord[i] = Morton index
// k_plan_items  per bucket (lower bound e of its estimates): halos with
//               e >= piece are split into min(max_pieces, ceil(e/piece))
//               pieces that separate warps count (every row set split
//               evenly); halos with e >= single are items of their own;
//               lighter halos go min(32, piece/e) to an item.  The buckets'
//               item counts are prefix-summed into a 256-entry table.
// k_queue       persistent warps claim items with one atomicAdd each (no
//               claim ever fails or retries), largest buckets first, so the
//               longest items start early and the light ones fill the tail.

__global__ void k_estimate(CountParams p, uint32_t* __restrict__ key, uint32_t* __restrict__ hist) {
    __shared__ uint32_t sh[kBuckets];
    for (int i = threadIdx.x; i < kBuckets; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < p.nhalos) {
        const float4 c = p.halos[i];
        const Image im = make_image(p, c.x, c.y, c.z);
        uint32_t e;
        if (im.nrows > 4096u) {
            e = 0x40000000u;  // far too many rows to walk here: certainly heavy
        } else {
            uint64_t sum = 0;
            for (int zz = im.z0; zz <= im.z1; ++zz) {
                const float gz = p.prune ? cell_gap(im.cz, zz, p.h[2], p.g.G[2]) : 0.0f;
                const float rz = __fsub_rn(p.r2p, __fmul_rn(gz, gz));
                for (int yy = im.y0; yy <= im.y1; ++yy) {
                    int xa = im.x0, xb = im.x1;
                    if (p.prune) {
                        const float gy = cell_gap(im.cy, yy, p.h[1], p.g.G[1]);
                        const float rem = __fadd_rn(__fsub_rn(rz, __fmul_rn(gy, gy)), p.r2slack);
                        if (rem < 0.0f) continue;
                        float xr = rem > 0.0f ? __fmul_rn(rem, rsqrtf(rem)) : 0.0f;
                        xr = __fadd_rn(xr, 1e-3f + 1e-6f * (fabsf(im.cx) + xr));
                        xa = max(xa, cell_of(__fsub_rn(im.cx, xr), p.g.inv_h[0], p.g.G[0]));
                        const float xh = __fadd_rn(im.cx, xr);
                        if (xh == xh) xb = min(xb, cell_of(xh, p.g.inv_h[0], p.g.G[0]));
                    }
                    if (xa > xb) continue;
                    const uint64_t rowcell = ((uint64_t)zz * (uint64_t)p.g.G[1] + (uint64_t)yy) * (uint64_t)p.g.G[0];
                    sum += __ldg(p.cs + rowcell + xb + 1) - __ldg(p.cs + rowcell + xa);
                }
            }
            if (p.periodic) {
                const int k = ((im.lox < kBoxLow) | (im.hix > kBoxUpp)) + ((im.loy < kBoxLow) | (im.hiy > kBoxUpp)) +
                              ((im.loz < kBoxLow) | (im.hiz > kBoxUpp));
                sum <<= k;
            }
            e = sum < 0x40000000ull ? (uint32_t)sum : 0x40000000u;
        }
        const uint32_t k = 255u - est_bucket(e);
        key[i] = k;
        atomicAdd(&sh[k], 1u);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kBuckets; k += blockDim.x)
        if (sh[k]) atomicAdd(hist + k, sh[k]);
}

template <int BIN, bool BIG>
__global__ void __launch_bounds__(CT_THREADS, 8) k_shell_count_queue(CountParams p, QueueParams q) {
    extern __shared__ uint32_t smem[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const SmemView v = setup_smem<BIG>(p, smem, tid, warp);
    __syncthreads();
    const uint32_t nitems = q.ctl[1];
    int bk = 0;  // claims only grow, so each warp's bucket search moves forward
    for (;;) {
        BucketPlan bp;
        uint32_t r;
        if (!claim_item(q, nitems, lane, &bk, &bp, &r)) break;
        if (bp.per == 0) {
            const uint32_t pos = bp.start + r / bp.pieces, part = r % bp.pieces;
            const float4 c = p.halos[q.ord[pos]];
            uint32_t* row = p.counts + (uint64_t)__float_as_uint(c.w) * (uint64_t)p.nrads;
            uint32_t* sink = BIG ? row : v.wcnt;
            const Image im = make_image(p, c.x, c.y, c.z);
            if (bp.pieces > 1) count_image_part<BIN, BIG>(p, im, sink, v.tab, v.lut, lane, part, bp.pieces);
            else count_image<BIN, BIG>(p, im, 0, sink, v.tab, v.lut, lane);
            if (p.periodic) count_shifted_images<BIN, BIG>(p, c, sink, v.tab, v.lut, lane, part, bp.pieces);
            if (!BIG) flush_counts(p, v.wcnt, row, lane);
        } else {
            const uint32_t first = r * bp.per;
            const uint32_t nb = min(bp.per, bp.count - first);
            const float4 c = (uint32_t)lane < nb ? p.halos[q.ord[bp.start + first + lane]]
                                                 : make_float4(0.f, 0.f, 0.f, 0.f);
            count_batch<BIN, BIG>(p, v.wp, nb, c, v.wcnt, v.tab, v.lut, lane);
        }
    }
}

template <int BIN, bool BIG>
int launch_variant(sjcs_ctx* ctx, const CountParams& p, size_t smem, cudaStream_t s, bool multi = false) {
    auto kern = multi ? k_shell_count_multi<BIN, BIG> : k_shell_count<BIN, BIG>;
    if (smem > 48 * 1024)
        SJCS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    SJCS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, CT_THREADS, smem));
    if (per_sm < 1) per_sm = 1;
    const uint64_t want = (p.nhalos + CT_WARPS - 1) / CT_WARPS;
    const uint64_t cap = (uint64_t)ctx->num_sms * (uint64_t)per_sm;
    const unsigned grid = (unsigned)(want < cap ? want : cap);
    kern<<<grid, CT_THREADS, smem, s>>>(p);
    SJCS_LAUNCH_CHECK();
    return SJCS_OK;
}

template <int BIN, bool BIG>
int launch_queue(sjcs_ctx* ctx, const CountParams& p, const Schedule& sc, size_t smem, cudaStream_t s) {
    const uint64_t n = p.nhalos;
    if (n * (uint64_t)sc.max_pieces >= (1ull << 32))
        return fail(SJCS_ERR_INVALID, "queue schedule: nhalos * max_pieces must stay below 2^32");
    const uint32_t ntiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
    StreamScratch scr(s);  // freed (stream-ordered) after the kernels below
    uint32_t *key, *ord, *ctl, *hist, *rhist;
    BucketPlan* plan;
    SJCS_CUDA_TRY(scr.alloc(&key, n * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&ord, n * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&ctl, 4 * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&hist, kBuckets * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&plan, kBuckets * sizeof(BucketPlan)));
    SJCS_CUDA_TRY(scr.alloc(&rhist, (uint64_t)RS_BINS * ntiles * sizeof(uint32_t)));
    SJCS_CUDA_TRY(cudaMemsetAsync(hist, 0, kBuckets * sizeof(uint32_t), s));
    k_estimate<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(p, key, hist);
    SJCS_LAUNCH_CHECK();
    int rc = order_and_plan(n, key, hist, sc, ord, plan, ctl, rhist, s);
    if (rc) return rc;
    auto kern = k_shell_count_queue<BIN, BIG>;
    if (smem > 48 * 1024)
        SJCS_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    SJCS_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, CT_THREADS, smem));
    if (per_sm < 1) per_sm = 1;
    kern<<<(unsigned)(ctx->num_sms * per_sm), CT_THREADS, smem, s>>>(p, QueueParams{ord, plan, ctl});
    SJCS_LAUNCH_CHECK();
    return SJCS_OK;
}

}  // namespace

namespace {

// Kernel parameters of a count of q against an index of geometry g.
CountParams count_params(const sjcs_query* q, const sjcs_index* idx) {
    CountParams p{};
    p.pts = idx->pts;
    p.cs = idx->cell_start;
    p.g = idx->geom;
    for (int a = 0; a < 3; ++a) p.h[a] = 1000.0f / (float)idx->geom.G[a];
    p.halos = q->halos;
    p.nhalos = q->nhalos;
    p.r2 = q->d_r2;
    p.lut = q->d_lut;
    p.nrads = q->nrads;
    p.pad = q->pad;
    p.nlut = q->nlut;
    p.lut_k0 = q->lut_k0;
    p.lut_shift = q->lut_shift;
    p.half = q->half;
    p.r2max = q->r2max;
    p.r2p = q->r2max * (1.0f + 1e-5f);
    p.r2slack = q->r2max * 1e-5f;
    p.periodic = (q->flags & SJCS_QUERY_PERIODIC) ? 1 : 0;
    p.prune = q->monotone && std::isfinite(q->r2max) ? 1 : 0;
    p.counts = q->counts;
    p.nidx = 1;
    p.mpts[0] = idx->pts;
    p.mcs[0] = idx->cell_start;
    return p;
}

int bin_mode(const sjcs_query* q) { return !q->monotone ? BIN_FIRST_MATCH : (q->nlut > 0 ? BIN_LUT : BIN_BSEARCH); }
bool big_tables(const sjcs_query* q) { return q->pad > kMaxSmemTable || q->nrads > kMaxSmemRads; }
size_t count_smem(const sjcs_query* q) {
    return CT_WARPS * sizeof(WarpPlans) +
           (big_tables(q) ? 0 : (size_t)(q->pad + q->nlut + CT_WARPS * q->nrads) * sizeof(uint32_t));
}

int launch_static(sjcs_ctx* ctx, const CountParams& p, int bin, bool big, size_t smem, cudaStream_t s, bool multi) {
    switch (bin) {
        case BIN_LUT:
            return big ? launch_variant<BIN_LUT, true>(ctx, p, smem, s, multi)
                       : launch_variant<BIN_LUT, false>(ctx, p, smem, s, multi);
        case BIN_BSEARCH:
            return big ? launch_variant<BIN_BSEARCH, true>(ctx, p, smem, s, multi)
                       : launch_variant<BIN_BSEARCH, false>(ctx, p, smem, s, multi);
        default:
            return big ? launch_variant<BIN_FIRST_MATCH, true>(ctx, p, smem, s, multi)
                       : launch_variant<BIN_FIRST_MATCH, false>(ctx, p, smem, s, multi);
    }
}

}  // namespace

int launch_shell_count(sjcs_ctx* ctx, const sjcs_query* q, const sjcs_index* idx, cudaStream_t s,
                       const Schedule* sc) {
    if (q->nhalos == 0 || idx->n == 0) return SJCS_OK;
    const CountParams p = count_params(q, idx);
    const int bin = bin_mode(q);
    const bool big = big_tables(q);
    const size_t smem = count_smem(q);
    if (sc && sc->mode == SJCS_SCHED_QUEUE) {
        switch (bin) {
            case BIN_LUT:
                return big ? launch_queue<BIN_LUT, true>(ctx, p, *sc, smem, s)
                           : launch_queue<BIN_LUT, false>(ctx, p, *sc, smem, s);
            case BIN_BSEARCH:
                return big ? launch_queue<BIN_BSEARCH, true>(ctx, p, *sc, smem, s)
                           : launch_queue<BIN_BSEARCH, false>(ctx, p, *sc, smem, s);
            default:
                return big ? launch_queue<BIN_FIRST_MATCH, true>(ctx, p, *sc, smem, s)
                           : launch_queue<BIN_FIRST_MATCH, false>(ctx, p, *sc, smem, s);
        }
    }
    return launch_static(ctx, p, bin, big, smem, s, false);
}

int launch_shell_count_multi(sjcs_ctx* ctx, const sjcs_query* q, const sjcs_index* const* idx, int k,
                             cudaStream_t s) {
    if (k < 1 || k > kMaxFused) return fail(SJCS_ERR_INVALID, "between 1 and %d indexes per fused count", kMaxFused);
    CountParams p = count_params(q, idx[0]);
    p.nidx = 0;
    for (int i = 0; i < k; ++i) {
        if (idx[i]->n == 0) continue;  // adds nothing
        p.mpts[p.nidx] = idx[i]->pts;
        p.mcs[p.nidx] = idx[i]->cell_start;
        ++p.nidx;
    }
    if (q->nhalos == 0 || p.nidx == 0) return SJCS_OK;
    return launch_static(ctx, p, bin_mode(q), big_tables(q), count_smem(q), s, true);
}

}  // namespace sjcs
