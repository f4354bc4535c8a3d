// Device code shared by the shell-count kernels (grid rows and Morton cells):
// the kernel parameters, the exact acceptance test and shell binning, and the
// flattening of per-lane slot ranges into coalesced candidate windows.
// The arithmetic contract is documented in shell_count.cu.
#pragma once

#include "sjcs_internal.cuh"

namespace sjcs {
namespace count {

enum BinMode { BIN_LUT = 0, BIN_BSEARCH = 1, BIN_FIRST_MATCH = 2 };
constexpr int kMaxFused = kMaxFusedIndexes;  // indexes counted in one pass by k_shell_count_multi

struct CountParams {
    const float4* __restrict__ pts;  // particles grouped by cell (x, y, z; .w not read)
    const uint32_t* __restrict__ cs;
    GridGeom g;
    float h[3];                      // cell edge per axis, 1000 / G
    const float4* __restrict__ halos;
    uint64_t nhalos;
    const float* __restrict__ r2;    // [pad], +inf past nrads
    const uint32_t* __restrict__ lut;
    int nrads;
    int pad;
    int nlut;
    uint32_t lut_k0;                 // bit pattern of r2[0]
    int lut_shift;
    float half;
    float r2max;
    float r2p;                       // r2max * (1 + 1e-5)
    float r2slack;                   // r2max * 1e-5
    int periodic;
    int prune;
    uint32_t* __restrict__ counts;
    // several indexes of one grid counted in one pass (k_shell_count_multi)
    int nidx;
    const float4* mpts[kMaxFused];
    const uint32_t* mcs[kMaxFused];
};

__device__ __forceinline__ float edge_margin(float v) { return 1e-3f + 2e-6f * fabsf(v); }

// Lower bound of |c - y| over every y whose cell index is k.
__device__ __forceinline__ float cell_gap(float c, int k, float h, int G) {
    const float lo_e = (float)k * h, hi_e = (float)(k + 1) * h;
    const float lo = (k == 0) ? -INFINITY : lo_e - edge_margin(lo_e);
    const float hi = (k == G - 1) ? INFINITY : hi_e + edge_margin(hi_e);
    return fmaxf(0.0f, fmaxf(lo - c, c - hi));
}

template <int BIN>
__device__ __forceinline__ int bin_of(const CountParams& p, const float* __restrict__ tab,
                                      const uint32_t* __restrict__ lut, float dist) {
    if (BIN == BIN_LUT) {
        const uint32_t key = __float_as_uint(dist);
        if (key < p.lut_k0) return 0;
        const int s = (int)lut[(key - p.lut_k0) >> p.lut_shift];
        return s + ((tab[s] <= dist) ? 1 : 0);
    } else {
        int s = 0;
        for (int step = p.pad >> 1; step > 0; step >>= 1) s += (tab[s + step - 1] <= dist) ? step : 0;
        return s;
    }
}

// Image set-up: the query box, its cell range and the clipping constants.
struct Image {
    float cx, cy, cz;
    float lox, hix, loy, hiy, loz, hiz;
    int x0, x1, y0, y1, z0, z1;
    int ny, nz;
    uint32_t nrows;  // saturated at 2^31
};

__device__ __forceinline__ Image make_image(const CountParams& p, float cx, float cy, float cz) {
    Image im;
    im.cx = cx;
    im.cy = cy;
    im.cz = cz;
    im.lox = __fsub_rn(cx, p.half);
    im.hix = __fadd_rn(cx, p.half);
    im.loy = __fsub_rn(cy, p.half);
    im.hiy = __fadd_rn(cy, p.half);
    im.loz = __fsub_rn(cz, p.half);
    im.hiz = __fadd_rn(cz, p.half);
    // A NaN bound passes every particle on that side of the box test, so it
    // must open the cell range to the grid edge (cell_of maps NaN to cell 0,
    // which is right for a lower bound only).
    im.x0 = cell_of(im.lox, p.g.inv_h[0], p.g.G[0]);
    im.x1 = (im.hix != im.hix) ? p.g.G[0] - 1 : cell_of(im.hix, p.g.inv_h[0], p.g.G[0]);
    im.y0 = cell_of(im.loy, p.g.inv_h[1], p.g.G[1]);
    im.y1 = (im.hiy != im.hiy) ? p.g.G[1] - 1 : cell_of(im.hiy, p.g.inv_h[1], p.g.G[1]);
    im.z0 = cell_of(im.loz, p.g.inv_h[2], p.g.G[2]);
    im.z1 = (im.hiz != im.hiz) ? p.g.G[2] - 1 : cell_of(im.hiz, p.g.inv_h[2], p.g.G[2]);
    im.ny = im.y1 - im.y0 + 1;
    im.nz = im.z1 - im.z0 + 1;
    const uint64_t nr = (uint64_t)im.ny * (uint64_t)im.nz;
    im.nrows = nr > 0x80000000ull ? 0x80000000u : (uint32_t)nr;
    return im;
}

template <int BIN, bool BIG>
__device__ __forceinline__ void test_candidate(const CountParams& p, const Image& im, const float4 pp, bool live,
                                               uint32_t* __restrict__ sink, const float* __restrict__ tab,
                                               const uint32_t* __restrict__ lut) {
    const bool inb = !(pp.x < im.lox) & !(im.hix < pp.x) & !(pp.y < im.loy) & !(im.hiy < pp.y) &
                     !(pp.z < im.loz) & !(im.hiz < pp.z);
    const float dx = __fsub_rn(pp.x, im.cx), dy = __fsub_rn(pp.y, im.cy), dz = __fsub_rn(pp.z, im.cz);
    const float dist = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    if (BIN != BIN_FIRST_MATCH) {
        if (live && inb && dist < p.r2max) atomicAdd(sink + bin_of<BIN>(p, tab, lut, dist), 1u);
    } else if (live && inb) {
        for (int i = 0; i < p.nrads; ++i) {
            if (dist < tab[i]) {
                atomicAdd(sink + i, 1u);
                break;
            }
        }
    }
}

// Scan the lanes' row lengths and test every candidate of those rows,
// two windows of 32 candidates per iteration so two loads are in flight.
template <int BIN, bool BIG>
__device__ __forceinline__ void run_rows(const CountParams& p, const Image& im, uint32_t start, uint32_t end,
                                         uint32_t* __restrict__ sink, const float* __restrict__ tab,
                                         const uint32_t* __restrict__ lut, int lane) {
    const uint32_t len = end - start;
    uint32_t incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    const uint32_t off = start - (incl - len);  // slot = t + off for t inside this row (mod 2^32)
    for (uint32_t wb = 0; wb < total; wb += 64) {
        const uint32_t t0 = wb + (uint32_t)lane, t1 = t0 + 32u;
        // row of t = #{rows j : incl_j <= t} (empty rows are skipped naturally)
        int r0 = 0, r1 = 0;
#pragma unroll
        for (int b = 16; b >= 1; b >>= 1) {
            const uint32_t v0 = __shfl_sync(0xffffffffu, incl, r0 + b - 1);
            const uint32_t v1 = __shfl_sync(0xffffffffu, incl, r1 + b - 1);
            r0 += (v0 <= t0) ? b : 0;
            r1 += (v1 <= t1) ? b : 0;
        }
        const uint32_t o0 = __shfl_sync(0xffffffffu, off, r0);
        const uint32_t o1 = __shfl_sync(0xffffffffu, off, r1);
        const bool l0 = t0 < total, l1 = t1 < total;
        const float4 p0 = l0 ? __ldg(p.pts + (t0 + o0)) : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 p1 = l1 ? __ldg(p.pts + (t1 + o1)) : make_float4(0.f, 0.f, 0.f, 0.f);
        test_candidate<BIN, BIG>(p, im, p0, l0, sink, tab, lut);
        test_candidate<BIN, BIG>(p, im, p1, l1, sink, tab, lut);
    }
}

// Piece `part` of `nparts` of the candidates of the lanes' rows: the
// contiguous share [total*part/nparts, total*(part+1)/nparts) of the
// flattened candidate sequence, so nparts warps sharing a halo split every
// row set evenly and together test each candidate once.
template <int BIN, bool BIG>
__device__ __forceinline__ void run_rows_part(const CountParams& p, const Image& im, uint32_t start, uint32_t end,
                                              uint32_t* __restrict__ sink, const float* __restrict__ tab,
                                              const uint32_t* __restrict__ lut, int lane, uint32_t part,
                                              uint32_t nparts) {
    const uint32_t len = end - start;
    uint32_t incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    const uint32_t off = start - (incl - len);
    const uint32_t tb = (uint32_t)(((uint64_t)total * part) / nparts);
    const uint32_t te = (uint32_t)(((uint64_t)total * (part + 1u)) / nparts);
    for (uint32_t wb = tb; wb < te; wb += 64) {
        const uint32_t t0 = wb + (uint32_t)lane, t1 = t0 + 32u;
        int r0 = 0, r1 = 0;
#pragma unroll
        for (int b = 16; b >= 1; b >>= 1) {
            const uint32_t v0 = __shfl_sync(0xffffffffu, incl, r0 + b - 1);
            const uint32_t v1 = __shfl_sync(0xffffffffu, incl, r1 + b - 1);
            r0 += (v0 <= t0) ? b : 0;
            r1 += (v1 <= t1) ? b : 0;
        }
        const uint32_t o0 = __shfl_sync(0xffffffffu, off, r0);
        const uint32_t o1 = __shfl_sync(0xffffffffu, off, r1);
        const bool l0 = t0 < te, l1 = t1 < te;
        const float4 p0 = l0 ? __ldg(p.pts + (t0 + o0)) : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 p1 = l1 ? __ldg(p.pts + (t1 + o1)) : make_float4(0.f, 0.f, 0.f, 0.f);
        test_candidate<BIN, BIG>(p, im, p0, l0, sink, tab, lut);
        test_candidate<BIN, BIG>(p, im, p1, l1, sink, tab, lut);
    }
}

// Shell bucket of an estimated candidate count, for ordering work by size:
// 0 for none, else 1 + 8*floor(log2 e) + the next 3 bits of e (<= 256 values;
// neighbouring buckets differ by a factor <= 2^(1/8)).
__device__ __forceinline__ uint32_t est_bucket(uint32_t e) {
    if (e == 0) return 0u;
    const int lg = 31 - __clz(e);
    const uint32_t mant = lg >= 3 ? (e >> (lg - 3)) & 7u : (e << (3 - lg)) & 7u;
    const uint32_t b = 1u + 8u * (uint32_t)lg + mant;
    return b < 255u ? b : 255u;  // 8 bits
}

}  // namespace count
}  // namespace sjcs
