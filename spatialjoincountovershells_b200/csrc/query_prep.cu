// Halo preparation: order the halos along a 30-bit Morton curve so that the
// warps resident at any moment search neighbouring halos and share particle
// lines in L1/L2.  The order changes nothing in the counts (each halo's counts
// go back to its own row); the reference walks halos in file order in chunks
// of 100 (threadJoin, src/astr_rcount/main.c:802-823).
#include "radix_sort.cuh"
#include "sjcs_internal.cuh"

namespace sjcs {
namespace {

__device__ __forceinline__ float3 load_halo(const char* base, size_t stride, uint64_t i) {
    const float* p = reinterpret_cast<const float*>(base + i * stride);
    return make_float3(p[0], p[1], p[2]);
}

struct KeysFromHalos {
    const char* __restrict__ base;
    size_t stride;
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const {
        const float3 h = load_halo(base, stride, i);
        return morton30(h.x, h.y, h.z);
    }
};

struct SinkHalos {
    const char* __restrict__ base;
    size_t stride;
    float4* __restrict__ out;
    __device__ __forceinline__ void operator()(uint32_t g, uint32_t, uint32_t v) const {
        const float3 h = load_halo(base, stride, v);
        out[g] = make_float4(h.x, h.y, h.z, __uint_as_float(v));
    }
};

}  // namespace

int sort_halos(sjcs_ctx* ctx, const float* d_halo_xyz, size_t stride_bytes, uint64_t nhalos,
               float4* out, cudaStream_t s) {
    (void)ctx;
    if (nhalos == 0) return SJCS_OK;
    const char* base = reinterpret_cast<const char*>(d_halo_xyz);
    const uint32_t ntiles = (uint32_t)((nhalos + RS_TILE - 1) / RS_TILE);
    uint32_t *ka, *kb, *va, *vb, *hist;
    StreamScratch scr(s);
    SJCS_CUDA_TRY(scr.alloc(&ka, nhalos * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&kb, nhalos * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&va, nhalos * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&vb, nhalos * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&hist, (uint64_t)RS_BINS * ntiles * sizeof(uint32_t)));
    const KeysFromHalos kh{base, stride_bytes};
    const int passes = 4;  // 30-bit keys
    uint32_t *kin = nullptr, *vin = nullptr, *kout = ka, *vout = va;
    for (int p = 0; p < passes; ++p) {
        const int shift = p * RS_BITS;
        const bool first = (p == 0), last = (p == passes - 1);
        if (first)
            k_radix_upsweep<<<ntiles, RS_THREADS, 0, s>>>(kh, nhalos, shift, hist, ntiles);
        else
            k_radix_upsweep<<<ntiles, RS_THREADS, 0, s>>>(KeysFromArray{kin}, nhalos, shift, hist, ntiles);
        SJCS_LAUNCH_CHECK();
        int rc = exclusive_scan_u32(hist, (uint64_t)RS_BINS * ntiles, s);
        if (rc) return rc;
        if (last) {
            const SinkHalos sink{base, stride_bytes, out};
            k_radix_downsweep<<<ntiles, RS_THREADS, 0, s>>>(KeysFromArray{kin}, ValsFromArray{vin}, nhalos,
                                                             shift, hist, ntiles, sink);
        } else {
            const SinkPairs sink{kout, vout};
            if (first)
                k_radix_downsweep<<<ntiles, RS_THREADS, 0, s>>>(kh, ValsIota{}, nhalos, shift, hist, ntiles,
                                                                 sink);
            else
                k_radix_downsweep<<<ntiles, RS_THREADS, 0, s>>>(KeysFromArray{kin}, ValsFromArray{vin}, nhalos,
                                                                 shift, hist, ntiles, sink);
        }
        SJCS_LAUNCH_CHECK();
        kin = kout;
        vin = vout;
        kout = (kout == ka) ? kb : ka;
        vout = (vout == va) ? vb : va;
    }
    return SJCS_OK;
}

}  // namespace sjcs
