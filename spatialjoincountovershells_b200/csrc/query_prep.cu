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

// payload: x, y, z and the halo's index in the caller's order
struct PayFromHalos {
    const char* __restrict__ base;
    size_t stride;
    __device__ __forceinline__ uint4 operator()(uint64_t i) const {
        const float3 h = load_halo(base, stride, i);
        return make_uint4(__float_as_uint(h.x), __float_as_uint(h.y), __float_as_uint(h.z), (uint32_t)i);
    }
};

struct SinkHalos {
    uint4* __restrict__ out;
    __device__ __forceinline__ void operator()(uint32_t g, uint32_t, const uint4& v) const { out[g] = v; }
};

}  // namespace

int sort_halos(sjcs_ctx* ctx, const float* d_halo_xyz, size_t stride_bytes, uint64_t nhalos,
               float4* out, cudaStream_t s) {
    (void)ctx;
    if (nhalos == 0) return SJCS_OK;
    const char* base = reinterpret_cast<const char*>(d_halo_xyz);
    const uint64_t ntiles = (nhalos + RS_TILE - 1) / RS_TILE;
    uint32_t *kx, *ky, *hist;
    uint4 *px, *py;
    StreamScratch scr(s);
    SJCS_CUDA_TRY(scr.alloc(&kx, nhalos * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&ky, nhalos * sizeof(uint32_t)));
    SJCS_CUDA_TRY(scr.alloc(&px, nhalos * sizeof(uint4)));
    SJCS_CUDA_TRY(scr.alloc(&py, nhalos * sizeof(uint4)));
    SJCS_CUDA_TRY(scr.alloc(&hist, (uint64_t)RS_BINS * ntiles * sizeof(uint32_t)));
    return radix_sort_records(nhalos, 30, KeysFromHalos{base, stride_bytes}, PayFromHalos{base, stride_bytes},
                              SinkHalos{reinterpret_cast<uint4*>(out)}, kx, px, ky, py, hist, s);
}

}  // namespace sjcs
