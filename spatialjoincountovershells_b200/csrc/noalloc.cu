// sjcs_count_noalloc: one particle file's shell counts for small inputs with
// no device allocation at all.
//
// Some callers cannot let a library call cudaMalloc: a host program whose
// framework has already reserved the GPU's memory for its own caching
// allocator (a library cudaMalloc then fails or fragments that pool), or a
// latency-critical loop that cannot absorb the device-wide synchronisation a
// cudaMalloc/cudaFree may imply.  For them this entry point builds the grid
// index and counts shells using only a fixed scratch area that lives in a
// file-scope __device__ array (SJCS_NOALLOC_SCRATCH_BYTES, about 9.3 MB),
// plus the caller's own input and output buffers.
//
// Every GPU that loads this library's module holds that array until the
// process exits.  With lazy module loading (the CUDA default since 12.2) the
// module, and with it the array, is loaded on a device by the first call made
// while that device is current -- its cudaGetSymbolAddress -- so that first
// call is when the driver sets the 9.3 MB aside: make it before a framework
// reserves the device's memory, or set CUDA_MODULE_LOADING=EAGER to load it
// with the library.  Make that first call before any stream capture too.
// All calls share the array and it keeps the last call's contents, so calls
// that overlap on the GPU (two streams, two host threads) race and must be
// serialised by the caller; the only state that must start at zero (the
// cell-table gap counter) is cleared by each call.
#include <cmath>
#include <cstring>
#include <mutex>

#include "radix_sort.cuh"
#include "sjcs_internal.cuh"

namespace sjcs {
namespace {

constexpr uint64_t kNP = SJCS_NOALLOC_MAX_PARTICLES;
constexpr uint64_t kNH = SJCS_NOALLOC_MAX_HALOS;
constexpr uint64_t kNC = SJCS_NOALLOC_MAX_CELLS;
constexpr int kNR = SJCS_NOALLOC_MAX_SHELLS;

constexpr uint64_t align256(uint64_t x) { return (x + 255) & ~uint64_t(255); }
constexpr uint64_t kTiles = (kNP + RS_TILE - 1) / RS_TILE;
// byte offsets of the sub-buffers (each 256-byte aligned)
constexpr uint64_t kOffPts = 0;
constexpr uint64_t kOffCells = align256(kOffPts + kNP * 16);
constexpr uint64_t kOffKFinal = align256(kOffCells + (kNC + 1) * 4);
constexpr uint64_t kOffKX = align256(kOffKFinal + kNP * 4);
constexpr uint64_t kOffKY = align256(kOffKX + kNP * 4);
constexpr uint64_t kOffPX = align256(kOffKY + kNP * 4);
constexpr uint64_t kOffPY = align256(kOffPX + kNP * 16);
constexpr uint64_t kOffHist = align256(kOffPY + kNP * 16);
constexpr uint64_t kOffPartials = align256(kOffHist + (uint64_t)RS_BINS * kTiles * 4);
constexpr uint64_t kOffGaps = align256(kOffPartials + 256 * 4);
constexpr uint64_t kOffNGaps = align256(kOffGaps + (uint64_t)kGridGaps * 12);
constexpr uint64_t kOffHalos = align256(kOffNGaps + 4);
constexpr uint64_t kOffR2 = align256(kOffHalos + kNH * 16);
constexpr uint64_t kScratchBytes = align256(kOffR2 + (uint64_t)kNR * 4);
static_assert(kScratchBytes == SJCS_NOALLOC_SCRATCH_BYTES, "keep the header's scratch size in step");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices];

// Device address of the scratch array on the current device (set up once).
int scratch_address(unsigned char** out) {
    int dev = 0;
    SJCS_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fail(SJCS_ERR_INVALID, "device %d beyond the supported %d", dev, kMaxDevices);
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(SJCS_ERR_CUDA, "cudaGetSymbolAddress of the scratch array failed on device %d: %s", dev,
                        cudaGetErrorString(e));
        g_scratch_addr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_scratch_addr[dev]);
    return SJCS_OK;
}

// The padded radius table travels as a kernel argument (copied at launch),
// so no host buffer has to outlive the call.
struct R2Table {
    float v[kNR];
};
__global__ void k_put_r2(R2Table t, int pad, float* __restrict__ out) {
    for (int i = threadIdx.x; i < pad; i += blockDim.x) out[i] = t.v[i];
}

__global__ void k_pack_halos(const char* __restrict__ base, size_t stride, uint64_t nh, float4* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nh) return;
    const float* p = reinterpret_cast<const float*>(base + i * stride);
    out[i] = make_float4(p[0], p[1], p[2], __uint_as_float((uint32_t)i));
}

}  // namespace
}  // namespace sjcs

using namespace sjcs;

extern "C" int sjcs_count_noalloc(const float* d_xyz, uint64_t n, const float* d_halo_xyz, size_t stride_bytes,
                                  uint64_t nhalos, const float* r2, int nrads, int flags, uint32_t* d_counts,
                                  void* stream) {
    if (n > kNP)
        return fail(SJCS_ERR_INVALID, "sjcs_count_noalloc: %llu particles exceed its limit of %llu",
                    (unsigned long long)n, (unsigned long long)kNP);
    if (nhalos > kNH)
        return fail(SJCS_ERR_INVALID, "sjcs_count_noalloc: %llu halos exceed its limit of %llu",
                    (unsigned long long)nhalos, (unsigned long long)kNH);
    if (nrads < 1 || nrads > kNR)
        return fail(SJCS_ERR_INVALID, "sjcs_count_noalloc: %d shells outside its limit of 1..%d", nrads, kNR);
    if (!r2) return fail(SJCS_ERR_INVALID, "sjcs_count_noalloc: r2 is NULL");
    if ((n && !d_xyz) || (nhalos && (!d_halo_xyz || !d_counts)))
        return fail(SJCS_ERR_INVALID, "sjcs_count_noalloc: NULL input or output pointer");
    if (stride_bytes < 3 * sizeof(float) || stride_bytes % sizeof(float))
        return fail(SJCS_ERR_INVALID, "sjcs_count_noalloc: stride_bytes must be a multiple of 4 and >= 12");
    if (flags & ~SJCS_QUERY_PERIODIC) return fail(SJCS_ERR_INVALID, "sjcs_count_noalloc: unknown flags 0x%x", flags);
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    unsigned char* base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;

    // radius table, as sjcs_query_create builds it (binary-search binning),
    // written by a kernel that receives it by value
    R2Table tab;
    int pad = 1;
    while (pad < nrads) pad <<= 1;
    bool mono = true;
    for (int i = 0; i < pad; ++i) tab.v[i] = i < nrads ? r2[i] : INFINITY;
    for (int i = 0; i < nrads; ++i) {
        if (std::isnan(r2[i])) mono = false;
        if (i + 1 < nrads && !(r2[i] <= r2[i + 1])) mono = false;
    }
    float* d_r2 = reinterpret_cast<float*>(base + kOffR2);
    k_put_r2<<<1, kNR, 0, s>>>(tab, pad, d_r2);
    SJCS_LAUNCH_CHECK();

    // the grid index, in the scratch array
    const float R = (float)std::sqrt((double)r2[nrads - 1]);
    GridGeom g = auto_grid(n, std::isfinite(R) ? R : 0.0f, nullptr);
    while (g.ncells > kNC) {
        int G[3] = {std::max(1, g.G[0] * 7 / 8), std::max(1, g.G[1] * 7 / 8), std::max(1, g.G[2] * 7 / 8)};
        for (int a = 0; a < 3; ++a) {
            g.G[a] = G[a];
            g.inv_h[a] = (float)G[a] / 1000.0f;
        }
        g.ncells = (uint64_t)G[0] * G[1] * G[2];
    }
    GridBuildBuffers b{};
    b.pts = reinterpret_cast<float4*>(base + kOffPts);
    b.cell_start = reinterpret_cast<uint32_t*>(base + kOffCells);
    b.kfinal = reinterpret_cast<uint32_t*>(base + kOffKFinal);
    b.kx = reinterpret_cast<uint32_t*>(base + kOffKX);
    b.ky = reinterpret_cast<uint32_t*>(base + kOffKY);
    b.px = reinterpret_cast<uint4*>(base + kOffPX);
    b.py = reinterpret_cast<uint4*>(base + kOffPY);
    b.hist = reinterpret_cast<uint32_t*>(base + kOffHist);
    b.partials = reinterpret_cast<uint32_t*>(base + kOffPartials);
    b.gaps = base + kOffGaps;
    b.ngaps = reinterpret_cast<uint32_t*>(base + kOffNGaps);
    rc = build_grid_into(d_xyz, n, g, b, s);
    if (rc) return rc;

    // halos in the caller's order (no sort: inputs are small)
    float4* halos = reinterpret_cast<float4*>(base + kOffHalos);
    if (nhalos) {
        k_pack_halos<<<(unsigned)((nhalos + 255) / 256), 256, 0, s>>>(reinterpret_cast<const char*>(d_halo_xyz),
                                                                       stride_bytes, nhalos, halos);
        SJCS_LAUNCH_CHECK();
    }

    // count through the regular kernel, on objects that only point at the scratch
    sjcs_ctx c;
    c.magic = kCtxMagic;
    SJCS_CUDA_TRY(cudaGetDevice(&c.device));
    SJCS_CUDA_TRY(cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, c.device));
    sjcs_index idx{};
    idx.n = n;
    idx.geom = g;
    idx.pts = b.pts;
    idx.cell_start = b.cell_start;
    sjcs_query q{};
    q.nhalos = nhalos;
    q.nrads = nrads;
    q.flags = flags;
    q.pad = pad;
    q.monotone = mono;
    q.r2max = r2[nrads - 1];
    q.R = R;
    q.half = (flags & SJCS_QUERY_PERIODIC) ? R : r2[nrads - 1];
    q.halos = halos;
    q.counts = d_counts;
    q.d_r2 = d_r2;
    q.d_lut = nullptr;
    q.nlut = 0;
    return launch_shell_count(&c, &q, &idx, s);
}
