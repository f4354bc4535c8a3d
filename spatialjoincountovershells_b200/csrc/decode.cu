// Compressed (Gadget-encoded) particles: decode on the device.
//
// A compressed file stores, per particle, three uint16 displacements from the
// particle's lattice cell; the cell comes from the particle id
// (id = file index + id_start).  The reference decodes on the host
// (decodeCompressedParticle, src/Gadget/BufVector3D.c:169-201, with
// id2posGadId, src/Gadget/GadId.c:38-54, and the parameters of
// initGadgetDecodeParams, src/Gadget/GadgetHeader.c:9-24); the index build
// then sees plain x,y,z floats.  Here the triplets are copied to the device
// (6 bytes per particle instead of 12) and decoded there, with the
// reference's integer types and its arithmetic as its build compiles it:
//   f   = fmaf(cell_interval, (float)ip, disp_min)           (float, contracted)
//   pos = (float)fma(unitsep, (double)displacement, (double)f)
// (the compiled reference matches this form on every tested input; see the
// oracle's restatement and the golden decode vectors).
#include <cmath>
#include <cstring>

#include "sjcs_internal.cuh"

namespace sjcs {
namespace {

// The 256-byte header, field for field (include/Gadget/GadgetHeader.h:4-27).
struct GadgetHeaderBytes {
    int npart[6];
    double mass[6];
    double time;
    double redshift;
    int flag_sfr;
    int flag_feedback;
    int npartTotal[6];
    int flag_cooling;
    int num_files;
    double BoxSize;
    double Omega0;
    double OmegaLambda;
    double HubbleParam;
    int flag_stellarage;
    int flag_metals;
    int hashsize;
    float disp_min;
    float disp_max;
    int pos_bits;
    long long id_start;
    long long id_end;
    char fill[56];
};
static_assert(sizeof(GadgetHeaderBytes) == 256, "Gadget header is 256 bytes");

__global__ void k_decode(const uint16_t* __restrict__ uv, uint64_t n, GadgetDecode g, float* __restrict__ xyz) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        // id2posGadId with the reference's types (long long ids, int indices)
        const long long ID = (long long)((unsigned long long)i + (unsigned long long)g.id_start);
        const long long IDt = (ID - 1) / g.ng3d;
        const long long IDg = ID - 1 - IDt * g.ng3d;
        const int ig = (int)(IDg / g.ng2d);
        const int jg = (int)((IDg - ig * g.ng2d) / g.ng1d);
        const int kg = (int)(IDg - ig * g.ng2d - jg * g.ng1d);
        const int it = (int)(IDt / g.nt2d);
        const int jt = (int)((IDt - it * g.nt2d) / g.nt1d);
        const int kt = (int)(IDt - it * g.nt2d - jt * g.nt1d);
        const int ip[3] = {(int)(it * g.ng1d + ig), (int)(jt * g.ng1d + jg), (int)(kt * g.ng1d + kg)};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float f = __fmaf_rn(g.cell_interval, __int2float_rn(ip[a]), g.disp_min);
            const double d = __fma_rn(g.unitsep, (double)uv[3 * i + a], (double)f);
            xyz[3 * i + a] = __double2float_rn(d);
        }
    }
}

}  // namespace

int gadget_decode_params(const void* header, GadgetDecode* out) {
    if (!header || !out) return fail(SJCS_ERR_INVALID, "Gadget header is NULL");
    GadgetHeaderBytes h;
    std::memcpy(&h, header, sizeof(h));
    // initGadgetDecodeParams with one tile (src/astr_rcount/main.c:744)
    const long long total = (long long)h.npartTotal[1] + ((long long)h.npartTotal[2] << 32);
    const int n1d = (int)std::pow((double)total + 0.5, 1 / 3.);
    if (n1d <= 0) return fail(SJCS_ERR_INVALID, "Gadget header: no particles in npartTotal");
    if (h.pos_bits < 0 || h.pos_bits > 62) return fail(SJCS_ERR_INVALID, "Gadget header: pos_bits %d", h.pos_bits);
    GadgetDecode g{};
    g.cell_interval = (float)(h.BoxSize / (double)n1d);
    const float span = h.disp_max - h.disp_min;  // float subtraction, as the reference
    g.unitsep = (double)span / std::pow(2.0, (double)h.pos_bits);
    g.disp_min = h.disp_min;
    g.id_start = h.id_start;
    // initGadId(gi, 1, n1d) (src/Gadget/GadId.c:28-35): Ng2D is an int product
    g.nt1d = 1;
    g.nt2d = 1;
    g.ng1d = n1d;
    g.ng2d = (long long)(int)((unsigned)n1d * (unsigned)n1d);
    g.ng3d = (long long)n1d * (long long)n1d * (long long)n1d;
    if (g.ng2d <= 0) return fail(SJCS_ERR_INVALID, "Gadget header: lattice of %d per axis is too large", n1d);
    *out = g;
    return SJCS_OK;
}

int launch_decode(const uint16_t* d_uv, uint64_t n, const GadgetDecode& g, float* d_xyz, cudaStream_t s) {
    if (n == 0) return SJCS_OK;
    const uint64_t want = (n + 255) / 256;
    const unsigned blocks = (unsigned)(want < 148ull * 32 ? want : 148ull * 32);
    k_decode<<<blocks, 256, 0, s>>>(d_uv, n, g, d_xyz);
    SJCS_LAUNCH_CHECK();
    return SJCS_OK;
}

}  // namespace sjcs
