/*
 * sjcs_oracle.h -- CPU restatement of the reference's periodic multi-shell
 * count, used ONLY as test infrastructure: the checker in tests/, in
 * __graft_entry__.smoke(), and the "port" CPU baseline in bench.py.  Nothing
 * in the product links or calls it.
 *
 * Pinned against (a) the periodic known-answer fixture of the reference
 * (TestData4PB: 8 corner particles, 2 corner halos, counts 1/3/3/1 per halo)
 * and (b) outputs of the reference program itself built from its own sources
 * into oracle/_ref/ (tests/golden/ holds the vectors and the script that
 * made them).
 */
#ifndef SJCS_ORACLE_H
#define SJCS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Logspace(2, log2(min), log2(max), n) then r[i] *= r[i] in fp32
 * (include/support_functions.h:18-34, src/astr_rcount/main.c:646-649).
 * use_fma selects the contracted form a + i*c -> fma(i, c, a) that gcc emits
 * for the reference's -march=native build on an FMA-capable host. */
int oracle_radius_table(double minrad, double maxrad, int nrads, int use_fma, float *r2);

/* counts[h*nrads + i] += particles of shell i around halo h.
 * particles: np x,y,z triplets.  halos: x of halo h at (char*)halo_xyz + h*stride.
 * periodic != 0 follows multiRangeCountWithPriodicBoundArraySTR
 * (src/objects/ArraySTR/MultiRangeCount.c:13-73), periodic == 0 follows
 * multiRangeCountArraySTR (:75-83).  Candidates come from a CPU cell grid;
 * the acceptance test is the reference's, literally.  nthreads <= 0: all cores. */
int oracle_count(const float *particles, uint64_t np, const float *halo_xyz, size_t stride,
                 uint64_t nhalos, const float *r2, int nrads, int periodic, uint64_t *counts,
                 int nthreads);

/* Same result, every particle tested against every image (tiny inputs only). */
/* Decode n compressed particles (uint16 triplets, ids id_start + i) with the
 * 256-byte Gadget header, restating decodeCompressedParticle
 * (src/Gadget/BufVector3D.c:169-201), id2posGadId (src/Gadget/GadId.c:38-54,
 * 80-146) and initGadgetDecodeParams (src/Gadget/GadgetHeader.c:9-24), in the
 * contracted form the reference's -march build computes.  Returns 0 or -1. */
int oracle_decode_compressed(const void *header, const uint16_t *uv, uint64_t n, float *xyz);

int oracle_count_brute(const float *particles, uint64_t np, const float *halo_xyz, size_t stride,
                       uint64_t nhalos, const float *r2, int nrads, int periodic, uint64_t *counts);

#ifdef __cplusplus
}
#endif

#endif
