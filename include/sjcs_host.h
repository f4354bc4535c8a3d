/*
 * sjcs_host.h -- host-side C ABI of libsjcs_host.so: the file formats and
 * data generators around the GPU hot path.  Everything here runs on the CPU
 * and needs no GPU; the astr_rcount-compatible driver (sjcs_rcount) and the
 * Python tests/benchmark use it.
 *
 * Formats are the reference's:
 *   particle file  headerless float32 x,y,z triplets; count = size / 12
 *                  (readDecodedParticles, src/Gadget/BufVector3D.c:285-308)
 *   halo file      16 header lines, then one text record per line: id = first
 *                  token (strtoul), mass = 3rd token, x y z = 9th..11th
 *                  tokens (strtof), single-space separated
 *                  (readHalos + GetDataFromLineFast, src/Gadget/BufHalo.c:76-119, 218-249)
 *   filter file    one id per line (strtol), merge-joined against halo ids
 *                  (readAndFilterHalos, src/Gadget/BufHalo.c:121-214)
 *   result text    outputResult, src/astr_rcount/main.c:371-442
 */
#ifndef SJCS_HOST_H
#define SJCS_HOST_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as the reference's Halo (include/Gadget/BufHalo.h:26-30): 24 bytes. */
typedef struct sjcs_halo {
    uint64_t id;
    float mass;
    float point[3];
} sjcs_halo;

/* ---- particle files ------------------------------------------------------- */

/* Number of particles in a decoded particle file (file size / 12), or -1 with
 * errno-style message when the file cannot be opened (GetFileSize,
 * src/Gadget/BufVector3D.c:391-400). */
int sjcs_particle_file_count(const char *path, uint64_t *n);
/* Read up to cap particles (n*3 floats) into buf; *n receives the count.
 * buf may be pinned memory from sjcs_host_alloc. */
int sjcs_read_particles(const char *path, float *buf, uint64_t cap, uint64_t *n);

/* ---- halo files ----------------------------------------------------------- */

/* Parse a halo file.  *out is malloc'd (free with sjcs_host_free_halos).
 * Same acceptance as the reference: 16 header lines must be present, a last
 * line without a newline is ignored, a record missing a field is an error.
 * nthreads <= 0: one thread per core (the result does not depend on it). */
int sjcs_read_halos(const char *path, sjcs_halo **out, uint64_t *n, int nthreads);
/* Keep only halos whose id appears in the filter file (same merge-join,
 * including its assumption that halo ids ascend). */
int sjcs_read_and_filter_halos(const char *path, const char *filter_path, sjcs_halo **out, uint64_t *n);
void sjcs_host_free_halos(sjcs_halo *h);
/* Message of the last failing call on this thread. */
const char *sjcs_host_last_error(void);

/* ---- result text ---------------------------------------------------------- */

/* Write the reference's result text to path (stdout if NULL): per halo
 * "id %lu" then one "  [lo ~ hi]: count" line per shell with the radii
 * (float)sqrt(r2[i]) printed with %f, then "\nTotal" and per-shell totals.
 * Totals reproduce the reference exactly, including that its running total
 * aliases halo 0's row (main.c:400), i.e. Total = sum over halos + halo 0.
 * Formatting is spread over nthreads threads; the bytes do not depend on it. */
int sjcs_write_result(const char *path, const sjcs_halo *halos, uint64_t nhalos, const float *r2, int nrads,
                      const uint64_t *counts, int nthreads);

/* ---- radius schedule (host copy of sjcs_radius_table, no CUDA needed) ---- */
int sjcs_host_radius_table(double minrad, double maxrad, int nrads, float *r2);

/* ---- data generators ------------------------------------------------------ */

/* MT19937 (Matsumoto & Nishimura 1998), seeded with init_genrand(seed). */
typedef struct sjcs_mt {
    uint32_t mt[624];
    int mti;
} sjcs_mt;
void sjcs_mt_seed(sjcs_mt *s, uint32_t seed);
uint32_t sjcs_mt_u32(sjcs_mt *s);
/* [0,1] inclusive: u32 * (1/(2^32-1)) */
double sjcs_mt_real1(sjcs_mt *s);

/* Particles exactly as uniform_decoded_particle_generator -n n -s seed
 * writes nfiles files: one MT stream, 3 x (float)(real1*1000) per particle.
 * out holds nfiles*n*3 floats, file after file. */
int sjcs_gen_uniform_particles(uint32_t seed, uint64_t nfiles, uint64_t n, float *out);
/* The halo text file uniform_halo_generator -n n -s seed writes (ids from
 * id0), byte for byte. */
int sjcs_gen_uniform_halo_file(const char *path, uint32_t seed, uint64_t n, uint64_t id0);
/* The same halos as the reference reads them back from that file (coordinates
 * and mass rounded through their printed text), without writing a file. */
int sjcs_gen_uniform_halos(uint32_t seed, uint64_t n, uint64_t id0, sjcs_halo *out, int nthreads);
/* Halos within `margin` of the box faces: each picks 1-3 axes that sit in
 * [0, margin) or (1000 - margin, 1000]; the first halos are the exact corners,
 * edge midpoints and 1000.0 cases.  Values are rounded through %f text like
 * generated halos.  Written by sjcs_write_halo_file when a file is needed. */
int sjcs_gen_face_halos(uint32_t seed, uint64_t n, uint64_t id0, float margin, sjcs_halo *out);
/* Clustered particles: nclumps isotropic Gaussian clumps (centres uniform in
 * the box, sigma log-uniform in [sig_lo, sig_hi], weights lognormal(0, wsig)
 * normalised) hold frac_clumped of the particles, the rest uniform; wrapped
 * into [0,1000).  Blocks of 2^20 particles draw from their own MT streams
 * (seeded from seed and the block number) on parallel threads. */
int sjcs_gen_clustered_particles(uint32_t seed, uint64_t n, uint32_t nclumps, double sig_lo, double sig_hi,
                                 double wsig, double frac_clumped, uint32_t clump_seed, float *out);
/* Clustered halos: frac_at_clumps of them at clump centres (same clump_seed as
 * the particles) with N(0, jitter) offsets, the rest uniform; %f-rounded. */
int sjcs_gen_clustered_halos(uint32_t seed, uint64_t n, uint64_t id0, uint32_t nclumps, double sig_lo,
                             double sig_hi, double wsig, double frac_at_clumps, double jitter,
                             uint32_t clump_seed, sjcs_halo *out);
/* Write halos in the generator's text format (16 dummy header lines). */
int sjcs_write_halo_file(const char *path, const sjcs_halo *h, uint64_t n);
/* Write particles as a decoded particle file. */
int sjcs_write_particle_file(const char *path, const float *xyz, uint64_t n);

/* ---- compressed (Gadget-encoded) particle files --------------------------
 * File: a Fortran record with the 256-byte header, then a record of
 * npart[1] x 3 uint16 displacements (readCompressedParticles,
 * src/Gadget/BufVector3D.c:110-135).  The header mirrors GadgetHeader
 * (include/Gadget/GadgetHeader.h:4-27) field for field. */
typedef struct sjcs_gadget_header {
    int       npart[6];
    double    mass[6];
    double    time;
    double    redshift;
    int       flag_sfr;
    int       flag_feedback;
    int       npartTotal[6];
    int       flag_cooling;
    int       num_files;
    double    BoxSize;
    double    Omega0;
    double    OmegaLambda;
    double    HubbleParam;
    int       flag_stellarage;
    int       flag_metals;
    int       hashsize;
    float     disp_min;
    float     disp_max;
    int       pos_bits;
    long long id_start;
    long long id_end;
    char      fill[56];
} sjcs_gadget_header;
/* Header only (readCompressedParticlesHeader, BufVector3D.c:90-108). */
int sjcs_read_compressed_header(const char *path, sjcs_gadget_header *hdr);
/* Header and the npart[1] uint16 triplets into uv (room for cap triplets). */
int sjcs_read_compressed_particles(const char *path, sjcs_gadget_header *hdr, uint16_t *uv, uint64_t cap,
                                   uint64_t *n);
int sjcs_write_compressed_file(const char *path, const sjcs_gadget_header *hdr, const uint16_t *uv, uint64_t n);
/* Synthetic compressed data (no real Gadget files are available): a lattice
 * of n1d^3 particles (ids id_start ..), box `box`, displacements uniform in
 * [0, 2^pos_bits) between disp_min and disp_max (MT19937 `seed`).  Fills hdr
 * and the first n triplets (n <= n1d^3). */
int sjcs_gen_compressed(uint32_t seed, int n1d, double box, float disp_min, float disp_max, int pos_bits,
                        long long id_start, uint64_t n, sjcs_gadget_header *hdr, uint16_t *uv);

#ifdef __cplusplus
}
#endif

#endif
