/*
 * sjcs_gen.c -- seeded synthetic inputs in the reference's formats.
 *
 * MT19937 is restated from its published description (M. Matsumoto and
 * T. Nishimura, "Mersenne Twister: a 623-dimensionally equidistributed
 * uniform pseudo-random number generator", ACM TOMACS 8(1), 1998): state of
 * 624 words, init_genrand recurrence x[i] = 1812433253*(x[i-1]^(x[i-1]>>30))+i,
 * twist with matrix 0x9908b0df, tempering (11, 7/0x9d2c5680, 15/0xefc60000, 18).
 * The reference's generators (src/uniform_decoded_particle_generator/main.c:42-68,
 * src/uniform_halo_generator/main.c:112-150) draw genrand_real1() in [0,1]
 * and scale by 1000; the uniform generators below reproduce their files
 * byte for byte.  The face-halo and clustered generators have no reference
 * counterpart: they are this project's, with the distributions of the
 * workload descriptions.
 */
#define _GNU_SOURCE
#include "../../include/sjcs_host.h"

#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define MT_N 624
#define MT_M 397

void sjcs_mt_seed(sjcs_mt *s, uint32_t seed)
{
    int i;
    s->mt[0] = seed;
    for (i = 1; i < MT_N; i++)
        s->mt[i] = 1812433253u * (s->mt[i - 1] ^ (s->mt[i - 1] >> 30)) + (uint32_t)i;
    s->mti = MT_N;
}

static void mt_twist(sjcs_mt *s)
{
    static const uint32_t mag[2] = {0u, 0x9908b0dfu};
    int k;
    uint32_t y;
    for (k = 0; k < MT_N - MT_M; k++) {
        y = (s->mt[k] & 0x80000000u) | (s->mt[k + 1] & 0x7fffffffu);
        s->mt[k] = s->mt[k + MT_M] ^ (y >> 1) ^ mag[y & 1u];
    }
    for (; k < MT_N - 1; k++) {
        y = (s->mt[k] & 0x80000000u) | (s->mt[k + 1] & 0x7fffffffu);
        s->mt[k] = s->mt[k + (MT_M - MT_N)] ^ (y >> 1) ^ mag[y & 1u];
    }
    y = (s->mt[MT_N - 1] & 0x80000000u) | (s->mt[0] & 0x7fffffffu);
    s->mt[MT_N - 1] = s->mt[MT_M - 1] ^ (y >> 1) ^ mag[y & 1u];
    s->mti = 0;
}

uint32_t sjcs_mt_u32(sjcs_mt *s)
{
    uint32_t y;
    if (s->mti >= MT_N)
        mt_twist(s);
    y = s->mt[s->mti++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

double sjcs_mt_real1(sjcs_mt *s) { return sjcs_mt_u32(s) * (1.0 / 4294967295.0); }

static double mt_real2(sjcs_mt *s) { return sjcs_mt_u32(s) * (1.0 / 4294967296.0); }

static double mt_normal(sjcs_mt *s)
{
    /* Box-Muller on (0,1] x [0,1) */
    double u1 = 1.0 - mt_real2(s), u2 = mt_real2(s);
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

int sjcs_gen_uniform_particles(uint32_t seed, uint64_t nfiles, uint64_t n, float *out)
{
    sjcs_mt s;
    uint64_t i, total = nfiles * n * 3;
    if (!out && total)
        return -1;
    sjcs_mt_seed(&s, seed);
    for (i = 0; i < total; ++i)
        out[i] = (float)(sjcs_mt_real1(&s) * (1000.0 - 0.0) + 0.0);
    return 0;
}

/* One generated halo line (src/uniform_halo_generator/main.c:136-141). */
static int halo_line(char *b, size_t cap, uint64_t id, float mass, const float pos[3])
{
    return snprintf(b, cap,
                    "%llu 0 %g 0 0 0 0 0 "
                    "%f %f %f 0 0 0 0 0 "
                    "0 0 0 0 0 0 0 0 "
                    "0 0 0 0 0 0 0 0 "
                    "0 0 0 0 0 0 0 0\n",
                    (unsigned long long)id, (double)mass, (double)pos[0], (double)pos[1], (double)pos[2]);
}

static void write_header(FILE *fp)
{
    int k;
    for (k = 0; k < 16; k++)
        fprintf(fp, "# dummy header %d\n", k);
}

int sjcs_gen_uniform_halo_file(const char *path, uint32_t seed, uint64_t n, uint64_t id0)
{
    sjcs_mt s;
    FILE *fp = fopen(path, "wb");
    uint64_t i;
    char b[512];
    if (!fp)
        return -1;
    sjcs_mt_seed(&s, seed);
    write_header(fp);
    for (i = 0; i < n; ++i) {
        float mass, pos[3];
        int a, k;
        mass = (float)(sjcs_mt_real1(&s) * (1000.0 * 1000.0) * (1000.0 * 1000.0));
        for (a = 0; a < 3; a++)
            pos[a] = (float)(sjcs_mt_real1(&s) * (1000.0 - 0.0) + 0.0);
        k = halo_line(b, sizeof(b), id0 + i, mass, pos);
        fwrite(b, 1, (size_t)k, fp);
    }
    return fclose(fp) == 0 ? 0 : -1;
}

/* Round a value through the text a halo file carries ("%f" for coordinates,
 * "%g" for the mass) and back through strtof, as the reader will see it. */
static float via_text(float v, int is_mass)
{
    char b[64];
    snprintf(b, sizeof(b), is_mass ? "%g" : "%f", (double)v);
    return strtof(b, NULL);
}

typedef struct RoundJob {
    sjcs_halo *h;
    uint64_t lo, hi;
} RoundJob;

static void *round_job(void *arg)
{
    RoundJob *j = arg;
    uint64_t i;
    for (i = j->lo; i < j->hi; ++i) {
        j->h[i].mass = via_text(j->h[i].mass, 1);
        j->h[i].point[0] = via_text(j->h[i].point[0], 0);
        j->h[i].point[1] = via_text(j->h[i].point[1], 0);
        j->h[i].point[2] = via_text(j->h[i].point[2], 0);
    }
    return NULL;
}

static void round_all(sjcs_halo *h, uint64_t n, int nthreads)
{
    RoundJob jobs[64];
    pthread_t th[64];
    int T = nthreads > 0 ? nthreads : (int)sysconf(_SC_NPROCESSORS_ONLN), t;
    if (T < 1)
        T = 1;
    if (T > 64)
        T = 64;
    if (n < 65536)
        T = 1;
    for (t = 0; t < T; ++t) {
        jobs[t].h = h;
        jobs[t].lo = n * t / T;
        jobs[t].hi = n * (t + 1) / T;
    }
    for (t = 1; t < T; ++t)
        pthread_create(&th[t], NULL, round_job, &jobs[t]);
    round_job(&jobs[0]);
    for (t = 1; t < T; ++t)
        pthread_join(th[t], NULL);
}

int sjcs_gen_uniform_halos(uint32_t seed, uint64_t n, uint64_t id0, sjcs_halo *out, int nthreads)
{
    sjcs_mt s;
    uint64_t i;
    if (!out && n)
        return -1;
    sjcs_mt_seed(&s, seed);
    for (i = 0; i < n; ++i) {
        int a;
        out[i].id = id0 + i;
        out[i].mass = (float)(sjcs_mt_real1(&s) * (1000.0 * 1000.0) * (1000.0 * 1000.0));
        for (a = 0; a < 3; a++)
            out[i].point[a] = (float)(sjcs_mt_real1(&s) * (1000.0 - 0.0) + 0.0);
    }
    round_all(out, n, nthreads);
    return 0;
}

int sjcs_gen_face_halos(uint32_t seed, uint64_t n, uint64_t id0, float margin, sjcs_halo *out)
{
    /* exact corners, edge and face points, and values at 1000.0 */
    static const float fixed[][3] = {
        {0.0f, 0.0f, 0.0f},         {1000.0f, 1000.0f, 1000.0f}, {0.0f, 1000.0f, 0.0f},
        {1000.0f, 0.0f, 1000.0f},   {0.0f, 500.0f, 500.0f},      {1000.0f, 500.0f, 500.0f},
        {500.0f, 0.0f, 1000.0f},    {999.999f, 0.000001f, 500.0f}, {0.000001f, 999.999f, 999.999f},
        {999.0f, 999.0f, 999.0f},   {5.0f, 995.0f, 500.0f},      {4.999999f, 995.000001f, 0.5f},
    };
    const uint64_t nfixed = sizeof(fixed) / sizeof(fixed[0]);
    sjcs_mt s;
    uint64_t i;
    if (!out && n)
        return -1;
    sjcs_mt_seed(&s, seed);
    for (i = 0; i < n; ++i) {
        int a;
        out[i].id = id0 + i;
        out[i].mass = (float)(sjcs_mt_real1(&s) * 1e12);
        if (i < nfixed) {
            memcpy(out[i].point, fixed[i], sizeof(out[i].point));
            continue;
        }
        {
            /* 1-3 axes near a face, each on a random side */
            int naxes = 1 + (int)(sjcs_mt_u32(&s) % 3u);
            int pick[3] = {0, 0, 0};
            int chosen = 0;
            while (chosen < naxes) {
                int ax = (int)(sjcs_mt_u32(&s) % 3u);
                if (!pick[ax]) {
                    pick[ax] = 1;
                    chosen++;
                }
            }
            for (a = 0; a < 3; a++) {
                double u = sjcs_mt_real1(&s);
                if (pick[a]) {
                    double d = u * margin;
                    out[i].point[a] = (sjcs_mt_u32(&s) & 1u) ? (float)(1000.0 - d) : (float)d;
                } else
                    out[i].point[a] = (float)(u * 1000.0);
            }
        }
    }
    round_all(out, n, 1);
    return 0;
}

typedef struct Clumps {
    uint32_t n;
    double *cx, *cy, *cz, *sig, *cdf;
} Clumps;

static int make_clumps(Clumps *c, uint32_t nclumps, double sig_lo, double sig_hi, double wsig, uint32_t seed)
{
    sjcs_mt s;
    uint32_t k;
    double tot = 0.0;
    c->n = nclumps;
    c->cx = malloc(nclumps * sizeof(double));
    c->cy = malloc(nclumps * sizeof(double));
    c->cz = malloc(nclumps * sizeof(double));
    c->sig = malloc(nclumps * sizeof(double));
    c->cdf = malloc(nclumps * sizeof(double));
    if (!c->cx || !c->cy || !c->cz || !c->sig || !c->cdf || nclumps == 0)
        return -1;
    sjcs_mt_seed(&s, seed);
    for (k = 0; k < nclumps; k++) {
        c->cx[k] = mt_real2(&s) * 1000.0;
        c->cy[k] = mt_real2(&s) * 1000.0;
        c->cz[k] = mt_real2(&s) * 1000.0;
        c->sig[k] = sig_lo * exp(mt_real2(&s) * log(sig_hi / sig_lo));
        tot += exp(wsig * mt_normal(&s));
        c->cdf[k] = tot;
    }
    for (k = 0; k < nclumps; k++)
        c->cdf[k] /= tot;
    return 0;
}

static void free_clumps(Clumps *c)
{
    free(c->cx);
    free(c->cy);
    free(c->cz);
    free(c->sig);
    free(c->cdf);
}

static uint32_t pick_clump(const Clumps *c, double u)
{
    uint32_t lo = 0, hi = c->n - 1;
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2;
        if (c->cdf[mid] < u)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

static float wrap1000(double v)
{
    v -= 1000.0 * floor(v / 1000.0);
    return (float)v;
}

/* The clustered generators draw each block of 2^20 items from its own MT19937
 * stream (seeded from the call's seed and the block number), so the blocks
 * are generated by parallel threads and the output does not depend on the
 * number of threads. */
#define GEN_BLOCK (1u << 20)

static uint32_t block_seed(uint32_t seed, uint64_t b)
{
    return seed * 2654435761u + (uint32_t)(b + 1) * 0x9e3779b9u;
}

typedef struct GenJob {
    const Clumps *c;
    uint32_t seed;
    uint64_t n, id0;
    double frac, jitter;
    float *pts;
    sjcs_halo *halos;
    uint64_t b0, b1; /* blocks of this job */
} GenJob;

static void *particle_job(void *arg)
{
    GenJob *j = arg;
    uint64_t b, i;
    for (b = j->b0; b < j->b1; ++b) {
        sjcs_mt s;
        const uint64_t lo = b * GEN_BLOCK, hi = lo + GEN_BLOCK < j->n ? lo + GEN_BLOCK : j->n;
        sjcs_mt_seed(&s, block_seed(j->seed, b));
        for (i = lo; i < hi; ++i) {
            float *p = j->pts + 3 * i;
            if (mt_real2(&s) < j->frac) {
                uint32_t k = pick_clump(j->c, mt_real2(&s));
                p[0] = wrap1000(j->c->cx[k] + j->c->sig[k] * mt_normal(&s));
                p[1] = wrap1000(j->c->cy[k] + j->c->sig[k] * mt_normal(&s));
                p[2] = wrap1000(j->c->cz[k] + j->c->sig[k] * mt_normal(&s));
            } else {
                p[0] = (float)(mt_real2(&s) * 1000.0);
                p[1] = (float)(mt_real2(&s) * 1000.0);
                p[2] = (float)(mt_real2(&s) * 1000.0);
            }
        }
    }
    return NULL;
}

static void *halo_job(void *arg)
{
    GenJob *j = arg;
    uint64_t b, i;
    for (b = j->b0; b < j->b1; ++b) {
        sjcs_mt s;
        const uint64_t lo = b * GEN_BLOCK, hi = lo + GEN_BLOCK < j->n ? lo + GEN_BLOCK : j->n;
        sjcs_mt_seed(&s, block_seed(j->seed, b));
        for (i = lo; i < hi; ++i) {
            sjcs_halo *h = j->halos + i;
            h->id = j->id0 + i;
            h->mass = (float)(mt_real2(&s) * 1e12);
            if (mt_real2(&s) < j->frac) {
                /* halos sit at clump centres (uniform over clumps, not weighted) */
                uint32_t k = (uint32_t)(sjcs_mt_u32(&s) % j->c->n);
                h->point[0] = wrap1000(j->c->cx[k] + j->jitter * mt_normal(&s));
                h->point[1] = wrap1000(j->c->cy[k] + j->jitter * mt_normal(&s));
                h->point[2] = wrap1000(j->c->cz[k] + j->jitter * mt_normal(&s));
            } else {
                h->point[0] = (float)(mt_real2(&s) * 1000.0);
                h->point[1] = (float)(mt_real2(&s) * 1000.0);
                h->point[2] = (float)(mt_real2(&s) * 1000.0);
            }
        }
    }
    return NULL;
}

/* Run fn over the blocks of job proto on up to 64 threads. */
static void run_blocks(GenJob proto, void *(*fn)(void *))
{
    GenJob jobs[64];
    pthread_t th[64];
    const uint64_t nb = (proto.n + GEN_BLOCK - 1) / GEN_BLOCK;
    long hw = sysconf(_SC_NPROCESSORS_ONLN);
    int T = hw < 1 ? 1 : (hw > 64 ? 64 : (int)hw), t;
    if ((uint64_t)T > nb)
        T = nb ? (int)nb : 1;
    for (t = 0; t < T; ++t) {
        jobs[t] = proto;
        jobs[t].b0 = nb * t / T;
        jobs[t].b1 = nb * (t + 1) / T;
    }
    for (t = 1; t < T; ++t)
        pthread_create(&th[t], NULL, fn, &jobs[t]);
    fn(&jobs[0]);
    for (t = 1; t < T; ++t)
        pthread_join(th[t], NULL);
}

int sjcs_gen_clustered_particles(uint32_t seed, uint64_t n, uint32_t nclumps, double sig_lo, double sig_hi,
                                 double wsig, double frac_clumped, uint32_t clump_seed, float *out)
{
    Clumps c;
    GenJob j;
    if (make_clumps(&c, nclumps, sig_lo, sig_hi, wsig, clump_seed) != 0) {
        free_clumps(&c);
        return -1;
    }
    memset(&j, 0, sizeof(j));
    j.c = &c;
    j.seed = seed;
    j.n = n;
    j.frac = frac_clumped;
    j.pts = out;
    run_blocks(j, particle_job);
    free_clumps(&c);
    return 0;
}

int sjcs_gen_clustered_halos(uint32_t seed, uint64_t n, uint64_t id0, uint32_t nclumps, double sig_lo,
                             double sig_hi, double wsig, double frac_at_clumps, double jitter,
                             uint32_t clump_seed, sjcs_halo *out)
{
    Clumps c;
    GenJob j;
    if (make_clumps(&c, nclumps, sig_lo, sig_hi, wsig, clump_seed) != 0) {
        free_clumps(&c);
        return -1;
    }
    memset(&j, 0, sizeof(j));
    j.c = &c;
    j.seed = seed;
    j.n = n;
    j.id0 = id0;
    j.frac = frac_at_clumps;
    j.jitter = jitter;
    j.halos = out;
    run_blocks(j, halo_job);
    free_clumps(&c);
    round_all(out, n, 0);
    return 0;
}

int sjcs_write_halo_file(const char *path, const sjcs_halo *h, uint64_t n)
{
    FILE *fp = fopen(path, "wb");
    uint64_t i;
    char b[512];
    if (!fp)
        return -1;
    write_header(fp);
    for (i = 0; i < n; ++i) {
        int k = halo_line(b, sizeof(b), h[i].id, h[i].mass, h[i].point);
        fwrite(b, 1, (size_t)k, fp);
    }
    return fclose(fp) == 0 ? 0 : -1;
}
