/*
 * sjcs_oracle.c -- CPU restatement of the reference's hot path.
 * TEST INFRASTRUCTURE ONLY (checker for tests/, smoke(), and the "port" CPU
 * baseline of bench.py).  The product never links, imports or calls it.
 *
 * Built with -ffp-contract=off and scalar float arithmetic (x86-64 SSE, so
 * every float operation rounds to fp32, round-to-nearest, no FTZ/DAZ).
 */
#include "sjcs_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define BOX_LOW 0.0
#define BOX_UPP 1000.0

/* include/support_functions.h:18-34 (Logspace) + src/astr_rcount/main.c:646-649 */
int oracle_radius_table(double minrad, double maxrad, int nrads, int use_fma, float *r2)
{
    double a, b, c, t;
    int i;

    if (nrads <= 0 || r2 == NULL)
        return -1;
    if (minrad > maxrad) { /* main.c:531-533 */
        t = minrad;
        minrad = maxrad;
        maxrad = t;
    }
    a = log2(minrad);
    b = log2(maxrad);
    c = (b - a) / (nrads - 1);
    for (i = 0; i < nrads - 1; ++i)
        r2[i] = (float)pow(2.0, use_fma ? fma((double)i, c, a) : a + i * c);
    r2[nrads - 1] = (float)pow(2.0, b);
    for (i = 0; i < nrads; ++i)
        r2[i] *= r2[i];
    return 0;
}

/* Query box: setQueryMbr, src/objects/RTree/Mbr.c:207-239 (fp32 sub/add). */
typedef struct Box {
    float lo[3], hi[3];
} Box;

static void set_box(Box *b, const float c[3], float half)
{
    int a;
    for (a = 0; a < 3; ++a) {
        b->lo[a] = c[a] - half;
        b->hi[a] = c[a] + half;
    }
}

/* checkOverlapMbr with a leaf MBR (low == upp == p), Mbr.c:167-205:
 * _mm_cmpnlt_ps(upp, qlow) and _mm_cmpnlt_ps(qupp, low) must hold on every
 * lane; cmpnlt is true for unordered operands, hence the negated "<". */
static int in_box(const Box *b, const float p[3])
{
    int a;
    for (a = 0; a < 3; ++a)
        if (p[a] < b->lo[a] || b->hi[a] < p[a])
            return 0;
    return 1;
}

/* CalcDistance, include/objects/RTree/Distance.h:5-25: _mm_dp_ps(d, d, 0x77)
 * with d = p - c is (d0*d0 + d1*d1) + (d2*d2 + 0), each step rounded to fp32. */
static float calc_distance(const float p[3], const float c[3])
{
    float d0 = p[0] - c[0], d1 = p[1] - c[1], d2 = p[2] - c[2];
    float s01 = d0 * d0 + d1 * d1;
    float s2 = d2 * d2 + 0.0f;
    return s01 + s2;
}

/* Leaf step of MultiRangeCountRecursive, MultiRangeCount.c:103-113. */
static void bin_leaf(const float p[3], const float c[3], const float *r2, int nrads, uint64_t *counts)
{
    float dist = calc_distance(p, c);
    int i;
    for (i = 0; i < nrads; ++i) {
        if (dist < r2[i]) {
            counts[i]++;
            break;
        }
    }
}

/* ---- candidate generation: a CPU cell grid ------------------------------- */

typedef struct Grid {
    int G;
    double inv_h;
    uint32_t *start; /* G^3 + 1 */
    float *pts;      /* sorted x,y,z */
} Grid;

static int cell1(double v, const Grid *g)
{
    double t;
    if (v != v)
        return 0;
    t = floor(v * g->inv_h);
    if (t < 0)
        t = 0;
    if (t > g->G - 1)
        t = g->G - 1;
    return (int)t;
}

static int grid_build(Grid *g, const float *p, uint64_t np, float half)
{
    uint64_t i, ncell;
    uint32_t *cnt, *cell;
    double h = half > 0 && half == half ? (double)half : 1000.0;
    int G = (int)floor(1000.0 / h);
    if (G < 1)
        G = 1;
    if (G > 128)
        G = 128;
    g->G = G;
    g->inv_h = G / 1000.0;
    ncell = (uint64_t)G * G * G;
    g->start = calloc(ncell + 1, sizeof(uint32_t));
    g->pts = malloc((np ? np : 1) * 3 * sizeof(float));
    cnt = calloc(ncell + 1, sizeof(uint32_t));
    cell = malloc((np ? np : 1) * sizeof(uint32_t));
    if (!g->start || !g->pts || !cnt || !cell)
        return -1;
    for (i = 0; i < np; ++i) {
        const float *q = p + 3 * i;
        uint32_t c = ((uint32_t)cell1(q[2], g) * G + (uint32_t)cell1(q[1], g)) * G + (uint32_t)cell1(q[0], g);
        cell[i] = c;
        cnt[c + 1]++;
    }
    for (i = 0; i < ncell; ++i)
        cnt[i + 1] += cnt[i];
    memcpy(g->start, cnt, (ncell + 1) * sizeof(uint32_t));
    for (i = 0; i < np; ++i) {
        uint32_t slot = cnt[cell[i]]++;
        memcpy(g->pts + 3 * (uint64_t)slot, p + 3 * i, 3 * sizeof(float));
    }
    free(cnt);
    free(cell);
    return 0;
}

static void grid_free(Grid *g)
{
    free(g->start);
    free(g->pts);
}

/* One image: every particle whose cell lies in the box's cell range, then the
 * reference's own acceptance (box test, distance, first-match shell).  A NaN
 * box bound accepts everything on that side, so it opens the range. */
static void search_image(const Grid *g, const float c[3], float half, const float *r2, int nrads,
                         uint64_t *counts)
{
    Box b;
    int lo[3], hi[3], a, x, y, z;
    set_box(&b, c, half);
    for (a = 0; a < 3; ++a) {
        lo[a] = cell1(b.lo[a], g);
        hi[a] = (b.hi[a] != b.hi[a]) ? g->G - 1 : cell1(b.hi[a], g);
    }
    for (z = lo[2]; z <= hi[2]; ++z)
        for (y = lo[1]; y <= hi[1]; ++y) {
            uint64_t row = ((uint64_t)z * g->G + y) * g->G;
            uint32_t s = g->start[row + lo[0]], e = g->start[row + hi[0] + 1], k;
            for (k = s; k < e; ++k) {
                const float *p = g->pts + 3 * (uint64_t)k;
                if (in_box(&b, p))
                    bin_leaf(p, c, r2, nrads, counts);
            }
        }
}

static void search_image_brute(const float *pts, uint64_t np, const float c[3], float half, const float *r2,
                               int nrads, uint64_t *counts)
{
    Box b;
    uint64_t k;
    set_box(&b, c, half);
    for (k = 0; k < np; ++k)
        if (in_box(&b, pts + 3 * k))
            bin_leaf(pts + 3 * k, c, r2, nrads, counts);
}

typedef void (*image_fn)(const void *src, const float c[3], float half, const float *r2, int nrads,
                         uint64_t *counts);

typedef struct BruteSrc {
    const float *pts;
    uint64_t np;
} BruteSrc;

static void img_grid(const void *src, const float c[3], float half, const float *r2, int nrads, uint64_t *counts)
{
    search_image((const Grid *)src, c, half, r2, nrads, counts);
}

static void img_brute(const void *src, const float c[3], float half, const float *r2, int nrads, uint64_t *counts)
{
    const BruteSrc *b = src;
    search_image_brute(b->pts, b->np, c, half, r2, nrads, counts);
}

/* multiRangeCountWithPriodicBoundArraySTR, MultiRangeCount.c:13-73:
 * search the base image, take the out-of-bound flags of the BASE box
 * (checkMinMaxOutOfBoundMbr, Mbr.c:284-313: low < 0 and upp > 1000 per lane),
 * then for i < j < k over the flagged axes shift the centre by +-1000 in fp32
 * (min flag first) and search again. */
static void count_halo(image_fn fn, const void *src, const float c0[3], const float *r2, int nrads, int periodic,
                       uint64_t *counts)
{
    float R = (float)sqrt((double)r2[nrads - 1]); /* MultiRangeCount.c:19 */
    float moved[3];
    Box base;
    int min_oob[3], max_oob[3], i, j, k;

    if (!periodic) {
        /* multiRangeCountArraySTR passes the squared radius as the half-width (:81) */
        fn(src, c0, r2[nrads - 1], r2, nrads, counts);
        return;
    }
    set_box(&base, c0, R);
    fn(src, c0, R, r2, nrads, counts);
    for (i = 0; i < 3; ++i) {
        min_oob[i] = base.lo[i] < BOX_LOW;
        max_oob[i] = base.hi[i] > BOX_UPP;
    }
    memcpy(moved, c0, sizeof(moved));
    for (i = 0; i < 3; ++i) {
        if (min_oob[i])
            moved[i] += BOX_UPP;
        else if (max_oob[i])
            moved[i] -= BOX_UPP;
        else
            continue;
        fn(src, moved, R, r2, nrads, counts);
        for (j = i + 1; j < 3; ++j) {
            if (min_oob[j])
                moved[j] += BOX_UPP;
            else if (max_oob[j])
                moved[j] -= BOX_UPP;
            else
                continue;
            fn(src, moved, R, r2, nrads, counts);
            for (k = j + 1; k < 3; ++k) {
                if (min_oob[k])
                    moved[k] += BOX_UPP;
                else if (max_oob[k])
                    moved[k] -= BOX_UPP;
                else
                    continue;
                fn(src, moved, R, r2, nrads, counts);
                moved[k] = c0[k];
            }
            moved[j] = c0[j];
        }
        moved[i] = c0[i];
    }
}

typedef struct Job {
    image_fn fn;
    const void *src;
    const char *halo;
    size_t stride;
    uint64_t lo, hi;
    const float *r2;
    int nrads, periodic;
    uint64_t *counts;
} Job;

static void *run_job(void *arg)
{
    Job *jb = arg;
    uint64_t h;
    for (h = jb->lo; h < jb->hi; ++h) {
        float c[3];
        memcpy(c, jb->halo + h * jb->stride, sizeof(c));
        count_halo(jb->fn, jb->src, c, jb->r2, jb->nrads, jb->periodic, jb->counts + h * (uint64_t)jb->nrads);
    }
    return NULL;
}

static int run_all(image_fn fn, const void *src, const float *halo_xyz, size_t stride, uint64_t nhalos,
                   const float *r2, int nrads, int periodic, uint64_t *counts, int nthreads)
{
    Job *jobs;
    pthread_t *th;
    int t;
    if (nthreads <= 0) {
        long n = sysconf(_SC_NPROCESSORS_ONLN);
        nthreads = n > 0 ? (int)n : 1;
    }
    if ((uint64_t)nthreads > nhalos)
        nthreads = nhalos ? (int)nhalos : 1;
    jobs = calloc(nthreads, sizeof(Job));
    th = calloc(nthreads, sizeof(pthread_t));
    if (!jobs || !th)
        return -1;
    for (t = 0; t < nthreads; ++t) {
        Job j = {fn, src, (const char *)halo_xyz, stride, nhalos * t / nthreads, nhalos * (t + 1) / nthreads,
                 r2, nrads, periodic, counts};
        jobs[t] = j;
    }
    for (t = 1; t < nthreads; ++t)
        pthread_create(&th[t], NULL, run_job, &jobs[t]);
    run_job(&jobs[0]);
    for (t = 1; t < nthreads; ++t)
        pthread_join(th[t], NULL);
    free(jobs);
    free(th);
    return 0;
}

int oracle_count(const float *particles, uint64_t np, const float *halo_xyz, size_t stride, uint64_t nhalos,
                 const float *r2, int nrads, int periodic, uint64_t *counts, int nthreads)
{
    Grid g;
    int rc;
    float half;
    if (nrads <= 0 || !r2 || (nhalos && (!halo_xyz || !counts)) || (np && !particles))
        return -1;
    half = periodic ? (float)sqrt((double)r2[nrads - 1]) : r2[nrads - 1];
    if (grid_build(&g, particles, np, half) != 0)
        return -1;
    rc = run_all(img_grid, &g, halo_xyz, stride, nhalos, r2, nrads, periodic, counts, nthreads);
    grid_free(&g);
    return rc;
}

int oracle_count_brute(const float *particles, uint64_t np, const float *halo_xyz, size_t stride,
                       uint64_t nhalos, const float *r2, int nrads, int periodic, uint64_t *counts)
{
    BruteSrc b = {particles, np};
    if (nrads <= 0 || !r2 || (nhalos && (!halo_xyz || !counts)) || (np && !particles))
        return -1;
    return run_all(img_brute, &b, halo_xyz, stride, nhalos, r2, nrads, periodic, counts, 1);
}


/* ---- compressed particles ----------------------------------------------- */

typedef struct {
    int npart[6];
    double mass[6];
    double time, redshift;
    int flag_sfr, flag_feedback;
    int npartTotal[6];
    int flag_cooling, num_files;
    double BoxSize, Omega0, OmegaLambda, HubbleParam;
    int flag_stellarage, flag_metals, hashsize;
    float disp_min, disp_max;
    int pos_bits;
    long long id_start, id_end;
    char fill[56];
} oracle_gadget_header;

int oracle_decode_compressed(const void *header, const uint16_t *uv, uint64_t n, float *xyz)
{
    oracle_gadget_header h;
    long long total, ng1d, ng2d, ng3d;
    int n1d, nt1d = 1, nt2d = 1;
    float cell_interval, span;
    double unitsep;
    uint64_t i;
    if (!header || (n && (!uv || !xyz)))
        return -1;
    memcpy(&h, header, sizeof(h));
    /* GadgetHeader.c:12-23, one tile */
    total = (long long)h.npartTotal[1] + ((long long)h.npartTotal[2] << 32);
    n1d = (int)pow((double)total + 0.5, 1 / 3.);
    if (n1d <= 0)
        return -1;
    cell_interval = (float)(h.BoxSize / (double)n1d);
    span = h.disp_max - h.disp_min;
    unitsep = (double)span / pow(2.0, (double)h.pos_bits);
    /* GadId.c:28-35: Ng2D is computed as an int product */
    ng1d = n1d;
    ng2d = (long long)(int)((unsigned)n1d * (unsigned)n1d);
    ng3d = (long long)n1d * (long long)n1d * (long long)n1d;
    for (i = 0; i < n; ++i) {
        const long long ID = (long long)((unsigned long long)i + (unsigned long long)h.id_start);
        const long long IDt = (ID - 1) / ng3d;                 /* IDall2IDpartGadId */
        const long long IDg = ID - 1 - IDt * ng3d;
        const int ig = (int)(IDg / ng2d);                      /* IDg2IndexGadId */
        const int jg = (int)((IDg - ig * ng2d) / ng1d);
        const int kg = (int)(IDg - ig * ng2d - jg * ng1d);
        const int it = (int)(IDt / nt2d);                      /* IDt2IndexGadId */
        const int jt = (int)((IDt - it * nt2d) / nt1d);
        const int kt = (int)(IDt - it * nt2d - jt * nt1d);
        const int ip[3] = {(int)(it * ng1d + ig), (int)(jt * ng1d + jg), (int)(kt * ng1d + kg)};
        int a;
        for (a = 0; a < 3; ++a) {
            const float f = fmaf(cell_interval, (float)ip[a], h.disp_min);
            xyz[3 * i + a] = (float)fma(unitsep, (double)uv[3 * i + a], (double)f);
        }
    }
    return 0;
}
