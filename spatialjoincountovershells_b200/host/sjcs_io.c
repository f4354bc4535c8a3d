/*
 * sjcs_io.c -- reference file formats on the host: decoded particle files,
 * halo text files (plain and id-filtered), the radius schedule and the result
 * text.  See include/sjcs_host.h for the format summary.
 */
#define _GNU_SOURCE
#include "../../include/sjcs_host.h"

#include <errno.h>
#include <fcntl.h>
#include <math.h>
#include <pthread.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

/* fgets buffer of the reference's halo reader (BUFSIZE, include/Gadget/BufHalo.h:12) */
#define LINE_BUF (1024 * 16)
/* N_HEADER_LINES, include/Gadget/BufHalo.h:8 */
#define N_HEADER 16

static __thread char g_err[1024];

static int host_fail(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return -1;
}

const char *sjcs_host_last_error(void) { return g_err; }

static int default_threads(int nthreads)
{
    long n;
    if (nthreads > 0)
        return nthreads;
    n = sysconf(_SC_NPROCESSORS_ONLN);
    if (n < 1)
        n = 1;
    if (n > 32)
        n = 32;
    return (int)n;
}

/* ---- particles ------------------------------------------------------------ */

int sjcs_particle_file_count(const char *path, uint64_t *n)
{
    struct stat st;
    if (!path || !n)
        return host_fail("invalid argument");
    if (stat(path, &st) != 0)
        return host_fail("ERROR: file %s not found in readDecodedParticles()", path);
    *n = (uint64_t)st.st_size / (3 * sizeof(float));
    return 0;
}

typedef struct ReadJob {
    int fd;
    char *dst;
    uint64_t off, len;
    int bad;
} ReadJob;

static void *read_job(void *arg)
{
    ReadJob *j = arg;
    uint64_t done = 0;
    while (done < j->len) {
        const uint64_t want = j->len - done;
        ssize_t r = pread(j->fd, j->dst + done, (size_t)(want > (1u << 30) ? (1u << 30) : want),
                          (off_t)(j->off + done));
        if (r <= 0) {
            j->bad = 1;
            return NULL;
        }
        done += (uint64_t)r;
    }
    return NULL;
}

/* The whole file into buf (readDecodedParticles, src/Gadget/BufVector3D.c:
 * 285-308, reads it with one fread).  Files of 64 MB or more are read as
 * contiguous stripes by several threads (positional reads), so copies out
 * of the page cache or from a striped device proceed in parallel. */
int sjcs_read_particles(const char *path, float *buf, uint64_t cap, uint64_t *n)
{
    uint64_t num;
    int fd, T, t, bad = 0;
    if (sjcs_particle_file_count(path, &num) != 0)
        return -1;
    if (num > cap)
        return host_fail("buffer holds %llu particles, file %s has %llu", (unsigned long long)cap, path,
                         (unsigned long long)num);
    fd = open(path, O_RDONLY);
    if (fd < 0)
        return host_fail("ERROR: file %s not found in readDecodedParticles()", path);
    {
        const uint64_t total = num * 3 * sizeof(float);
        ReadJob jobs[32];
        pthread_t th[32];
        int started[32] = {0};
        T = total >= (64ull << 20) ? default_threads(0) : 1;
        if (T > 16)
            T = 16;
        for (t = 0; t < T; ++t) {
            /* stripes on 1 MB boundaries */
            const uint64_t lo = (total * (uint64_t)t / (uint64_t)T) & ~((1ull << 20) - 1);
            const uint64_t hi = (t == T - 1) ? total : (total * (uint64_t)(t + 1) / (uint64_t)T) & ~((1ull << 20) - 1);
            jobs[t].fd = fd;
            jobs[t].dst = (char *)buf + lo;
            jobs[t].off = lo;
            jobs[t].len = hi - lo;
            jobs[t].bad = 0;
        }
        for (t = 1; t < T; ++t)
            started[t] = pthread_create(&th[t], NULL, read_job, &jobs[t]) == 0;
        for (t = 0; t < T; ++t)
            if (!started[t])
                read_job(&jobs[t]); /* stripe 0, and any stripe whose thread did not start */
        for (t = 1; t < T; ++t)
            if (started[t])
                pthread_join(th[t], NULL);
        for (t = 0; t < T; ++t)
            bad |= jobs[t].bad;
    }
    close(fd);
    if (bad)
        return host_fail("short read on %s", path);
    *n = num;
    return 0;
}

int sjcs_write_particle_file(const char *path, const float *xyz, uint64_t n)
{
    FILE *fp = fopen(path, "wb");
    if (!fp)
        return host_fail("ERROR: cannot open %s", path);
    if (n && fwrite(xyz, 3 * sizeof(float), n, fp) != n) {
        fclose(fp);
        return host_fail("ERROR: while writing %s", path);
    }
    if (fclose(fp) != 0)
        return host_fail("ERROR: while writing %s", path);
    return 0;
}

/* ---- halos ---------------------------------------------------------------- */

/* GetDataFromLineFast, src/Gadget/BufHalo.c:218-249: id = strtoul of the
 * line, mass after the 2nd space, x after 6 more spaces, y and z after one
 * more each.  str is NUL-terminated like the reference's fgets buffer. */
/* Fast exact forms of strtof / strtoul for the plain decimal tokens the halo
 * files hold ("123.456789", "-0.5", "42"); anything else -- leading blanks,
 * exponents, hex, inf/nan, more than 19 significant digits, a value whose
 * conversion cannot be proven correctly rounded -- returns 0 and the caller
 * uses the C library, so the result always equals strtof's / strtoul's.
 *
 * A token is [-+]digits[.digits] ending at a character that cannot continue
 * a number.  Its value is m / 10^k exactly.  With m < 2^24 and k <= 10 both
 * are floats, and one float division is correctly rounded (Clinger).  With
 * m < 2^53 and k <= 22 both are doubles, the double quotient q is correctly
 * rounded, and rounding q to float equals rounding m / 10^k to float unless
 * q lies exactly on a midpoint between two floats (rounding is monotone and
 * every such midpoint is a double, so q can reach the other side of one only
 * by landing on it); q near a midpoint therefore goes to strtof. */
static const float kPow10f[11] = {1e0f, 1e1f, 1e2f, 1e3f, 1e4f, 1e5f, 1e6f, 1e7f, 1e8f, 1e9f, 1e10f};
static const double kPow10d[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
                                   1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};

static int continues_number(char c)
{
    return (c >= '0' && c <= '9') || c == '.' || (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z');
}

static int fast_f32(const char *s, float *out)
{
    int neg = 0, digits = 0, k = 0;
    uint64_t m = 0;
    if (*s == '-' || *s == '+')
        neg = (*s++ == '-');
    if (*s < '0' || *s > '9')
        return 0;
    while (*s >= '0' && *s <= '9') {
        if (m || *s != '0')
            ++digits;
        m = m * 10u + (uint64_t)(*s++ - '0');
        if (digits > 19)
            return 0;
    }
    if (*s == '.') {
        ++s;
        while (*s >= '0' && *s <= '9') {
            if (m || *s != '0')
                ++digits;
            m = m * 10u + (uint64_t)(*s++ - '0');
            ++k;
            if (digits > 19 || k > 22)
                return 0;
        }
    }
    if (continues_number(*s))
        return 0;
    if (m < (1u << 24) && k <= 10) {
        const float v = (float)m / kPow10f[k];
        *out = neg ? -v : v;
        return 1;
    }
    if (m < (1ull << 53)) {
        const double q = (double)m / kPow10d[k];
        uint64_t bits;
        memcpy(&bits, &q, sizeof(bits));
        {
            const int e = (int)((bits >> 52) & 0x7ff) - 1023;
            const uint32_t excess = (uint32_t)(bits & 0x1fffffffu); /* double bits below a float's */
            if (q == 0.0 || e < -126 || e > 127)
                return 0;
            if (excess >= 0x0ffffffeu && excess <= 0x10000002u)
                return 0; /* at or next to a midpoint */
        }
        *out = neg ? -(float)q : (float)q;
        return 1;
    }
    return 0;
}

static int fast_u64(const char *s, unsigned long *out)
{
    uint64_t m = 0;
    int n = 0;
    if (*s < '0' || *s > '9')
        return 0;
    while (*s >= '0' && *s <= '9') {
        m = m * 10u + (uint64_t)(*s++ - '0');
        if (++n > 19)
            return 0;
    }
    *out = (unsigned long)m;
    return 1;
}

static float f32_token(const char *s)
{
    float v;
    return fast_f32(s, &v) ? v : strtof(s, NULL);
}

static int parse_record(char *str, sjcs_halo *h)
{
    int i;
    {
        unsigned long id;
        h->id = fast_u64(str, &id) ? id : strtoul(str, NULL, 10);
    }
    for (i = 0; i < 2; i++) {
        if ((str = strchr(str, ' ')) == NULL)
            return -1;
        str++;
    }
    h->mass = f32_token(str);
    for (i = 0; i < 6; i++) {
        if ((str = strchr(str, ' ')) == NULL)
            return -1;
        str++;
    }
    h->point[0] = f32_token(str);
    if ((str = strchr(str, ' ')) == NULL)
        return -1;
    str++;
    h->point[1] = f32_token(str);
    if ((str = strchr(str, ' ')) == NULL)
        return -1;
    str++;
    h->point[2] = f32_token(str);
    return 0;
}

typedef struct HaloVec {
    sjcs_halo *h;
    uint64_t n, cap;
} HaloVec;

static int hv_push(HaloVec *v, const sjcs_halo *h)
{
    if (v->n == v->cap) {
        uint64_t nc = v->cap ? v->cap * 2 : 1024;
        sjcs_halo *p = realloc(v->h, nc * sizeof(sjcs_halo));
        if (!p)
            return -1;
        v->h = p;
        v->cap = nc;
    }
    v->h[v->n++] = *h;
    return 0;
}

/* The reference's reader, literally (readHalos, src/Gadget/BufHalo.c:76-119):
 * fgets pieces of at most LINE_BUF-1 bytes, 16 header pieces, stop at the
 * first fgets that reaches end of file. */
static int read_halos_fgets(const char *path, sjcs_halo **out, uint64_t *n)
{
    char tmp[LINE_BUF];
    FILE *fp;
    HaloVec v = {0};
    int row;
    if ((fp = fopen(path, "r")) == NULL)
        return host_fail("ERROR: file %s not found in readHalos().", path);
    tmp[0] = '\0';
    for (row = 0; row < N_HEADER; row++) {
        (void)!fgets(tmp, sizeof(tmp), fp);
        if (feof(fp)) {
            fclose(fp);
            return host_fail("ERROR: file %s does not contain headers in readHalos().", path);
        }
    }
    for (;;) {
        sjcs_halo h;
        (void)!fgets(tmp, sizeof(tmp), fp);
        if (feof(fp))
            break;
        if (parse_record(tmp, &h) < 0) {
            fclose(fp);
            free(v.h);
            return host_fail("ERROR: contents in file %s may be incorrect in readHalos().", path);
        }
        if (hv_push(&v, &h) != 0) {
            fclose(fp);
            free(v.h);
            return host_fail("ERROR: memory shortage in readHalos()");
        }
    }
    fclose(fp);
    *out = v.h ? v.h : malloc(sizeof(sjcs_halo));
    *n = v.n;
    return 0;
}

typedef struct ParseJob {
    const char *lo, *hi; /* [lo, hi): whole '\n'-terminated lines */
    sjcs_halo *dst;      /* NULL in the counting pass */
    uint64_t nlines;
    int bad;
} ParseJob;

static void *parse_job(void *arg)
{
    ParseJob *j = arg;
    const char *p = j->lo;
    char tmp[LINE_BUF];
    uint64_t k = 0;
    while (p < j->hi) {
        const char *nl = memchr(p, '\n', (size_t)(j->hi - p));
        size_t len = (size_t)(nl - p) + 1;
        if (j->dst) {
            memcpy(tmp, p, len);
            tmp[len] = '\0';
            if (parse_record(tmp, &j->dst[k]) < 0) {
                j->bad = 1;
                return NULL;
            }
        }
        k++;
        p = nl + 1;
    }
    j->nlines = k;
    return NULL;
}

int sjcs_read_halos(const char *path, sjcs_halo **out, uint64_t *n, int nthreads)
{
    int fd, T, t, row;
    struct stat st;
    const char *base, *p, *end, *data_end;
    ParseJob *jobs;
    pthread_t *th;
    uint64_t total = 0;
    if (!path || !out || !n)
        return host_fail("invalid argument");
    fd = open(path, O_RDONLY);
    if (fd < 0)
        return host_fail("ERROR: file %s not found in readHalos().", path);
    if (fstat(fd, &st) != 0 || st.st_size == 0) {
        close(fd);
        return host_fail("ERROR: file %s does not contain headers in readHalos().", path);
    }
    base = mmap(NULL, (size_t)st.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
    close(fd);
    if (base == MAP_FAILED)
        return read_halos_fgets(path, out, n);
    end = base + st.st_size;
    /* Any line of LINE_BUF-1 bytes or more makes fgets split it into several
     * records: leave such files to the literal reader. */
    {
        const char *q = base;
        while (q < end) {
            const char *nl = memchr(q, '\n', (size_t)(end - q));
            const char *le = nl ? nl + 1 : end;
            if (le - q >= LINE_BUF - 1) {
                munmap((void *)base, (size_t)st.st_size);
                return read_halos_fgets(path, out, n);
            }
            q = le;
        }
    }
    /* 16 header lines, each newline-terminated (an unterminated 16th line
     * makes fgets reach end of file: the reference reports missing headers). */
    p = base;
    for (row = 0; row < N_HEADER; row++) {
        const char *nl = memchr(p, '\n', (size_t)(end - p));
        if (!nl) {
            munmap((void *)base, (size_t)st.st_size);
            return host_fail("ERROR: file %s does not contain headers in readHalos().", path);
        }
        p = nl + 1;
    }
    /* records: every newline-terminated line; a final unterminated line is
     * dropped because its fgets reaches end of file. */
    data_end = end;
    while (data_end > p && data_end[-1] != '\n')
        data_end--;
    T = default_threads(nthreads);
    if ((uint64_t)(data_end - p) < (1u << 20))
        T = 1;
    jobs = calloc(T, sizeof(ParseJob));
    th = calloc(T, sizeof(pthread_t));
    if (!jobs || !th) {
        munmap((void *)base, (size_t)st.st_size);
        free(jobs);
        free(th);
        return host_fail("ERROR: memory shortage in readHalos()");
    }
    {
        const char *q = p;
        for (t = 0; t < T; t++) {
            const char *cut = p + (uint64_t)(data_end - p) * (t + 1) / T;
            if (t == T - 1)
                cut = data_end;
            else {
                if (cut < q)
                    cut = q;
                while (cut < data_end && cut[-1] != '\n')
                    cut++;
            }
            jobs[t].lo = q;
            jobs[t].hi = cut;
            q = cut;
        }
    }
    for (t = 1; t < T; t++)
        pthread_create(&th[t], NULL, parse_job, &jobs[t]);
    parse_job(&jobs[0]);
    for (t = 1; t < T; t++)
        pthread_join(th[t], NULL);
    for (t = 0; t < T; t++)
        total += jobs[t].nlines;
    *out = malloc((total ? total : 1) * sizeof(sjcs_halo));
    if (!*out) {
        munmap((void *)base, (size_t)st.st_size);
        free(jobs);
        free(th);
        return host_fail("ERROR: memory shortage in readHalos()");
    }
    {
        uint64_t off = 0;
        for (t = 0; t < T; t++) {
            jobs[t].dst = *out + off;
            off += jobs[t].nlines;
        }
    }
    for (t = 1; t < T; t++)
        pthread_create(&th[t], NULL, parse_job, &jobs[t]);
    parse_job(&jobs[0]);
    for (t = 1; t < T; t++)
        pthread_join(th[t], NULL);
    munmap((void *)base, (size_t)st.st_size);
    for (t = 0; t < T; t++) {
        if (jobs[t].bad) {
            free(*out);
            *out = NULL;
            free(jobs);
            free(th);
            return host_fail("ERROR: contents in file %s may be incorrect in readHalos().", path);
        }
    }
    free(jobs);
    free(th);
    *n = total;
    return 0;
}

void sjcs_host_free_halos(sjcs_halo *h) { free(h); }

static int cmp_u64(const void *a, const void *b)
{
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return (x > y) - (x < y);
}

/* readAndFilterHalos + ConstructFilterIdList, src/Gadget/BufHalo.c:121-214, 132-180 */
int sjcs_read_and_filter_halos(const char *path, const char *filter_path, sjcs_halo **out, uint64_t *n)
{
    char tmp[LINE_BUF];
    FILE *fp;
    uint64_t nfilters = 0, row, fr;
    uint64_t *filter;
    HaloVec v = {0};
    int hrow, finished = 0;

    if ((fp = fopen(filter_path, "r")) == NULL)
        return host_fail("ERROR: file %s not found in ConstructFilterIdList().", filter_path);
    for (;;) {
        if (fgets(tmp, sizeof(tmp), fp) == NULL && feof(fp))
            break;
        if (ferror(fp)) {
            fclose(fp);
            return host_fail("ERROR: while reading %s in ConstructFilterIdList()", filter_path);
        }
        nfilters++;
    }
    filter = malloc((nfilters ? nfilters : 1) * sizeof(uint64_t));
    if (!filter) {
        fclose(fp);
        return host_fail("ERROR: memory shortage");
    }
    rewind(fp);
    for (row = 0; row < nfilters; row++) {
        if (fgets(tmp, sizeof(tmp), fp) == NULL && feof(fp))
            break;
        filter[row] = (uint64_t)strtol(tmp, NULL, 10);
    }
    fclose(fp);
    /* the reference radix-sorts the ids as unsigned 64-bit keys */
    qsort(filter, nfilters, sizeof(uint64_t), cmp_u64);

    if ((fp = fopen(path, "r")) == NULL) {
        free(filter);
        return host_fail("ERROR: file %s not found in readAndFilterHalos().", path);
    }
    tmp[0] = '\0';
    for (hrow = 0; hrow < N_HEADER; hrow++) {
        (void)!fgets(tmp, sizeof(tmp), fp);
        if (feof(fp)) {
            fclose(fp);
            free(filter);
            return host_fail("ERROR: file %s does not contain headers in readAndFilterHalos().", path);
        }
    }
    fr = 0;
    for (;;) {
        sjcs_halo h;
        (void)!fgets(tmp, sizeof(tmp), fp);
        if (feof(fp))
            break;
        if (parse_record(tmp, &h) < 0) {
            fclose(fp);
            free(filter);
            free(v.h);
            return host_fail("ERROR: contents in file %s may be incorrect in readAndFilterHalos().", path);
        }
        /* An empty filter list reads past its end in the reference; here it
         * simply keeps nothing. */
        if (nfilters == 0)
            break;
        if (h.id < filter[fr])
            continue;
        else if (h.id > filter[fr]) {
            while (h.id > filter[fr]) {
                fr++;
                if (fr >= nfilters) {
                    finished = 1;
                    break;
                }
            }
        }
        if (finished)
            break;
        if (h.id == filter[fr] && hv_push(&v, &h) != 0) {
            fclose(fp);
            free(filter);
            free(v.h);
            return host_fail("ERROR: memory shortage in readAndFilterHalos()");
        }
    }
    fclose(fp);
    free(filter);
    *out = v.h ? v.h : malloc(sizeof(sjcs_halo));
    *n = v.n;
    return 0;
}

/* ---- radius schedule ------------------------------------------------------ */

int sjcs_host_radius_table(double minrad, double maxrad, int nrads, float *r2)
{
    double a, b, c, t;
    int i;
    if (nrads <= 0 || !r2)
        return host_fail("nrads must be > 0");
    if (minrad > maxrad) {
        t = minrad;
        minrad = maxrad;
        maxrad = t;
    }
    /* Logspace(2, log2(min), log2(max), n) (include/support_functions.h:18-34);
     * a + i*c is one fused multiply-add in the reference's -march=native build. */
    a = log2(minrad);
    b = log2(maxrad);
    c = (b - a) / (nrads - 1);
    for (i = 0; i < nrads - 1; ++i)
        r2[i] = (float)pow(2.0, fma((double)i, c, a));
    r2[nrads - 1] = (float)pow(2.0, b);
    for (i = 0; i < nrads; ++i)
        r2[i] = r2[i] * r2[i];
    return 0;
}

/* ---- result text ---------------------------------------------------------- */

static size_t put_u64(char *dst, uint64_t v)
{
    char tmp[24];
    size_t k = 0, i;
    do {
        tmp[k++] = (char)('0' + v % 10);
        v /= 10;
    } while (v);
    for (i = 0; i < k; ++i)
        dst[i] = tmp[k - 1 - i];
    return k;
}

typedef struct FmtJob {
    const sjcs_halo *halos;
    const uint64_t *counts;
    uint64_t lo, hi;
    int nrads;
    char **labels;
    size_t *label_len;
    char *buf;
    size_t len;
} FmtJob;

static size_t dec_len(uint64_t v)
{
    size_t k = 1;
    while (v >= 10) {
        v /= 10;
        ++k;
    }
    return k;
}

/* Bytes fmt_job writes for halos [lo, hi) (into j->len). */
static void *len_job(void *arg)
{
    FmtJob *j = arg;
    uint64_t h;
    size_t len = 0, labels = 0;
    int i;
    for (i = 0; i < j->nrads; ++i)
        labels += j->label_len[i] + 1;
    for (h = j->lo; h < j->hi; ++h) {
        const uint64_t *c = j->counts + h * (uint64_t)j->nrads;
        len += 4 + dec_len(j->halos[h].id) + labels;
        for (i = 0; i < j->nrads; ++i)
            len += dec_len(c[i]);
    }
    j->len = len;
    return NULL;
}

static void *fmt_job(void *arg)
{
    FmtJob *j = arg;
    char *o = j->buf;
    uint64_t h;
    int i;
    for (h = j->lo; h < j->hi; ++h) {
        const uint64_t *c = j->counts + h * (uint64_t)j->nrads;
        memcpy(o, "id ", 3);
        o += 3;
        o += put_u64(o, j->halos[h].id);
        *o++ = '\n';
        for (i = 0; i < j->nrads; ++i) {
            memcpy(o, j->labels[i], j->label_len[i]);
            o += j->label_len[i];
            o += put_u64(o, c[i]);
            *o++ = '\n';
        }
    }
    j->len = (size_t)(o - j->buf);
    return NULL;
}

/* Run fn over jobs[0..n) on threads (inline where a thread cannot start). */
static void run_jobs(void *(*fn)(void *), FmtJob *jobs, int n, pthread_t *th, int *started)
{
    int t;
    for (t = 1; t < n; ++t)
        started[t] = pthread_create(&th[t], NULL, fn, &jobs[t]) == 0;
    started[0] = 0;
    for (t = 0; t < n; ++t)
        if (!started[t])
            fn(&jobs[t]);
    for (t = 1; t < n; ++t)
        if (started[t])
            pthread_join(th[t], NULL);
}

/* Mapped writer for regular files: the exact size is computed first (one
 * parallel pass over the counts), the file's blocks are allocated up front
 * (so running out of space is an error here, never a fault while writing the
 * mapping), and every thread formats its halos straight into a shared mapping
 * at its own offset: no single writer to wait for.  Returns 0 = written,
 * -1 = failed (error set), 1 = use the stream writer (not a regular file, or
 * the file system cannot preallocate or map it). */
static int write_result_mapped(const char *path, const sjcs_halo *halos, uint64_t nhalos, const uint64_t *counts,
                               int nrads, char **labels, size_t *label_len, const uint64_t *total, int T)
{
    struct stat st;
    int fd, t, njobs, rc = -1;
    FmtJob *jobs = NULL;
    pthread_t *th = NULL;
    int *started = NULL;
    size_t maxline = 0, tail_len = 0, body = 0, size;
    char *tail = NULL, *map;
    uint64_t off;
    if (stat(path, &st) == 0 && !S_ISREG(st.st_mode))
        return 1;
    for (t = 0; t < nrads; ++t)
        if (label_len[t] > maxline)
            maxline = label_len[t];
    njobs = T * 4;
    if ((uint64_t)njobs > nhalos)
        njobs = nhalos ? (int)nhalos : 1;
    jobs = calloc((size_t)njobs, sizeof(FmtJob));
    th = calloc((size_t)njobs, sizeof(pthread_t));
    started = calloc((size_t)njobs, sizeof(int));
    tail = malloc(8 + (size_t)nrads * (maxline + 22));
    if (!jobs || !th || !started || !tail) {
        host_fail("ERROR: memory shortage in outputResult()");
        goto out;
    }
    for (t = 0; t < njobs; ++t) {
        jobs[t].halos = halos;
        jobs[t].counts = counts;
        jobs[t].lo = nhalos * (uint64_t)t / (uint64_t)njobs;
        jobs[t].hi = nhalos * (uint64_t)(t + 1) / (uint64_t)njobs;
        jobs[t].nrads = nrads;
        jobs[t].labels = labels;
        jobs[t].label_len = label_len;
    }
    run_jobs(len_job, jobs, njobs, th, started);
    for (t = 0; t < njobs; ++t)
        body += jobs[t].len;
    /* the Total block: the running total is halo 0's own row (main.c:400, 413) */
    memcpy(tail, "\nTotal\n", 7);
    tail_len = 7;
    for (t = 0; t < nrads; ++t) {
        memcpy(tail + tail_len, labels[t], label_len[t]);
        tail_len += label_len[t];
        tail_len += put_u64(tail + tail_len, total[t]);
        tail[tail_len++] = '\n';
    }
    size = body + tail_len;
    fd = open(path, O_RDWR | O_CREAT | O_TRUNC, 0666);
    if (fd < 0) {
        host_fail("Cannot create %s in outputResult().", path);
        goto out;
    }
    if (fallocate(fd, 0, 0, (off_t)size) != 0) {
        const int e = errno;
        close(fd);
        if (e == ENOSPC || e == EFBIG || e == EDQUOT)
            host_fail("ERROR: while writing %s in outputResult()", path);
        else
            rc = 1;
        goto out;
    }
    map = mmap(NULL, size, PROT_READ | PROT_WRITE, MAP_SHARED, fd, 0);
    if (map == MAP_FAILED) {
        close(fd);
        rc = 1;
        goto out;
    }
    off = 0;
    for (t = 0; t < njobs; ++t) {
        jobs[t].buf = map + off;
        off += jobs[t].len;
    }
    run_jobs(fmt_job, jobs, njobs, th, started);
    memcpy(map + body, tail, tail_len);
    rc = 0;
    if (munmap(map, size) != 0)
        rc = host_fail("ERROR: while writing %s in outputResult()", path);
    if (close(fd) != 0 && rc == 0)
        rc = host_fail("ERROR: while writing %s in outputResult()", path);
out:
    free(jobs);
    free(th);
    free(started);
    free(tail);
    return rc;
}

int sjcs_write_result(const char *path, const sjcs_halo *halos, uint64_t nhalos, const float *r2, int nrads,
                      const uint64_t *counts, int nthreads)
{
    FILE *fp;
    char **labels = NULL;
    size_t *label_len = NULL, maxline;
    float *rad = NULL;
    uint64_t *total = NULL, h;
    int i, T, rc = -1;
    FmtJob *jobs = NULL; /* two rounds of T jobs: one is written while the other is formatted */
    pthread_t *th = NULL;
    int *started = NULL;
    const uint64_t per_job = 8192;

    if (nrads <= 0 || !r2)
        return host_fail("invalid radius table");
    /* radiuses were squared for the search; print (float)sqrt of them (main.c:386-387) */
    rad = malloc(nrads * sizeof(float));
    labels = calloc(nrads, sizeof(char *));
    label_len = calloc(nrads, sizeof(size_t));
    total = calloc(nrads, sizeof(uint64_t));
    if (!rad || !labels || !label_len || !total)
        goto out;
    for (i = 0; i < nrads; ++i)
        rad[i] = (float)sqrt((double)r2[i]);
    maxline = 0;
    for (i = 0; i < nrads; ++i) {
        char b[256];
        int k = (i == 0) ? snprintf(b, sizeof(b), "  [0.0 ~ %f]: ", rad[0])
                         : snprintf(b, sizeof(b), "  [%f ~ %f]: ", rad[i - 1], rad[i]);
        labels[i] = strdup(b);
        label_len[i] = (size_t)k;
        if ((size_t)k > maxline)
            maxline = (size_t)k;
        if (!labels[i])
            goto out;
    }
    /* Total = sum over all halos, plus halo 0 once more: the reference's
     * running total is halo 0's own row (main.c:400, 413). */
    for (h = 0; h < nhalos; ++h)
        for (i = 0; i < nrads; ++i)
            total[i] += counts[h * (uint64_t)nrads + i];
    if (nhalos)
        for (i = 0; i < nrads; ++i)
            total[i] += counts[i];

    if (path) {
        const int m = write_result_mapped(path, halos, nhalos, counts, nrads, labels, label_len, total,
                                          default_threads(nthreads));
        if (m <= 0) {
            rc = m;
            goto out;
        }
    }
    fp = path ? fopen(path, "w") : stdout;
    if (!fp) {
        host_fail("Cannot create %s in outputResult().", path);
        goto out;
    }
    T = default_threads(nthreads);
    jobs = calloc(2 * (size_t)T, sizeof(FmtJob));
    th = calloc(2 * (size_t)T, sizeof(pthread_t));
    started = calloc(2 * (size_t)T, sizeof(int));
    if (!jobs || !th || !started)
        goto close_out;
    for (i = 0; i < 2 * T; ++i) {
        jobs[i].buf = malloc(per_job * (24 + (size_t)nrads * (maxline + 22)));
        if (!jobs[i].buf)
            goto close_out;
    }
    /* Round r is formatted by threads into job set r % 2 while this thread
     * writes round r - 1 from the other set, in halo order. */
    {
        int prev_used = 0, r = 0, werr = 0;
        for (h = 0; h < nhalos || prev_used; ++r) {
            FmtJob *cur = jobs + (size_t)(r & 1) * T, *prev = jobs + (size_t)((r + 1) & 1) * T;
            pthread_t *cth = th + (size_t)(r & 1) * T;
            int *cst = started + (size_t)(r & 1) * T;
            int used = 0;
            for (i = 0; i < T && h < nhalos; ++i) {
                uint64_t e = h + per_job < nhalos ? h + per_job : nhalos;
                cur[i].halos = halos;
                cur[i].counts = counts;
                cur[i].lo = h;
                cur[i].hi = e;
                cur[i].nrads = nrads;
                cur[i].labels = labels;
                cur[i].label_len = label_len;
                h = e;
                used++;
            }
            for (i = 0; i < used; ++i)
                cst[i] = pthread_create(&cth[i], NULL, fmt_job, &cur[i]) == 0;
            for (i = 0; i < prev_used && !werr; ++i)
                werr = fwrite(prev[i].buf, 1, prev[i].len, fp) != prev[i].len;
            for (i = 0; i < used; ++i) {
                if (cst[i])
                    pthread_join(cth[i], NULL);
                else
                    fmt_job(&cur[i]); /* no thread: format it here */
            }
            if (werr) {
                host_fail("ERROR: while writing %s in outputResult()", path ? path : "(stdout)");
                goto close_out;
            }
            prev_used = used;
        }
    }
    fputs("\nTotal\n", fp);
    for (i = 0; i < nrads; ++i) {
        char b[32];
        size_t k = put_u64(b, total[i]);
        fwrite(labels[i], 1, label_len[i], fp);
        fwrite(b, 1, k, fp);
        fputc('\n', fp);
    }
    if (ferror(fp)) {
        host_fail("ERROR: while writing %s in outputResult()", path ? path : "(stdout)");
        goto close_out;
    }
    rc = 0;
close_out:
    if (fp != stdout) {
        if (fclose(fp) != 0 && rc == 0)
            rc = host_fail("ERROR: while writing %s in outputResult()", path);
    } else
        fflush(stdout);
out:
    if (jobs)
        for (i = 0; i < 2 * T; ++i)
            free(jobs[i].buf);
    free(jobs);
    free(th);
    free(started);
    if (labels)
        for (i = 0; i < nrads; ++i)
            free(labels[i]);
    free(labels);
    free(label_len);
    free(rad);
    free(total);
    return rc;
}


/* ---- compressed (Gadget-encoded) particle files --------------------------- */

_Static_assert(sizeof(sjcs_gadget_header) == 256, "the Gadget header is 256 bytes");

int sjcs_read_compressed_header(const char *path, sjcs_gadget_header *hdr)
{
    FILE *fp;
    if (!path || !hdr)
        return host_fail("invalid argument");
    fp = fopen(path, "rb");
    if (!fp)
        return host_fail("ERROR: file %s not found in readCompressedParticlesHeader()", path);
    if (fseek(fp, (long)sizeof(int), SEEK_SET) != 0 || fread(hdr, sizeof(*hdr), 1, fp) != 1) {
        fclose(fp);
        return host_fail("short read on %s (Gadget header)", path);
    }
    fclose(fp);
    if (hdr->npart[1] < 0)
        return host_fail("%s: negative particle count in the header", path);
    return 0;
}

int sjcs_read_compressed_particles(const char *path, sjcs_gadget_header *hdr, uint16_t *uv, uint64_t cap,
                                   uint64_t *n)
{
    FILE *fp;
    uint64_t num;
    if (!path || !hdr || !n)
        return host_fail("invalid argument");
    if (sjcs_read_compressed_header(path, hdr) != 0)
        return -1;
    num = (uint64_t)hdr->npart[1];
    if (!uv) { /* count only */
        *n = num;
        return 0;
    }
    if (num > cap)
        return host_fail("buffer holds %llu particles, file %s has %llu", (unsigned long long)cap, path,
                         (unsigned long long)num);
    fp = fopen(path, "rb");
    if (!fp)
        return host_fail("ERROR: file %s not found in readCompressedParticles()", path);
    /* record marker, header, end marker + next record's marker */
    if (fseek(fp, (long)(sizeof(int) + sizeof(*hdr) + 2 * sizeof(int)), SEEK_SET) != 0 ||
        fread(uv, 3 * sizeof(uint16_t), (size_t)num, fp) != (size_t)num) {
        fclose(fp);
        return host_fail("short read on %s (compressed particles)", path);
    }
    fclose(fp);
    *n = num;
    return 0;
}

int sjcs_write_compressed_file(const char *path, const sjcs_gadget_header *hdr, const uint16_t *uv, uint64_t n)
{
    FILE *fp;
    int m;
    if (!path || !hdr || (n && !uv))
        return host_fail("invalid argument");
    fp = fopen(path, "wb");
    if (!fp)
        return host_fail("cannot create %s", path);
    m = (int)sizeof(*hdr);
    fwrite(&m, sizeof(m), 1, fp);
    fwrite(hdr, sizeof(*hdr), 1, fp);
    fwrite(&m, sizeof(m), 1, fp);
    m = (int)(n * 3 * sizeof(uint16_t));
    fwrite(&m, sizeof(m), 1, fp);
    if (n)
        fwrite(uv, 3 * sizeof(uint16_t), (size_t)n, fp);
    fwrite(&m, sizeof(m), 1, fp);
    if (fclose(fp) != 0)
        return host_fail("write failed on %s", path);
    return 0;
}

int sjcs_gen_compressed(uint32_t seed, int n1d, double box, float disp_min, float disp_max, int pos_bits,
                        long long id_start, uint64_t n, sjcs_gadget_header *hdr, uint16_t *uv)
{
    sjcs_mt mt;
    uint64_t i, total;
    uint32_t mask;
    if (!hdr || n1d <= 0 || pos_bits <= 0 || pos_bits > 16 || (n && !uv))
        return host_fail("invalid argument");
    total = (uint64_t)n1d * (uint64_t)n1d * (uint64_t)n1d;
    if (n > total || n > 0x7fffffffull)
        return host_fail("n (%llu) exceeds the lattice (%llu) or 2^31-1", (unsigned long long)n,
                         (unsigned long long)total);
    memset(hdr, 0, sizeof(*hdr));
    hdr->npart[1] = (int)n;
    hdr->npartTotal[1] = (int)(total & 0xffffffffull);
    hdr->npartTotal[2] = (int)(total >> 32);
    hdr->num_files = 1;
    hdr->BoxSize = box;
    hdr->disp_min = disp_min;
    hdr->disp_max = disp_max;
    hdr->pos_bits = pos_bits;
    hdr->id_start = id_start;
    hdr->id_end = id_start + (long long)n - 1;
    mask = (pos_bits >= 16) ? 0xffffu : ((1u << pos_bits) - 1u);
    sjcs_mt_seed(&mt, seed);
    for (i = 0; i < 3 * n; ++i)
        uv[i] = (uint16_t)(sjcs_mt_u32(&mt) & mask);
    return 0;
}
