/*
 * sjcs_rcount -- drop-in for the reference's astr_rcount driver
 * (src/astr_rcount/main.c), with the index build and the shell count on the
 * GPU through libsjcs.so.
 *
 * Kept from the reference: the command line (same options, same parsing
 * rules: last occurrence wins, a file list runs to the next argument starting
 * with '-'), the validation rules and messages (main.c:506-602), the
 * "--execution info--" block (main.c:604-621), the ">>>> ... time" lines, the
 * radius schedule (Logspace then squaring, main.c:644-649), counts accumulated
 * across particle files, and the result text including its Total block
 * (main.c:371-442).
 *
 * Changed: --thread / --next-setup size the host threads that parse the halo
 * file and format the result (the GPU does the work the thread pool did);
 * --backlog B keeps up to B particle files read, copied and indexed ahead on
 * the build stream while the count stream searches the current one (the
 * reference's backlog pipeline, main.c:266-350, on two CUDA streams); a
 * missing or unreadable input file is reported and the program exits with
 * status 1 where the reference dereferences a NULL buffer.  --compressed
 * files are read as uint16 triplets (half the bytes of decoded floats) and
 * decoded on the GPU, bit-identically to decodeCompressedParticle.
 *
 * Added (GPU options, all optional): --index grid|morton|learned picks the
 * index form; --schedule auto|static|queue the count schedule; --autotune
 * times the schedules on the first file and keeps the fastest; --graph runs
 * every file step (copy, build, count) as a captured CUDA graph, reading the
 * next file into a second pinned buffer while the current step runs.
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdbool.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include "../../include/sjcs.h"
#include "../../include/sjcs_host.h"

#define TMP_BUFSIZE 1024
#define BOOL2STRING(b) ((b) ? "true" : "false")

/* ---- option parsing (src/GetOption/GetOption.c) --------------------------- */

enum { OPT_INT, OPT_STRING_PTR };

static int get_option_value(int argc, char *argv[], void *dst, int type, const char *opt, int offset)
{
    size_t optlen = strlen(opt);
    int i;
    for (i = 1; i < argc; i++) {
        if (strlen(argv[i]) != optlen)
            continue;
        if (memcmp(argv[i], opt, optlen) == 0) {
            i += offset + 1;
            if (i >= argc)
                return -1;
            if (type == OPT_INT)
                *(int *)dst = (int)strtol(argv[i], NULL, 10);
            else
                *(char **)dst = argv[i];
        }
    }
    return 0;
}

static void get_option_range(int argc, char *argv[], int *beg, int *end, const char *opt)
{
    size_t optlen = strlen(opt);
    int i, j;
    for (i = 1; i < argc; i++) {
        if (strlen(argv[i]) != optlen)
            continue;
        if (memcmp(argv[i], opt, optlen) == 0) {
            for (j = i + 1; j < argc && *argv[j] != '-'; j++)
                ;
            if (j != i + 1) {
                *beg = i + 1;
                *end = j;
            }
        }
    }
}

static bool get_option_flag(int argc, char *argv[], const char *opt)
{
    size_t optlen = strlen(opt);
    int i;
    for (i = 1; i < argc; i++) {
        if (strlen(argv[i]) != optlen)
            continue;
        if (memcmp(argv[i], opt, optlen) == 0)
            return true;
    }
    return false;
}

/* ---- timing lines (include/time.h) ---------------------------------------- */

static double now_us(void)
{
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec * 1e6 + tv.tv_usec;
}

static void print_ms(const char *msg, double t0)
{
    long diff = (long)(now_us() - t0);
    printf("%s: %ld milli seconds\n", msg, diff / 1000);
}

static void set_error(bool *flag, char *buf, const char *msg)
{
    if (!*flag) {
        *flag = true;
        strcpy(buf, msg);
    }
}

static void usage_exit(char *argv[])
{
    fprintf(stderr,
            "Usage: %s \n"
            "          --thread #_of_threads_used_in_this_process\n"
            "          --next-setup #_of_threads_to_build_next_index_in_background\n"
            "          --particle-files particle_files(1 or more) [--compressed]\n"
            "          --halo-file halo_file [--filter-file filter_id_list_file]\n"
            "          --radius minimum_radius:maximum_radius:#_of_bins\n"
            "          [--backlog max_#_of_backlog_indexes]\n"
            "          [--first-setup #_of_indexes_be_firstly_built:#_of_threads_to_build_each_index]\n"
            "          [--output-file output_file_name]\n",
            argv[0]);
    exit(EXIT_FAILURE);
}

static void die_lib(const char *what)
{
    fprintf(stderr, "ERROR: %s: %s\n", what, sjcs_last_error());
    exit(EXIT_FAILURE);
}

/* ---- GPU options ------------------------------------------------------------ */

static int g_index_kind = SJCS_INDEX_GRID;

/* Context preparation for the particle files, run beside the halo parse. */
static struct {
    sjcs_ctx *ctx;
    uint64_t n;
    pthread_t th;
    int started;
} g_prepare;

static void *prepare_files(void *arg)
{
    (void)arg;
    sjcs_ctx_prepare_files(g_prepare.ctx, g_prepare.n);
    return NULL;
}
static bool g_autotune = false;
static bool g_compressed = false; /* --compressed: Gadget-encoded particle files, decoded on the GPU */

static void autotune_once(sjcs_ctx *ctx, sjcs_query *q, sjcs_index *idx)
{
    sjcs_schedule chosen;
    float ms[16];
    int nt = 0, i;
    double t0;
    if (!g_autotune)
        return;
    g_autotune = false;
    t0 = now_us();
    if (sjcs_autotune(ctx, q, idx, &chosen, ms, 16, &nt) != SJCS_OK)
        die_lib("autotune");
    printf("  autotune: schedule %s (piece %u, max pieces %u); trials:",
           chosen.mode == SJCS_SCHED_QUEUE ? "queue" : "static", chosen.piece, chosen.max_pieces);
    for (i = 0; i < nt && i < 16; i++)
        printf(" %.2f", ms[i]);
    printf(" ms\n");
    print_ms(">>>> autotuning time", t0);
}

/* ---- one particle file in flight ------------------------------------------ */

typedef struct Pending {
    int file;
    float *host; /* pinned: x,y,z floats, or uint16 triplets of a compressed file */
    uint64_t n;
    sjcs_index *idx;
} Pending;

/* A compressed file: header and triplets into pinned memory, then the build
 * that decodes on the device (constructIndexWithSameThreadPool's compressed
 * branch, src/astr_rcount/main.c:739-763). */
static void start_index_compressed(sjcs_ctx *ctx, const char *fname, const sjcs_index_opts *opts, Pending *p)
{
    sjcs_gadget_header hdr;
    uint64_t n = 0;
    double t0 = now_us();
    if (sjcs_read_compressed_particles(fname, &hdr, NULL, 0, &n) != 0) {
        fprintf(stderr, "%s\n", sjcs_host_last_error());
        exit(EXIT_FAILURE);
    }
    if (sjcs_host_alloc((n ? n : 1) * 3 * sizeof(uint16_t), (void **)&p->host) != SJCS_OK)
        die_lib("pinned buffer");
    if (sjcs_read_compressed_particles(fname, &hdr, (uint16_t *)p->host, n, &p->n) != 0) {
        fprintf(stderr, "%s\n", sjcs_host_last_error());
        exit(EXIT_FAILURE);
    }
    print_ms(">>>> particles reading time", t0);
    if (sjcs_index_build_compressed(ctx, (const uint16_t *)p->host, p->n, &hdr, opts, &p->idx) != SJCS_OK)
        die_lib("index build");
}

/* Read a particle file into pinned memory and queue its index build.
 * Replaces constructIndexWithSameThreadPool (main.c:732-786). */
static void start_index(sjcs_ctx *ctx, const char *fname, float radius_hint, Pending *p)
{
    sjcs_index_opts opts;
    uint64_t n = 0;
    double t0;
    memset(&opts, 0, sizeof(opts));
    opts.kind = g_index_kind;
    opts.radius_hint = radius_hint;
    if (g_compressed) {
        start_index_compressed(ctx, fname, &opts, p);
        return;
    }
    t0 = now_us();
    if (sjcs_particle_file_count(fname, &n) != 0) {
        fprintf(stderr, "%s\n", sjcs_host_last_error());
        exit(EXIT_FAILURE);
    }
    /* read in chunks through the context's staging slots, each chunk copied
     * to the device as soon as it is read; the build is queued behind them */
    p->host = NULL;
    p->n = n;
    if (sjcs_index_build_file(ctx, fname, &opts, &p->idx) != SJCS_OK)
        die_lib("particle file read / index build");
    print_ms(">>>> particles reading time", t0);
}

static void finish_index(Pending *p, double t0)
{
    if (sjcs_index_wait(p->idx) != SJCS_OK)
        die_lib("index build");
    sjcs_host_free(p->host);
    p->host = NULL;
    if (t0 >= 0)
        print_ms(g_compressed ? ">>>> particles decoding + index construction time" : ">>>> index construction time",
                 t0);
    printf("  # of particles = %llu\n", (unsigned long long)p->n);
}

static void search_and_destroy(sjcs_ctx *ctx, sjcs_query *q, Pending *p)
{
    double t0;
    autotune_once(ctx, q, p->idx);
    t0 = now_us();
    if (sjcs_query_count(ctx, q, p->idx) != SJCS_OK)
        die_lib("shell count");
    if (sjcs_ctx_sync(ctx) != SJCS_OK)
        die_lib("shell count");
    print_ms(">>>> searching time", t0);
    t0 = now_us();
    sjcs_index_destroy(p->idx);
    p->idx = NULL;
    print_ms(">>>> index destruction time", t0);
}

/* noBacklogExecution, main.c:235-264 */
static void no_backlog(sjcs_ctx *ctx, sjcs_query *q, char **files, int nfiles, float radius_hint)
{
    int i;
    puts("  -- with no backlog execution");
    for (i = 0; i < nfiles; i++) {
        Pending p;
        double t0;
        memset(&p, 0, sizeof(p));
        p.file = i;
        start_index(ctx, files[i], radius_hint, &p);
        t0 = now_us();
        finish_index(&p, t0);
        search_and_destroy(ctx, q, &p);
    }
}

/* withBacklogExecution, main.c:266-350: up to maxbacklogs files are read and
 * indexed ahead (first_nbacklogs of them before the first search); each
 * search overlaps the reading and building of the files behind it. */
static void with_backlog(sjcs_ctx *ctx, sjcs_query *q, char **files, int nfiles, int maxbacklogs,
                         int first_nbacklogs, float radius_hint)
{
    Pending *ring = calloc((size_t)maxbacklogs + 1, sizeof(Pending));
    int head = 0, count = 0, next = 0, i, cap = maxbacklogs + 1;
    puts("  -- with backlog execution");
    while (count < first_nbacklogs && next < nfiles) {
        Pending *p = &ring[(head + count) % cap];
        memset(p, 0, sizeof(*p));
        p->file = next;
        printf("index %d\n", next);
        start_index(ctx, files[next], radius_hint, p);
        next++;
        count++;
    }
    for (i = 0; i < nfiles; i++) {
        Pending *cur;
        double t0;
        if (count == 0) { /* nothing ahead: build it now */
            Pending *p = &ring[head];
            memset(p, 0, sizeof(*p));
            p->file = next;
            printf("index %d\n", next);
            start_index(ctx, files[next], radius_hint, p);
            next++;
            count++;
        }
        cur = &ring[head];
        t0 = now_us();
        finish_index(cur, -1.0);
        print_ms(">>>> index getting time", t0);
        head = (head + 1) % cap;
        count--;
        autotune_once(ctx, q, cur->idx);
        t0 = now_us();
        if (sjcs_query_count(ctx, q, cur->idx) != SJCS_OK)
            die_lib("shell count");
        /* read and queue the next files while the search runs */
        while (count < maxbacklogs && next < nfiles) {
            Pending *p = &ring[(head + count) % cap];
            memset(p, 0, sizeof(*p));
            p->file = next;
            printf("index %d\n", next);
            start_index(ctx, files[next], radius_hint, p);
            next++;
            count++;
        }
        /* wait for this file's search only; the builds queued behind it keep running */
        if (sjcs_query_wait(q) != SJCS_OK)
            die_lib("shell count");
        print_ms(">>>> searching time", t0);
        t0 = now_us();
        sjcs_index_destroy(cur->idx);
        cur->idx = NULL;
        print_ms(">>>> index destruction time", t0);
    }
    free(ring);
}

/* Every file step as a captured CUDA graph; two steps over two pinned
 * buffers alternate so the next file is read while the current step runs. */
static void report_step(sjcs_step *st, int file)
{
    float ms = 0.0f;
    if (sjcs_step_time(st, &ms) != SJCS_OK)
        die_lib("file step");
    printf(">>>> file %d step time (copy + build + search): %.2f milli seconds\n", file, ms);
}

static void graph_steps(sjcs_ctx *ctx, sjcs_query *q, char **files, int nfiles, float radius_hint)
{
    sjcs_step *st[2] = {NULL, NULL};
    float *buf[2] = {NULL, NULL};
    uint64_t bufcap[2] = {0, 0}, stepn[2] = {0, 0};
    int last[2] = {-1, -1};
    sjcs_index_opts opts;
    int i;
    memset(&opts, 0, sizeof(opts));
    opts.kind = g_index_kind;
    opts.radius_hint = radius_hint;
    puts("  -- with captured file steps (CUDA graphs)");
    for (i = 0; i < nfiles; i++) {
        const int b = i & 1;
        uint64_t n = 0, got = 0;
        double t0 = now_us();
        if (sjcs_particle_file_count(files[i], &n) != 0) {
            fprintf(stderr, "%s\n", sjcs_host_last_error());
            exit(EXIT_FAILURE);
        }
        if (st[b] && last[b] >= 0) { /* this buffer's previous step must be done before the refill */
            report_step(st[b], last[b]);
            last[b] = -1;
        }
        if (!buf[b] || n > bufcap[b]) {
            if (st[b])
                sjcs_step_destroy(st[b]);
            st[b] = NULL;
            if (buf[b])
                sjcs_host_free(buf[b]);
            if (sjcs_host_alloc((n ? n : 1) * 3 * sizeof(float), (void **)&buf[b]) != SJCS_OK)
                die_lib("pinned buffer");
            bufcap[b] = n;
        }
        if (sjcs_read_particles(files[i], buf[b], n, &got) != 0) {
            fprintf(stderr, "%s\n", sjcs_host_last_error());
            exit(EXIT_FAILURE);
        }
        print_ms(">>>> particles reading time", t0);
        printf("  # of particles = %llu\n", (unsigned long long)got);
        if (got == 0)
            continue; /* an empty file adds nothing */
        if (g_autotune) { /* tune on this file with an ordinary build before capturing */
            sjcs_index *idx = NULL;
            if (sjcs_index_build(ctx, buf[b], got, &opts, &idx) != SJCS_OK || sjcs_index_wait(idx) != SJCS_OK)
                die_lib("index build");
            autotune_once(ctx, q, idx);
            sjcs_index_destroy(idx);
        }
        if (st[b] && got != stepn[b]) { /* a captured step replays one particle count only */
            sjcs_step_destroy(st[b]);
            st[b] = NULL;
        }
        if (!st[b]) {
            if (sjcs_step_create(ctx, q, buf[b], got, &opts, &st[b]) != SJCS_OK)
                die_lib("file step capture");
            stepn[b] = got;
        }
        if (sjcs_step_launch(ctx, st[b]) != SJCS_OK)
            die_lib("file step");
        last[b] = i;
    }
    for (i = 0; i < 2; i++) {
        const int b = (nfiles + i) & 1; /* the older of the two last steps first */
        if (st[b] && last[b] >= 0)
            report_step(st[b], last[b]);
    }
    for (i = 0; i < 2; i++) {
        if (st[i])
            sjcs_step_destroy(st[i]);
        if (buf[i])
            sjcs_host_free(buf[i]);
    }
}

int main(int argc, char *argv[])
{
    char *outfile_name = NULL;
    int particle_beg = -1, particle_end = -1;
    bool particle_compressed;
    char *halo_name = NULL, *halo_filter_name = NULL;
    int nrads = 0;
    double minrad = 0.0, maxrad = 0.0;
    char *range_str = NULL;
    int maxbacklogs = 0, nthreads = -1, nsetups = -1;
    int first_nbacklogs = 1, first_nsetups = 1;
    char *setup_str = NULL;
    bool errflag = false;
    char errmsg[TMP_BUFSIZE];
    int i;
    sjcs_halo *halos = NULL;
    uint64_t nhalos = 0;
    float *r2;
    uint64_t *counts;
    sjcs_ctx *ctx = NULL;
    sjcs_query *q = NULL;
    double t0, t_total;
    char *index_str = NULL, *sched_str = NULL;
    int sched_mode = SJCS_SCHED_AUTO;
    bool use_graph = false;

    /*** argument processing (main.c:492-602) ***/
    get_option_value(argc, argv, &outfile_name, OPT_STRING_PTR, "--output-file", 0);
    get_option_range(argc, argv, &particle_beg, &particle_end, "--particle-files");
    particle_compressed = get_option_flag(argc, argv, "--compressed");
    get_option_value(argc, argv, &halo_name, OPT_STRING_PTR, "--halo-file", 0);
    get_option_value(argc, argv, &halo_filter_name, OPT_STRING_PTR, "--filter-file", 0);

    get_option_value(argc, argv, &range_str, OPT_STRING_PTR, "--radius", 0);
    if (range_str != NULL) {
        char *delimp;
        minrad = strtod(range_str, NULL);
        if ((delimp = strchr(range_str, ':')) != NULL) {
            maxrad = strtod(delimp + 1, NULL);
            if ((delimp = strrchr(range_str, ':')) != NULL)
                nrads = (int)strtol(delimp + 1, NULL, 10);
        }
    }
    if (range_str == NULL || nrads <= 0 || minrad <= 0 || maxrad <= 0) {
        set_error(&errflag, errmsg,
                  "# of ranges, minimum range, maximum range must be > 0.\n"
                  "      use --radius and fix.\n");
    } else if (minrad == maxrad) {
        set_error(&errflag, errmsg,
                  "minimum range must be <  maximum range.\n"
                  "      use --radius and fix.\n");
    }
    if (minrad > maxrad) {
        double t = minrad;
        minrad = maxrad;
        maxrad = t;
    }

    get_option_value(argc, argv, &maxbacklogs, OPT_INT, "--backlog", 0);
    if (maxbacklogs < 0) {
        set_error(&errflag, errmsg,
                  "max # of backlog indexes must be >= 0.\n"
                  "      use --backlog and fix.\n");
    }
    get_option_value(argc, argv, &nthreads, OPT_INT, "--thread", 0);
    get_option_value(argc, argv, &nsetups, OPT_INT, "--next-setup", 0);
    /* GPU options (not in the reference) */
    get_option_value(argc, argv, &index_str, OPT_STRING_PTR, "--index", 0);
    get_option_value(argc, argv, &sched_str, OPT_STRING_PTR, "--schedule", 0);
    g_autotune = get_option_flag(argc, argv, "--autotune");
    use_graph = get_option_flag(argc, argv, "--graph");
    if (index_str != NULL) {
        if (strcmp(index_str, "grid") == 0)
            g_index_kind = SJCS_INDEX_GRID;
        else if (strcmp(index_str, "morton") == 0)
            g_index_kind = SJCS_INDEX_MORTON;
        else if (strcmp(index_str, "learned") == 0)
            g_index_kind = SJCS_INDEX_LEARNED;
        else
            set_error(&errflag, errmsg, "ERROR: --index must be grid, morton or learned");
    }
    if (sched_str != NULL) {
        if (strcmp(sched_str, "auto") == 0)
            sched_mode = SJCS_SCHED_AUTO;
        else if (strcmp(sched_str, "static") == 0)
            sched_mode = SJCS_SCHED_STATIC;
        else if (strcmp(sched_str, "queue") == 0)
            sched_mode = SJCS_SCHED_QUEUE;
        else
            set_error(&errflag, errmsg, "ERROR: --schedule must be auto, static or queue");
    }
    if (nthreads < 1) {
        set_error(&errflag, errmsg,
                  "# of threads must be >= 1.\n"
                  "      use --thread and fix.\n");
    }
    if (nsetups < 1) {
        set_error(&errflag, errmsg,
                  "# of backlog index construction threads must be >= 1.\n"
                  "      use --next-setup and fix.\n");
    }
    get_option_value(argc, argv, &setup_str, OPT_STRING_PTR, "--first-setup", 0);
    if (setup_str != NULL) {
        char *delimp;
        first_nbacklogs = (int)strtol(setup_str, NULL, 10);
        if ((delimp = strchr(setup_str, ':')) != NULL)
            first_nsetups = (int)strtol(delimp + 1, NULL, 10);
    }
    if (maxbacklogs == 0) {
        if (nthreads < nsetups) {
            set_error(&errflag, errmsg,
                      "in noBacklogExecution; # of threads must be"
                      ">= # of index construction threads.\n"
                      "      use --thread, --next-setup and fix.\n");
        }
    } else {
        if ((nthreads < (nsetups + 1) || nthreads < (first_nsetups + 1))) {
            set_error(&errflag, errmsg,
                      "in withBacklogExecution; # of threads must be"
                      "> # of index construction threads.\n"
                      "      use --thread, --next-setup, --first-setup and fix.\n");
        }
        if (maxbacklogs < first_nbacklogs) {
            set_error(&errflag, errmsg,
                      "in withBacklogExecution; max # of backlog indexes must be"
                      "> # of first backlog indexes.\n"
                      "      use --backlog, --first-setup and fix.\n");
        }
    }
    if (particle_beg <= 0) {
        set_error(&errflag, errmsg,
                  "particle file is missing.\n"
                  "      use --particle-files and fix.\n");
    }
    if (halo_name == NULL) {
        set_error(&errflag, errmsg,
                  "halo file is missing.\n"
                  "      use --halo-file and fix.\n");
    }

    puts("\n--execution info--");
    printf("  particle files (compressed = %s): \n", BOOL2STRING(particle_compressed));
    for (i = particle_beg; i < particle_end; i++)
        printf("   |- %s\n", argv[i]);
    printf("  halo file = %s\n"
           "  halo filter file = %s\n"
           "  # of threads in thread pool = %d\n"
           "  # of index construction threads = %d\n"
           "  # of radiuses = %d\n"
           "   |- minimum = %f, maximum = %f\n"
           "  max # of backlog indexes = %d\n"
           "  %s# of first backlog indexes = %d\n"
           "  %s# of first index construction threads = %d\n",
           halo_name ? halo_name : "(null)", halo_filter_name ? halo_filter_name : "(null)", nthreads, nsetups,
           nrads, minrad, maxrad, maxbacklogs, (maxbacklogs == 0) ? "! ignored ! " : "", first_nbacklogs,
           (maxbacklogs == 0) ? "! ignored ! " : "", first_nsetups);
    fflush(stdout);

    if (errflag) {
        fprintf(stderr, "\n => %s\n", errmsg);
        usage_exit(argv);
    }
    g_compressed = particle_compressed;
    if (particle_compressed && use_graph) {
        puts("  (--graph captures steps over decoded particle files; compressed files run uncaptured)");
        use_graph = false;
    }

    /*** initialize ***/
    if (sjcs_ctx_create(0, &ctx) != SJCS_OK)
        die_lib("GPU context");
    /* page-lock the file staging slots and grow the device pool for the
     * largest particle file while the halo file is parsed */
    {
        uint64_t n, maxn = 0;
        int k;
        for (k = particle_beg; k < particle_end; ++k)
            if (sjcs_particle_file_count(argv[k], &n) == 0 && n > maxn)
                maxn = n;
        g_prepare.ctx = ctx;
        g_prepare.n = particle_compressed || use_graph ? 0 : maxn;
        g_prepare.started = g_prepare.n && pthread_create(&g_prepare.th, NULL, prepare_files, &g_prepare) == 0;
    }

    t0 = now_us();
    if (halo_filter_name == NULL) {
        if (sjcs_read_halos(halo_name, &halos, &nhalos, nthreads) != 0) {
            fprintf(stderr, "%s\n", sjcs_host_last_error());
            exit(EXIT_FAILURE);
        }
    } else {
        if (sjcs_read_and_filter_halos(halo_name, halo_filter_name, &halos, &nhalos) != 0) {
            fprintf(stderr, "%s\n", sjcs_host_last_error());
            exit(EXIT_FAILURE);
        }
    }
    print_ms(">>>> halo data reading time", t0);
    printf("  # of halos = %lu\n", (unsigned long)nhalos);
    if (g_prepare.started)
        pthread_join(g_prepare.th, NULL); /* a failed preparation only means a slower first file */

    r2 = malloc(sizeof(float) * nrads);
    if (sjcs_radius_table(minrad, maxrad, nrads, r2) != SJCS_OK)
        die_lib("radius table");
    counts = calloc(1, sizeof(uint64_t) * (size_t)nrads * (nhalos ? nhalos : 1));
    if (!r2 || !counts) {
        fprintf(stderr, "ERROR: memory shortage\n");
        exit(EXIT_FAILURE);
    }
    if (sjcs_query_create(ctx, nhalos ? halos[0].point : NULL, sizeof(sjcs_halo), nhalos, r2, nrads,
                          SJCS_QUERY_PERIODIC, &q) != SJCS_OK)
        die_lib("halo upload");
    if (sched_mode != SJCS_SCHED_AUTO) {
        sjcs_schedule sc;
        memset(&sc, 0, sizeof(sc));
        sc.mode = sched_mode;
        if (sjcs_query_set_schedule(ctx, q, &sc) != SJCS_OK)
            die_lib("schedule");
    }
    if (index_str || sched_str || g_autotune || use_graph)
        printf("  GPU: index %s, schedule %s%s%s\n", index_str ? index_str : "grid", sched_str ? sched_str : "auto",
               g_autotune ? ", autotuned" : "", use_graph ? ", captured file steps" : "");

    /*** execution ***/
    t_total = now_us();
    {
        const float radius_hint = (float)sqrt((double)r2[nrads - 1]);
        char **files = &argv[particle_beg];
        const int nfiles = particle_end - particle_beg;
        if (use_graph)
            graph_steps(ctx, q, files, nfiles, radius_hint);
        else if (maxbacklogs == 0)
            no_backlog(ctx, q, files, nfiles, radius_hint);
        else
            with_backlog(ctx, q, files, nfiles, maxbacklogs, first_nbacklogs, radius_hint);
    }
    if (sjcs_query_read_counts(ctx, q, counts, 1) != SJCS_OK)
        die_lib("count read-back");
    print_ms(">>>> total searching time", t_total);

    /*** result processing ***/
    t0 = now_us();
    fflush(stdout);
    if (sjcs_write_result(outfile_name, halos, nhalos, r2, nrads, counts, nthreads) != 0) {
        fprintf(stderr, "%s\n", sjcs_host_last_error());
        exit(EXIT_FAILURE);
    }
    print_ms(">>>> result writing time", t0);

    sjcs_query_destroy(q);
    sjcs_ctx_destroy(ctx);
    sjcs_host_free_halos(halos);
    free(r2);
    free(counts);
    return 0;
}
