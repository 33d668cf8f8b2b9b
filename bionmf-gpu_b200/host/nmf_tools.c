/*
 * nmf_tools.c -- the two utilities NMF-mGPU ships beside its solver, on this
 * project's matrix I/O (nmfio.c).  One source, two programs (built with
 * -DNMF_TOOL_GENERATE or -DNMF_TOOL_CONVERT):
 *
 * generate_matrix <output_filename> <rows> <columns> [ -e <native> ] [ <max_value> ]
 *     (reference: src/tools/generate_matrix.c:290-446)
 *     Writes a rows x columns matrix of uniform values in [0, max_value]
 *     (default 1.0): every entry, row by row, is (float)random() /
 *     (float)RAND_MAX * max_value in single precision, from glibc's
 *     srandom(seed) generator -- the reference's formula and order, so the same
 *     seed gives the same matrix.  The seed is $NMFB_SEED when set, else read
 *     from /dev/urandom (the reference's get_seed without FIXED_INIT,
 *     src/common.c:1218-1258).  max_value must lie in (FLT_MIN, FLT_MAX).
 *     The file is written exactly as named, untagged, in the format of -e
 *     (absent: ASCII text, 0: non-native binary, 1: native binary).
 *
 * file_converter <filename> [ -b <native> ] [ -cr ] [ -e <native> ]
 *     (reference: src/tools/file_converter.c:160-309)
 *     Loads <filename> (ASCII text unless -b: 0 = non-native binary, 1 =
 *     native; -c / -r: numeric column headers / row labels in text input) and
 *     writes it with its tags to "<filename><ext>" in the output format of -e,
 *     ext being ".txt", ".dat" or ".native.dat".
 *
 * Both accept the solver's other option letters (-k -i -j -t -z) and ignore
 * them, as the reference's shared argument parser does (src/common.c:847-1119).
 * Exit status: EXIT_SUCCESS or EXIT_FAILURE, messages on stderr.
 */
#define _GNU_SOURCE 1
#include <errno.h>
#include <float.h>
#include <getopt.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include "nmfio.h"

#if !defined(NMF_TOOL_GENERATE) && !defined(NMF_TOOL_CONVERT)
#error "build with -DNMF_TOOL_GENERATE or -DNMF_TOOL_CONVERT"
#endif

struct tool_args {
    int in_fmt, out_fmt, num_hdrs, num_lbls, help;
};

static int parse_format(const char *arg, int *fmt, const char *what)
{
    char *end = NULL;
    errno = 0;
    long v = strtol(arg, &end, 10);
    if (*end || errno || v < 0) {
        fprintf(stderr, "Error: Invalid binary mode for %s: '%s'\nIt must be a non-negative integer value.\n", what,
                arg);
        return -1;
    }
    *fmt = v ? NMFIO_NATIVE : NMFIO_BINARY;
    return 0;
}

/* The solver's option set: formats and tag flags are used, the rest skipped. */
static int parse_options(int argc, char **argv, struct tool_args *a)
{
    memset(a, 0, sizeof(*a));
    a->in_fmt = a->out_fmt = NMFIO_ASCII;
    int opt;
    opterr = 0;
    while ((opt = getopt(argc, argv, "+:B:b:CcE:e:HhI:i:J:j:K:k:RrT:t:Z:z:")) != -1) {
        switch (opt) {
        case 'B': case 'b':
            if (parse_format(optarg, &a->in_fmt, "input file")) return -1;
            break;
        case 'E': case 'e':
            if (parse_format(optarg, &a->out_fmt, "output file(s)")) return -1;
            break;
        case 'C': case 'c': a->num_hdrs = 1; break;
        case 'R': case 'r': a->num_lbls = 1; break;
        case 'H': case 'h': a->help = 1; break;
        case 'I': case 'i': case 'J': case 'j': case 'K': case 'k': case 'T': case 't': case 'Z': case 'z':
            break;   /* read for compatibility, ignored */
        case ':':
            fprintf(stderr, "Error: option -%c requires an argument.\n", optopt);
            return -1;
        default:
            fprintf(stderr, "Error: invalid option '-%c'.\n", optopt);
            return -1;
        }
    }
    return 0;
}

/* Operands and options may come in any order (the reference's parser lets
 * getopt permute them): options, with their arguments, are moved in front of
 * the operands, which are returned in their order. */
static int split_args(int argc, char **argv, struct tool_args *a, char **operands, int max_ops, int *nops)
{
    char *args[256];
    int na = 0, nop = 0;
    if (argc > 255) {
        fprintf(stderr, "Error: too many arguments.\n");
        return -1;
    }
    args[na++] = argv[0];
    /* options first, operands after: a stable partition that keeps option
     * arguments with their options */
    for (int i = 1; i < argc; i++) {
        const char *s = argv[i];
        if (s[0] == '-' && s[1] != '\0') {
            args[na++] = argv[i];
            char const o = s[1];
            int const takes = strchr("BbEeIiJjKkTtZz", o) != NULL && s[2] == '\0';
            if (takes && i + 1 < argc) args[na++] = argv[++i];
        } else {
            if (nop == max_ops) {
                fprintf(stderr, "Error: too many arguments.\n");
                return -1;
            }
            operands[nop++] = argv[i];
        }
    }
    if (parse_options(na, args, a)) return -1;
    *nops = nop;
    return 0;
}

#ifdef NMF_TOOL_GENERATE
static uint32_t tool_seed(void)
{
    const char *s = getenv("NMFB_SEED");
    if (s && *s) return (uint32_t)strtoul(s, NULL, 10);
    uint32_t seed = 0;
    FILE *f = fopen("/dev/urandom", "rb");
    if (!f || fread(&seed, sizeof(seed), 1, f) != 1) {
        struct timeval tv;
        gettimeofday(&tv, NULL);
        seed = (uint32_t)tv.tv_usec;
    }
    if (f) fclose(f);
    return seed;
}

static int parse_dim(const char *arg, const char *what, uint32_t *out)
{
    char *end = NULL;
    errno = 0;
    long long v = strtoll(arg, &end, 10);
    if (*end || errno || v <= 0 || v > 0x7fffffffLL) {
        fprintf(stderr, "Error. Invalid number of %s: '%s'\nIt must be a positive integer.\n", what, arg);
        return -1;
    }
    *out = (uint32_t)v;
    return 0;
}

int main(int argc, char **argv)
{
    struct tool_args a;
    char *ops[4];
    int nops = 0;
    if (split_args(argc, argv, &a, ops, 4, &nops)) return EXIT_FAILURE;
    if (a.help) {
        printf("Tool to generate (in CPU) a matrix with random values\n\n"
               "Usage:\n\t%s <output_filename> <rows> <columns> [ -e <native_format> ] [ <max_value> ]\n"
               "\t%s -h\n\n<max_value>\tRange for random values: [0.0 ... <max_value>] (default 1).\n"
               "-e <native>\tBinary output: 0 = non-native (LE double), 1 = native. Default: ASCII text.\n"
               "Environment: NMFB_SEED (generator seed; default from /dev/urandom).\n\n", argv[0], argv[0]);
        return EXIT_SUCCESS;
    }
    if (nops < 3) {
        fprintf(stderr, "Error: No matrix dimensions. Not enough arguments.\nSee help (option '-h').\n");
        return EXIT_FAILURE;
    }
    uint32_t rows = 0, cols = 0;
    if (parse_dim(ops[1], "rows", &rows) || parse_dim(ops[2], "columns", &cols)) return EXIT_FAILURE;
    if ((uint64_t)rows * cols > (uint64_t)0x7fffffff) {
        fprintf(stderr, "Error: output matrix will be too large.\n");
        return EXIT_FAILURE;
    }
    float maxv = 1.0f;
    if (nops >= 4) {
        char *end = NULL;
        errno = 0;
        float const v = strtof(ops[3], &end);
        if (*end || errno || !isfinite(v)) {
            fprintf(stderr, "Error: invalid maximum value: '%s'\n", ops[3]);
            return EXIT_FAILURE;
        }
        if (v <= FLT_MIN || v >= FLT_MAX) {
            fprintf(stderr, "Error: invalid maximum value: %g\nValid values are in range (%g .. %g).\n", v, FLT_MIN,
                    FLT_MAX);
            return EXIT_FAILURE;
        }
        maxv = v;
    }
    float *M = (float *)malloc((size_t)rows * cols * sizeof(float));
    if (!M) {
        fprintf(stderr, "Error: malloc(%zu items) failed\n", (size_t)rows * cols);
        return EXIT_FAILURE;
    }
    printf("Generating a %u-by-%u data matrix (%zu items), with random values in range [0 .. %g]...\n", rows, cols,
           (size_t)rows * cols, maxv);
    if (rows == 1 || cols == 1)
        fprintf(stderr, "\nNote, however, that (row or column) vectors are not a valid input for the NMF algorithm.\n");
    srandom(tool_seed());
    float const denom = (float)RAND_MAX;
    for (size_t e = 0; e < (size_t)rows * cols; e++) {
        float const num = (float)random();
        M[e] = (num / denom) * maxv;
    }
    int const rc = nmfio_save(ops[0], a.out_fmt, M, rows, cols, cols, 0, NULL);
    free(M);
    if (rc) {
        fprintf(stderr, "Error writing '%s': %s\n", ops[0], nmfio_error());
        return EXIT_FAILURE;
    }
    return EXIT_SUCCESS;
}
#endif /* NMF_TOOL_GENERATE */

#ifdef NMF_TOOL_CONVERT
int main(int argc, char **argv)
{
    struct tool_args a;
    char *ops[2];
    int nops = 0;
    if (split_args(argc, argv, &a, ops, 2, &nops)) return EXIT_FAILURE;
    if (a.help) {
        printf("\t<< ASCII-Binary file converter >>\n\n"
               "Usage:\n\t%s <filename> [ -b <native_format> ] [ -cr ] [ -e <native_format> ]\n\t%s -h\n\n"
               "<filename>\tInput data matrix.\n"
               "-b <native>\tBinary input: 0 = non-native (LE double), 1 = native. Default: ASCII text.\n"
               "-c, -r\t\tInput text file has numeric column headers / row labels.\n"
               "-e <native>\tBinary output: 0 = non-native, 1 = native. Default: ASCII text.\n"
               "Output: <filename><ext>, ext = .txt, .dat or .native.dat.\n\n", argv[0], argv[0]);
        return EXIT_SUCCESS;
    }
    if (nops < 1) {
        fprintf(stderr, "Error: No input file. Not enough arguments.\nSee help (option '-h').\n");
        return EXIT_FAILURE;
    }
    nmfio_matrix m;
    if (nmfio_load(ops[0], a.in_fmt, a.num_hdrs, a.num_lbls, &m)) {
        fprintf(stderr, "Error reading '%s': %s\n", ops[0], nmfio_error());
        return EXIT_FAILURE;
    }
    const char *ext = nmfio_extension(a.out_fmt);
    size_t const len = strlen(ops[0]) + strlen(ext) + 1;
    char *out = (char *)malloc(len);
    if (!out) {
        nmfio_free(&m);
        fprintf(stderr, "Error setting output filename\n");
        return EXIT_FAILURE;
    }
    snprintf(out, len, "%s%s", ops[0], ext);
    printf("Output file: %s\n", out);
    int const rc = nmfio_save(out, a.out_fmt, m.data, m.rows, m.cols, m.cols, 0, &m.tags);
    if (rc) fprintf(stderr, "Error writing '%s': %s\n", out, nmfio_error());
    free(out);
    nmfio_free(&m);
    return rc ? EXIT_FAILURE : EXIT_SUCCESS;
}
#endif /* NMF_TOOL_CONVERT */
