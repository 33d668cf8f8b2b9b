/*
 * nmf_gpu_main.c -- the NMF_GPU command line on the B200 engine.
 *
 * Drop-in for the reference's single-GPU program (src/NMF_GPU.c:1034-1269):
 * same options (getopt string of src/common.c:910), same defaults
 * (include/common_defaults.h: K=2, -i 2000, -j 10, -t 40, device 0), same input
 * formats and output files (<file>_W<ext> with N x K, <file>_H<ext> with K x M,
 * tagged with "Factor_<i>" when the input has tags, src/NMF_GPU.c:933-1029) and
 * the same result lines on stdout:
 *     NMF: Algorithm converged in <n> iterations.   |   NMF: <n> iterations performed.
 *     Distance between V and W*H: <%g>
 * followed by lines the reference does not print (KL divergence, timing).
 *
 * Environment (no option letters are added to the reference's set):
 *   NMFB_SEED   seed of the CPU_RANDOM initialisation (default: /dev/urandom,
 *               as the reference's get_seed, src/common.c:1218-1258)
 *   NMFB_ARM    fused (default), fused_tf32, plain
 */
#define _GNU_SOURCE 1
#include <errno.h>
#include <getopt.h>
#include <inttypes.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>
#include <time.h>

#include "../../include/nmfb200.h"
#include "nmfio.h"

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static int usage(const char *exe)
{
    printf("\n\t<< nmf-b200: KL-NMF on NVIDIA B200 (drop-in for NMF_GPU) >>\n\n"
           "Usage:\n\t%s <filename> [ -b <native> ] [ -cr ] [ -k <factorization_rank> ] [ -i <nIters> ] "
           "[ -j <niter_test_conv> ]\n\t\t[ -t <stop_threshold> ] [ -e <native> ] [ -z <GPU_device> ]\n\t%s -h\n\n"
           "<filename>\tInput data matrix.\n"
           "-B,-b <native>\tBinary input file: 0 = non-native (LE double, signature), 1 = native.\n"
           "-C,-c\t\tInput text file has numeric column headers.\n"
           "-R,-r\t\tInput text file has numeric row labels.\n"
           "-E,-e <native>\tBinary output files (0 = non-native, 1 = native). Default: ASCII text.\n"
           "-K,-k <rank>\tFactorization rank (default: 2).\n"
           "-I,-i <nIters>\tMaximum number of iterations (default: 2000).\n"
           "-J,-j <n>\tConvergence test every <n> iterations (default: 10).\n"
           "-T,-t <n>\tStop after the classification is unchanged in <n> consecutive tests (default: 40).\n"
           "-Z,-z <device>\tGPU device (default: 0).\n"
           "-H,-h\t\tThis help.\n\n"
           "Environment: NMFB_SEED (initialisation seed), NMFB_ARM (fused | fused_tf32 | plain).\n\n",
           exe, exe);
    return EXIT_SUCCESS;
}

static int parse_uint(const char *arg, long long lo, long long hi, uint32_t *out)
{
    char *end = NULL;
    errno = 0;
    long long v = strtoll(arg, &end, 10);
    if (*end || errno || v < lo || v > hi) return -1;
    *out = (uint32_t)v;
    return 0;
}

static uint32_t seed_from_system(void)
{
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

int main(int argc, char **argv)
{
    int in_fmt = NMFIO_ASCII, out_fmt = NMFIO_ASCII, num_hdrs = 0, num_lbls = 0;
    uint32_t k = 2, n_iters = 2000, niter_test_conv = 10, stop_threshold = 40, device = 0, v;
    int opt;
    opterr = 0;
    while ((opt = getopt(argc, argv, ":B:b:CcE:e:HhI:i:J:j:K:k:RrT:t:Z:z:")) != -1) {
        switch (opt) {
        case 'B': case 'b':
            if (parse_uint(optarg, 0, 0x7fffffff, &v)) {
                fprintf(stderr, "Error: Invalid binary mode for input file: '%s'\nIt must be a non-negative integer value.\n", optarg);
                return EXIT_FAILURE;
            }
            in_fmt = v ? NMFIO_NATIVE : NMFIO_BINARY;
            break;
        case 'C': case 'c': num_hdrs = 1; break;
        case 'R': case 'r': num_lbls = 1; break;
        case 'E': case 'e':
            if (parse_uint(optarg, 0, 0x7fffffff, &v)) {
                fprintf(stderr, "Error: Invalid binary mode for output file(s): '%s'\nIt must be a non-negative integer value.\n", optarg);
                return EXIT_FAILURE;
            }
            out_fmt = v ? NMFIO_NATIVE : NMFIO_BINARY;
            break;
        case 'H': case 'h': return usage(argv[0]);
        case 'I': case 'i':
            if (parse_uint(optarg, 1, 0xffffffffLL, &n_iters)) {
                fprintf(stderr, "Error: Invalid number of iterations: '%s'\nIt must be a positive integer value.\n", optarg);
                return EXIT_FAILURE;
            }
            break;
        case 'J': case 'j':
            if (parse_uint(optarg, 1, 0xffffffffLL, &niter_test_conv)) {
                fprintf(stderr, "Error: Invalid number of iterations for convergence test: '%s'\nIt must be a positive integer value.\n", optarg);
                return EXIT_FAILURE;
            }
            break;
        case 'K': case 'k':
            if (parse_uint(optarg, 2, 256, &k)) {
                fprintf(stderr, "Error: invalid factorization rank: '%s'\nIt must be an integer value in the range [2 .. 256].\n", optarg);
                return EXIT_FAILURE;
            }
            break;
        case 'T': case 't':
            if (parse_uint(optarg, 1, 0xffffffffLL, &stop_threshold)) {
                fprintf(stderr, "Error: invalid stopping threshold '%s'\nIt must be a positive integer value.\n", optarg);
                return EXIT_FAILURE;
            }
            break;
        case 'Z': case 'z':
            if (parse_uint(optarg, 0, 0x7fffffff, &device)) {
                fprintf(stderr, "Error: invalid basis device ID number '%s'\nIt must be a non-negative integer value.\n", optarg);
                return EXIT_FAILURE;
            }
            break;
        case ':':
            fprintf(stderr, "Error: option -%c requires an argument.\nSee help (option '-h').\n", optopt);
            return EXIT_FAILURE;
        default: break;
        }
    }
    if (optind >= argc) {
        fprintf(stderr, "Error: No filename. Not enough arguments.\nSee help (option '-h').\n");
        return EXIT_FAILURE;
    }
    const char *filename = argv[optind];
    printf("\t<<< nmf-b200: Non-negative Matrix Factorization on B200 >>>\n\t\t\t\tSingle-GPU version\n");

    double const t_start = now_s();
    nmfio_matrix V;
    if (nmfio_load(filename, in_fmt, num_hdrs, num_lbls, &V) != 0) {
        fprintf(stderr, "Error reading input file: %s\n", nmfio_error());
        return EXIT_FAILURE;
    }
    printf("\tMatrix dimensions: %u x %u (%zu items)\n", V.rows, V.cols, (size_t)V.rows * V.cols);
    uint32_t const n = V.rows, m = V.cols;
    if (k > (n < m ? n : m)) {
        fprintf(stderr, "Error: invalid factorization rank: K=%u.\nIt must not be greater than any of matrix dimensions.\n", k);
        nmfio_free(&V);
        return EXIT_FAILURE;
    }
    int arm = NMFB_ARM_FUSED;
    const char *arm_env = getenv("NMFB_ARM");
    if (arm_env && !strcmp(arm_env, "plain")) arm = NMFB_ARM_PLAIN;
    if (arm_env && !strcmp(arm_env, "fused_tf32")) arm = NMFB_ARM_FUSED_TF32;
    if (arm != NMFB_ARM_PLAIN && k > 64) {
        printf("\tFactorization rank %u > 64: using the unfused kernels.\n", k);
        arm = NMFB_ARM_PLAIN;
    }
    uint32_t seed = seed_from_system();
    const char *seed_env = getenv("NMFB_SEED");
    if (seed_env) seed = (uint32_t)strtoul(seed_env, NULL, 10);

    nmfb_ctx *ctx = NULL;
    int rc = nmfb_create(&ctx, (int)device, n, m, k, arm);
    if (rc == NMFB_OK) rc = nmfb_set_V(ctx, V.data, m);
    if (rc == NMFB_OK) rc = nmfb_init_random(ctx, seed);
    if (rc != NMFB_OK) {
        fprintf(stderr, "Error setting up the GPU: %s\n", nmfb_last_error(ctx));
        nmfb_destroy(ctx);
        nmfio_free(&V);
        return EXIT_FAILURE;
    }
    printf("Starting NMF( K=%u )...\n", k);
    fflush(stdout);
    double const t_nmf = now_s();
    uint32_t iterations = 0;
    int converged = 0;
    rc = nmfb_run(ctx, n_iters, niter_test_conv, stop_threshold, &iterations, &converged);
    if (rc != NMFB_OK) {
        fprintf(stderr, "Error in NMF: %s\n", nmfb_last_error(ctx));
        nmfb_destroy(ctx);
        nmfio_free(&V);
        return EXIT_FAILURE;
    }
    double const t_done = now_s();
    if (converged)
        printf("NMF: Algorithm converged in %u iterations.\n", iterations);
    else
        printf("NMF: %u iterations performed.\n", iterations);

    float *W = (float *)malloc((size_t)n * k * sizeof(float));
    float *H = (float *)malloc((size_t)m * k * sizeof(float));
    double dot_V = 0.0, dot_VWH = 0.0, kl = 0.0;
    if (!W || !H) rc = NMFB_ENOMEM;
    if (rc == NMFB_OK) rc = nmfb_get_W(ctx, W, k);
    if (rc == NMFB_OK) rc = nmfb_get_H(ctx, H, k);
    if (rc == NMFB_OK) rc = nmfb_dot_product_VWH(ctx, &dot_V, &dot_VWH);
    if (rc == NMFB_OK) rc = nmfb_kl_divergence(ctx, &kl);
    if (rc != NMFB_OK) {
        fprintf(stderr, "Error reading results: %s\n", nmfb_last_error(ctx));
        nmfb_destroy(ctx);
        nmfio_free(&V);
        free(W);
        free(H);
        return EXIT_FAILURE;
    }
    printf("Distance between V and W*H: %g\n", sqrt(dot_VWH) / sqrt(dot_V));
    printf("KL divergence D(V || W*H): %.10g\n", kl);
    printf("NMF time: %g seconds (%g iterations/s).\n", t_done - t_nmf, (double)iterations / (t_done - t_nmf));

    /* Output files (src/NMF_GPU.c:933-1029). */
    int const tagged = V.tags.name || V.tags.headers || V.tags.labels;
    char **factors = tagged ? nmfio_make_tags("Factor_", k) : NULL;
    nmfio_tags tw = {V.tags.name, factors, V.tags.labels};
    nmfio_tags th = {V.tags.name, factors, V.tags.headers};
    size_t const fl = strlen(filename) + 32;
    char *out = (char *)malloc(fl);
    int status = EXIT_SUCCESS;
    snprintf(out, fl, "%s_W%s", filename, nmfio_extension(out_fmt));
    if (nmfio_save(out, out_fmt, W, n, k, k, 0, tagged ? &tw : NULL) != 0) {
        fprintf(stderr, "Error writing matrix W: %s\n", nmfio_error());
        status = EXIT_FAILURE;
    }
    snprintf(out, fl, "%s_H%s", filename, nmfio_extension(out_fmt));
    if (status == EXIT_SUCCESS && nmfio_save(out, out_fmt, H, m, k, k, 1, tagged ? &th : NULL) != 0) {
        fprintf(stderr, "Error writing matrix H: %s\n", nmfio_error());
        status = EXIT_FAILURE;
    }
    printf("Total elapsed time: %g seconds.\n", now_s() - t_start);
    if (status == EXIT_SUCCESS) printf("Done.\n");
    free(out);
    nmfio_free_list(factors, k);
    free(W);
    free(H);
    nmfb_destroy(ctx);
    nmfio_free(&V);
    return status;
}
