/*
 * nmf_oracle.c -- CPU restatement of the NMF-mGPU single-GPU KL-NMF loop.
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker of the CUDA engine and the
 * timed CPU baseline ("port").  Never linked into the product.
 * Every function cites the reference file:line it restates (see the header
 * and nmf_oracle_core.inc).  Built without -ffast-math so that NaN handling
 * and IEEE division are exact.
 */
#define _DEFAULT_SOURCE 1
#include "nmf_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* R_MIN of the single-precision build (include/real_type.h:120-124). */
#define ORACLE_R_MIN FLT_MIN

#define REAL float
#define SFX f32
#include "nmf_oracle_core.inc"
#undef REAL
#undef SFX

#define REAL double
#define SFX f64
#include "nmf_oracle_core.inc"
#undef REAL
#undef SFX

void oracle_init_random(uint32_t seed, uint32_t n, uint32_t m, uint32_t k,
                        float *W, size_t ldw, float *H, size_t ldh)
{
    /* src/NMF_routines.c:206-233 (srandom) and :299-307 (values). */
    srandom(seed);
    for (uint32_t i = 0; i < n; i++) {
        float *p = W + (size_t)i * ldw;
        for (uint32_t c = 0; c < k; c++)
            p[c] = ((float)random()) / ((float)RAND_MAX) + FLT_MIN;
        for (size_t c = k; c < ldw; c++)
            p[c] = 1.0f;
    }
    for (uint32_t j = 0; j < m; j++) {
        float *p = H + (size_t)j * ldh;
        for (uint32_t c = 0; c < k; c++)
            p[c] = ((float)random()) / ((float)RAND_MAX) + FLT_MIN;
        for (size_t c = k; c < ldh; c++)
            p[c] = 1.0f;
    }
}

uint64_t oracle_difference(const uint32_t *cls, const uint32_t *last, uint32_t m)
{
    /* src/common.c:1195-1209, literally O(m^2). */
    uint64_t diff = 0;
    for (uint32_t i = 0; i + 1 < m; i++)
        for (uint32_t j = i + 1; j < m; j++) {
            int const conn = (cls[j] == cls[i]);
            int const conn_last = (last[j] == last[i]);
            diff += (uint64_t)(conn != conn_last);
        }
    return diff;
}

void oracle_dot_VWH(uint32_t n, uint32_t m, uint32_t k, const float *V, size_t ldv,
                    const float *W, size_t ldw, const float *H, size_t ldh,
                    double *dot_V, double *dot_VWH)
{
    double sv = 0.0, sd = 0.0;
    #pragma omp parallel for reduction(+ : sv, sd) schedule(static)
    for (uint32_t i = 0; i < n; i++) {
        for (uint32_t j = 0; j < m; j++) {
            double wh = 0.0;
            for (uint32_t c = 0; c < k; c++)
                wh += (double)W[(size_t)i * ldw + c] * (double)H[(size_t)j * ldh + c];
            double const v = V[(size_t)i * ldv + j];
            sv += v * v;
            sd += (v - wh) * (v - wh);
        }
    }
    *dot_V = sv;
    *dot_VWH = sd;
}

double oracle_kl_divergence(uint32_t n, uint32_t m, uint32_t k, const float *V, size_t ldv,
                            const float *W, size_t ldw, const float *H, size_t ldh)
{
    double d = 0.0;
    #pragma omp parallel for reduction(+ : d) schedule(static)
    for (uint32_t i = 0; i < n; i++) {
        for (uint32_t j = 0; j < m; j++) {
            double wh = 0.0;
            for (uint32_t c = 0; c < k; c++)
                wh += (double)W[(size_t)i * ldw + c] * (double)H[(size_t)j * ldh + c];
            double const v = V[(size_t)i * ldv + j];
            d += (v > 0.0 ? v * log(v / wh) : 0.0) - v + wh;
        }
    }
    return d;
}

void oracle_consensus(const uint32_t *labels, uint32_t nruns, uint32_t m, uint32_t *C)
{
    for (uint32_t a = 0; a < m; a++)
        for (uint32_t b = 0; b < m; b++) {
            uint32_t cnt = 0;
            for (uint32_t r = 0; r < nruns; r++)
                cnt += labels[(size_t)r * m + a] == labels[(size_t)r * m + b];
            C[(size_t)a * m + b] = cnt;
        }
}

double oracle_cophenetic_dist(const double *D, uint32_t m)
{
    size_t const mm = (size_t)m * m;
    double *Dw = malloc(mm * sizeof(double));
    double *coph = calloc(mm, sizeof(double));
    uint32_t *cid = malloc(m * sizeof(uint32_t));
    uint32_t *size = malloc(m * sizeof(uint32_t));
    if (!Dw || !coph || !cid || !size) {
        free(Dw); free(coph); free(cid); free(size);
        return NAN;
    }
    memcpy(Dw, D, mm * sizeof(double));
    for (uint32_t a = 0; a < m; a++) {
        cid[a] = a;
        size[a] = 1;
    }
    for (uint32_t step = 0; step + 1 < m; step++) {
        double best = INFINITY;
        uint32_t A = 0, B = 0;
        for (uint32_t a = 0; a < m; a++) {
            if (!size[a]) continue;
            for (uint32_t b = a + 1; b < m; b++)
                if (size[b] && Dw[(size_t)a * m + b] < best) {
                    best = Dw[(size_t)a * m + b];
                    A = a;
                    B = b;
                }
        }
        for (uint32_t x = 0; x < m; x++)
            for (uint32_t y = 0; y < m; y++)
                if ((cid[x] == A && cid[y] == B) || (cid[x] == B && cid[y] == A)) coph[(size_t)x * m + y] = best;
        double const na = size[A], nb = size[B];
        for (uint32_t x = 0; x < m; x++) {
            if (x == A || x == B || !size[x]) continue;
            double const d = (na * Dw[(size_t)A * m + x] + nb * Dw[(size_t)B * m + x]) / (na + nb);
            Dw[(size_t)A * m + x] = d;
            Dw[(size_t)x * m + A] = d;
        }
        for (uint32_t x = 0; x < m; x++)
            if (cid[x] == B) cid[x] = A;
        size[A] += size[B];
        size[B] = 0;
    }
    double const np = (double)m * (m - 1) / 2.0;
    double sx = 0.0, sy = 0.0;
    for (uint32_t a = 0; a < m; a++)
        for (uint32_t b = a + 1; b < m; b++) {
            sx += D[(size_t)a * m + b];
            sy += coph[(size_t)a * m + b];
        }
    double const mx = sx / np, my = sy / np;
    double cxy = 0.0, cxx = 0.0, cyy = 0.0;
    for (uint32_t a = 0; a < m; a++)
        for (uint32_t b = a + 1; b < m; b++) {
            double const x = D[(size_t)a * m + b] - mx, y = coph[(size_t)a * m + b] - my;
            cxy += x * y;
            cxx += x * x;
            cyy += y * y;
        }
    free(Dw); free(coph); free(cid); free(size);
    return (cxx > 0.0 && cyy > 0.0) ? cxy / sqrt(cxx * cyy) : 0.0;
}

double oracle_cophenetic(const uint32_t *C, uint32_t m, uint32_t nruns)
{
    size_t const mm = (size_t)m * m;
    double *D = malloc(mm * sizeof(double));
    if (!D) return NAN;
    for (uint32_t a = 0; a < m; a++)
        for (uint32_t b = 0; b < m; b++)
            D[(size_t)a * m + b] = (a == b) ? 0.0 : 1.0 - (double)C[(size_t)a * m + b] / (double)nruns;
    double const r = oracle_cophenetic_dist(D, m);
    free(D);
    return r;
}

int oracle_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
