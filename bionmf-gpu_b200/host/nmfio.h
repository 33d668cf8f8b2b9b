/*
 * nmfio.h -- matrix file formats of NMF-mGPU (host side of the drop-in CLI).
 *
 * Formats (documented in the reference's doc/user_guide.txt.md, section 3):
 *   NMFIO_ASCII      tab- (or single-space-) separated text, with an optional
 *                    description string and column headers on the first line and
 *                    optional row labels at the start of every line; empty
 *                    entries read as 0.0; values written with "%g".
 *   NMFIO_BINARY     "non-native" binary: u32 signature 0xEDB10EA1, u32 rows,
 *                    u32 columns, rows*columns little-endian float64 row-major,
 *                    then the optional tags as text (row labels line, column
 *                    headers line, name).
 *   NMFIO_NATIVE     "native" binary: u32 rows, u32 columns, float32 data,
 *                    then the optional tags; no checks, no transposition.
 * Loaded data must be finite and non-negative with no all-zero row or column
 * (src/matrix_io/matrix_io.c:1951-2102).
 */
#ifndef NMFIO_H
#define NMFIO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { NMFIO_ASCII = 0, NMFIO_BINARY = 1, NMFIO_NATIVE = 2 };

typedef struct {
    char *name;        /* description string or NULL */
    char **headers;    /* column headers (cols entries) or NULL */
    char **labels;     /* row labels (rows entries) or NULL */
} nmfio_tags;

typedef struct {
    float *data;       /* rows x cols, row-major, leading dimension cols */
    uint32_t rows, cols;
    nmfio_tags tags;
} nmfio_matrix;

/* Load a matrix; returns 0 or -1 (message in nmfio_error()). */
int nmfio_load(const char *filename, int format, int numeric_headers, int numeric_labels, nmfio_matrix *out);

/* Save rows x cols from `data` (leading dimension ld).  With transpose != 0 the
 * file holds the transpose (cols rows of rows values), as the reference writes H.
 * `tags` may be NULL; for transpose, headers and labels swap roles. */
int nmfio_save(const char *filename, int format, const float *data, uint32_t rows, uint32_t cols, size_t ld,
               int transpose, const nmfio_tags *tags);

/* Tags "<prefix>0" .. "<prefix>(n-1)" (the reference's "Factor_" labels). */
char **nmfio_make_tags(const char *prefix, uint32_t n);

void nmfio_free_tags(nmfio_tags *t, uint32_t rows, uint32_t cols);
void nmfio_free_list(char **list, uint32_t n);
void nmfio_free(nmfio_matrix *m);

/* Last error message of this thread. */
const char *nmfio_error(void);

/* File-name extension of a format: ".txt", ".dat", ".native.dat". */
const char *nmfio_extension(int format);

#ifdef __cplusplus
}
#endif
#endif
