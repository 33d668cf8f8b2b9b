/*
 * nmfio.c -- matrix file formats of NMF-mGPU (see nmfio.h).  Own implementation
 * of the formats documented by the reference (doc/user_guide.txt.md sec. 3;
 * reader validation rules of src/matrix_io/matrix_io.c:1951-2102, binary
 * signature :109-114, "%g" text output :3160-3200).
 */
#define _GNU_SOURCE 1
#include "nmfio.h"

#include <ctype.h>
#include <errno.h>
#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NMFIO_SIGNATURE 0xEDB10EA1u

static __thread char g_err[512];

static int fail(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return -1;
}

const char *nmfio_error(void) { return g_err; }

const char *nmfio_extension(int format)
{
    switch (format) {
    case NMFIO_BINARY: return ".dat";
    case NMFIO_NATIVE: return ".native.dat";
    default: return ".txt";
    }
}

/* ----------------------------------------------------------------- helpers */
static char *xstrdup_n(const char *s, size_t n)
{
    char *r = (char *)malloc(n + 1);
    if (!r) return NULL;
    memcpy(r, s, n);
    r[n] = '\0';
    return r;
}

void nmfio_free_list(char **list, uint32_t n)
{
    if (!list) return;
    for (uint32_t i = 0; i < n; i++) free(list[i]);
    free(list);
}

void nmfio_free_tags(nmfio_tags *t, uint32_t rows, uint32_t cols)
{
    if (!t) return;
    free(t->name);
    nmfio_free_list(t->headers, cols);
    nmfio_free_list(t->labels, rows);
    t->name = NULL;
    t->headers = t->labels = NULL;
}

void nmfio_free(nmfio_matrix *m)
{
    if (!m) return;
    free(m->data);
    nmfio_free_tags(&m->tags, m->rows, m->cols);
    memset(m, 0, sizeof(*m));
}

char **nmfio_make_tags(const char *prefix, uint32_t n)
{
    char **t = (char **)calloc(n ? n : 1, sizeof(char *));
    if (!t) return NULL;
    for (uint32_t i = 0; i < n; i++) {
        char buf[256];
        snprintf(buf, sizeof(buf), "%s%u", prefix, i);
        t[i] = strdup(buf);
    }
    return t;
}

/* A token is numeric when strtod consumes it entirely (empty = 0.0). */
static int parse_number(const char *s, size_t n, double *v)
{
    if (n == 0) {
        *v = 0.0;
        return 1;
    }
    char buf[128];
    if (n >= sizeof(buf)) return 0;
    memcpy(buf, s, n);
    buf[n] = '\0';
    char *end = NULL;
    errno = 0;
    double x = strtod(buf, &end);
    if (end == buf || *end != '\0' || errno == ERANGE) return 0;
    *v = x;
    return 1;
}

typedef struct {
    const char *p;
    size_t n;
} tok_t;

/* Split [s, e) on `delim`; returns the number of tokens (tokens may be empty). */
static size_t split(const char *s, const char *e, char delim, tok_t *toks, size_t cap)
{
    size_t k = 0;
    const char *t = s;
    for (const char *c = s;; c++) {
        if (c == e || *c == delim) {
            if (k < cap) {
                toks[k].p = t;
                toks[k].n = (size_t)(c - t);
            }
            k++;
            if (c == e) break;
            t = c + 1;
        }
    }
    return k;
}

static int validate(const float *data, uint32_t rows, uint32_t cols)
{
    double *colsum = (double *)calloc(cols, sizeof(double));
    if (!colsum) return fail("out of memory");
    for (uint32_t i = 0; i < rows; i++) {
        double rs = 0.0;
        for (uint32_t j = 0; j < cols; j++) {
            float const v = data[(size_t)i * cols + j];
            if (!isfinite(v)) {
                free(colsum);
                return fail("invalid value at row %u, column %u: '%g'", i, j, (double)v);
            }
            if (v < 0.0f) {
                free(colsum);
                return fail("negative value(s) detected at row %u (e.g., %g)", i, (double)v);
            }
            rs += v;
            colsum[j] += v;
        }
        if (rs < FLT_MIN) {
            free(colsum);
            return fail("\"empty\" row %u detected: all rows and columns must have at least one positive value", i);
        }
    }
    for (uint32_t j = 0; j < cols; j++)
        if (colsum[j] < FLT_MIN) {
            free(colsum);
            return fail("\"empty\" column %u detected: all rows and columns must have at least one positive value", j);
        }
    free(colsum);
    return 0;
}

static char *read_file(const char *fn, size_t *len)
{
    FILE *f = fopen(fn, "rb");
    if (!f) {
        fail("cannot open '%s': %s", fn, strerror(errno));
        return NULL;
    }
    if (fseek(f, 0, SEEK_END) != 0) {
        fclose(f);
        fail("cannot seek '%s'", fn);
        return NULL;
    }
    long const sz = ftell(f);
    rewind(f);
    char *buf = (char *)malloc((size_t)sz + 1);
    if (!buf) {
        fclose(f);
        fail("out of memory reading '%s'", fn);
        return NULL;
    }
    size_t const got = fread(buf, 1, (size_t)sz, f);
    fclose(f);
    buf[got] = '\0';
    *len = got;
    return buf;
}

/* Tag block after binary data: row labels line, column headers line, name. */
static void read_trailing_tags(const char *s, const char *e, uint32_t rows, uint32_t cols, nmfio_tags *t)
{
    const char *lines[3] = {0}, *ends[3] = {0};
    int nl = 0;
    const char *p = s;
    while (p < e && nl < 3) {
        const char *q = p;
        while (q < e && *q != '\n') q++;
        const char *qe = (q > p && q[-1] == '\r') ? q - 1 : q;
        lines[nl] = p;
        ends[nl] = qe;
        nl++;
        p = (q < e) ? q + 1 : e;
    }
    if (nl >= 1 && ends[0] > lines[0]) {
        tok_t *tk = (tok_t *)malloc(sizeof(tok_t) * (rows + 1));
        if (tk && split(lines[0], ends[0], '\t', tk, rows + 1) == rows) {
            t->labels = (char **)calloc(rows, sizeof(char *));
            for (uint32_t i = 0; t->labels && i < rows; i++) t->labels[i] = xstrdup_n(tk[i].p, tk[i].n);
        }
        free(tk);
    }
    if (nl >= 2 && ends[1] > lines[1]) {
        tok_t *tk = (tok_t *)malloc(sizeof(tok_t) * (cols + 1));
        if (tk && split(lines[1], ends[1], '\t', tk, cols + 1) == cols) {
            t->headers = (char **)calloc(cols, sizeof(char *));
            for (uint32_t j = 0; t->headers && j < cols; j++) t->headers[j] = xstrdup_n(tk[j].p, tk[j].n);
        }
        free(tk);
    }
    if (nl >= 3 && ends[2] > lines[2]) t->name = xstrdup_n(lines[2], (size_t)(ends[2] - lines[2]));
}

/* ------------------------------------------------------------------- ASCII */
static int load_ascii(const char *fn, int numeric_headers, int numeric_labels, nmfio_matrix *out)
{
    size_t len = 0;
    char *buf = read_file(fn, &len);
    if (!buf) return -1;
    /* line table */
    size_t nlines = 0, cap = 1024;
    const char **ls = (const char **)malloc(cap * sizeof(char *));
    const char **le = (const char **)malloc(cap * sizeof(char *));
    const char *p = buf, *end = buf + len;
    while (p < end) {
        const char *q = memchr(p, '\n', (size_t)(end - p));
        if (!q) q = end;
        const char *qe = (q > p && q[-1] == '\r') ? q - 1 : q;
        if (nlines == cap) {
            cap *= 2;
            ls = (const char **)realloc(ls, cap * sizeof(char *));
            le = (const char **)realloc(le, cap * sizeof(char *));
        }
        ls[nlines] = p;
        le[nlines] = qe;
        nlines++;
        p = (q < end) ? q + 1 : end;
    }
    while (nlines > 0 && le[nlines - 1] == ls[nlines - 1]) nlines--; /* trailing blank lines */
    if (nlines < 2) {
        free(ls);
        free(le);
        free(buf);
        return fail("'%s': not enough lines for a matrix (at least two rows are required)", fn);
    }
    char const delim = memchr(ls[0], '\t', (size_t)(le[0] - ls[0])) ? '\t' : ' ';
    size_t const maxtok = 1 + (size_t)(le[0] - ls[0]) + (size_t)(le[1] - ls[1]);
    tok_t *t0 = (tok_t *)malloc(sizeof(tok_t) * (maxtok + 1));
    tok_t *t1 = (tok_t *)malloc(sizeof(tok_t) * (maxtok + 1));
    size_t const n0 = split(ls[0], le[0], delim, t0, maxtok + 1);
    size_t const n1 = split(ls[1], le[1], delim, t1, maxtok + 1);
    double dv;
    /* headers: forced, or some token of the first line is not a number */
    int has_headers = numeric_headers;
    for (size_t i = 0; !has_headers && i < n0; i++)
        if (!parse_number(t0[i].p, t0[i].n, &dv)) has_headers = 1;
    /* labels: forced, or the first token of the first data line is not a number */
    const tok_t *first_data = has_headers ? t1 : t0;
    size_t const nfirst = has_headers ? n1 : n0;
    int has_labels = numeric_labels || !parse_number(first_data[0].p, first_data[0].n, &dv);
    size_t const ncols = nfirst - (size_t)has_labels;
    size_t const nrows = nlines - (size_t)has_headers;
    int rc = 0;
    nmfio_matrix m;
    memset(&m, 0, sizeof(m));
    if (ncols < 2 || nrows < 2) {
        rc = fail("'%s': both matrix dimensions must be greater than 1 (rows=%zu, columns=%zu)", fn, nrows, ncols);
        goto done;
    }
    m.rows = (uint32_t)nrows;
    m.cols = (uint32_t)ncols;
    m.data = (float *)malloc(nrows * ncols * sizeof(float));
    if (!m.data) {
        rc = fail("out of memory for a %zu x %zu matrix", nrows, ncols);
        goto done;
    }
    if (has_headers) {
        size_t off = 0;
        if (n0 == ncols + 1) {
            m.tags.name = xstrdup_n(t0[0].p, t0[0].n);
            off = 1;
        } else if (n0 != ncols) {
            rc = fail("'%s': the header line has %zu entries for %zu columns", fn, n0, ncols);
            goto done;
        }
        m.tags.headers = (char **)calloc(ncols, sizeof(char *));
        for (size_t j = 0; j < ncols; j++) m.tags.headers[j] = xstrdup_n(t0[off + j].p, t0[off + j].n);
    }
    if (has_labels) m.tags.labels = (char **)calloc(nrows, sizeof(char *));
    {
        size_t const need = ncols + (size_t)has_labels;
        tok_t *tk = (tok_t *)malloc(sizeof(tok_t) * (need + 1));
        for (size_t i = 0; i < nrows && rc == 0; i++) {
            size_t const li = i + (size_t)has_headers;
            size_t const nt = split(ls[li], le[li], delim, tk, need + 1);
            if (nt != need) {
                rc = fail("'%s': line %zu has %zu entries, expected %zu", fn, li + 1, nt, need);
                break;
            }
            if (has_labels) m.tags.labels[i] = xstrdup_n(tk[0].p, tk[0].n);
            for (size_t j = 0; j < ncols; j++) {
                const tok_t *x = &tk[j + (size_t)has_labels];
                if (!parse_number(x->p, x->n, &dv)) {
                    rc = fail("'%s': invalid numeric value at line %zu, column %zu: '%.*s'", fn, li + 1, j + 1,
                              (int)(x->n > 40 ? 40 : x->n), x->p);
                    break;
                }
                m.data[i * ncols + j] = (float)dv;
            }
        }
        free(tk);
    }
    if (rc == 0) rc = validate(m.data, m.rows, m.cols);
done:
    free(t0);
    free(t1);
    free(ls);
    free(le);
    free(buf);
    if (rc == 0)
        *out = m;
    else
        nmfio_free(&m);
    return rc;
}

/* ------------------------------------------------------------------ binary */
static int load_binary(const char *fn, int native, nmfio_matrix *out)
{
    size_t len = 0;
    char *buf = read_file(fn, &len);
    if (!buf) return -1;
    size_t pos = 0;
    uint32_t hdr[3];
    int rc = 0;
    nmfio_matrix m;
    memset(&m, 0, sizeof(m));
    size_t const nh = native ? 2 : 3;
    if (len < nh * 4) {
        free(buf);
        return fail("'%s': premature end-of-file; invalid file format", fn);
    }
    memcpy(hdr, buf, nh * 4);
    pos = nh * 4;
    if (!native && hdr[0] != NMFIO_SIGNATURE) {
        free(buf);
        return fail("'%s': invalid signature %X; invalid file format", fn, hdr[0]);
    }
    m.rows = native ? hdr[0] : hdr[1];
    m.cols = native ? hdr[1] : hdr[2];
    if (m.rows < 2 || m.cols < 2) {
        free(buf);
        return fail("'%s': both matrix dimensions must be greater than 1", fn);
    }
    size_t const nitems = (size_t)m.rows * m.cols;
    size_t const esz = native ? sizeof(float) : sizeof(double);
    if (len - pos < nitems * esz) {
        free(buf);
        return fail("'%s': premature end-of-file; invalid file format", fn);
    }
    m.data = (float *)malloc(nitems * sizeof(float));
    if (!m.data) {
        free(buf);
        return fail("out of memory");
    }
    if (native) {
        memcpy(m.data, buf + pos, nitems * sizeof(float));
    } else {
        for (size_t e = 0; e < nitems; e++) {
            double d;
            memcpy(&d, buf + pos + e * sizeof(double), sizeof(double));
            m.data[e] = (float)d;
        }
    }
    pos += nitems * esz;
    read_trailing_tags(buf + pos, buf + len, m.rows, m.cols, &m.tags);
    free(buf);
    if (!native) rc = validate(m.data, m.rows, m.cols);
    if (rc == 0)
        *out = m;
    else
        nmfio_free(&m);
    return rc;
}

int nmfio_load(const char *filename, int format, int numeric_headers, int numeric_labels, nmfio_matrix *out)
{
    if (!filename || !out) return fail("null argument");
    memset(out, 0, sizeof(*out));
    switch (format) {
    case NMFIO_ASCII: return load_ascii(filename, numeric_headers, numeric_labels, out);
    case NMFIO_BINARY: return load_binary(filename, 0, out);
    case NMFIO_NATIVE: return load_binary(filename, 1, out);
    default: return fail("unknown file format %d", format);
    }
}

/* ------------------------------------------------------------------ saving */
static void write_tag_line(FILE *f, char **tags, uint32_t n)
{
    for (uint32_t i = 0; i < n; i++) fprintf(f, "%s%s", i ? "\t" : "", tags[i] ? tags[i] : "");
}

int nmfio_save(const char *filename, int format, const float *data, uint32_t rows, uint32_t cols, size_t ld,
               int transpose, const nmfio_tags *tags)
{
    uint32_t const major = transpose ? cols : rows, minor = transpose ? rows : cols;
    char *name = tags ? tags->name : NULL;
    char **headers = tags ? (transpose ? tags->labels : tags->headers) : NULL;
    char **labels = tags ? (transpose ? tags->headers : tags->labels) : NULL;
    FILE *f = fopen(filename, format == NMFIO_ASCII ? "w" : "wb");
    if (!f) return fail("cannot create '%s': %s", filename, strerror(errno));
#define ELEM(a, b) (transpose ? data[(size_t)(b) * ld + (a)] : data[(size_t)(a) * ld + (b)])
    if (format == NMFIO_ASCII) {
        if (name) fprintf(f, "%s%s", name, headers ? "\t" : "\n");
        if (headers) {
            write_tag_line(f, headers, minor);
            fputc('\n', f);
        }
        for (uint32_t i = 0; i < major; i++) {
            if (labels) fprintf(f, "%s\t", labels[i] ? labels[i] : "");
            for (uint32_t j = 0; j < minor; j++) fprintf(f, j ? "\t%g" : "%g", (double)ELEM(i, j));
            fputc('\n', f);
        }
    } else {
        if (format == NMFIO_BINARY) {
            uint32_t const h[3] = {NMFIO_SIGNATURE, major, minor};
            fwrite(h, sizeof(uint32_t), 3, f);
            for (uint32_t i = 0; i < major; i++)
                for (uint32_t j = 0; j < minor; j++) {
                    double const d = (double)ELEM(i, j);
                    fwrite(&d, sizeof(double), 1, f);
                }
        } else {
            /* native: no transposition (the reference skips it in this mode) */
            uint32_t const h[2] = {rows, cols};
            fwrite(h, sizeof(uint32_t), 2, f);
            for (uint32_t i = 0; i < rows; i++) fwrite(data + (size_t)i * ld, sizeof(float), cols, f);
            labels = tags ? tags->labels : NULL;
            headers = tags ? tags->headers : NULL;
        }
        if (labels || headers || name) {
            uint32_t const nl = (format == NMFIO_NATIVE) ? rows : major, nc = (format == NMFIO_NATIVE) ? cols : minor;
            if (labels) write_tag_line(f, labels, nl);
            if (headers || name) {
                fputc('\n', f);
                if (headers) write_tag_line(f, headers, nc);
                if (name) fprintf(f, "\n%s", name);
            }
        }
    }
#undef ELEM
    if (ferror(f)) {
        fclose(f);
        return fail("write error on '%s'", filename);
    }
    if (fclose(f) != 0) return fail("cannot close '%s': %s", filename, strerror(errno));
    return 0;
}
