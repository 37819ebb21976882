/*
 * CLI helpers with the reference's behaviour (include/opt_parser.h,
 * include/results_writer.h): the option lists of mpi_cc_benchmark and the
 * CSV layout its results are appended to.  The golden fixtures in
 * tests/golden/ (made by the reference's own opt_parser.c and
 * results_writer.c) pin both.
 */
#include <ctype.h>
#include <errno.h>
#include <limits.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <sys/types.h>

#include "opt_parser.h"
#include "results_writer.h"

/* ---------------------------------------------------------- opt parser */

void opt_int_list_init(OptIntList *l)
{
    if (l) {
        l->values = NULL;
        l->size = l->capacity = 0;
    }
}

void opt_int_list_free(OptIntList *l)
{
    if (l) {
        free(l->values);
        opt_int_list_init(l);
    }
}

int opt_int_list_append(OptIntList *l, int value)
{
    if (!l || value <= 0)
        return -1;
    if (l->size == l->capacity) {
        size_t nc = l->capacity ? l->capacity * 2 : 8;
        int *p = (int *)realloc(l->values, nc * sizeof(int));
        if (!p)
            return -1;
        l->values = p;
        l->capacity = nc;
    }
    l->values[l->size++] = value;
    return 0;
}

static int int_cmp(const void *a, const void *b)
{
    int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

void opt_int_list_sort_unique(OptIntList *l)
{
    if (!l || l->size == 0)
        return;
    qsort(l->values, l->size, sizeof(int), int_cmp);
    size_t w = 1;
    for (size_t r = 1; r < l->size; ++r)
        if (l->values[r] != l->values[w - 1])
            l->values[w++] = l->values[r];
    l->size = w;
}

int opt_parse_positive_int(const char *text, int *out)
{
    if (!text || !*text || !out)
        return -1;
    char *end = NULL;
    errno = 0;
    long v = strtol(text, &end, 10);
    if (errno || end == text || *end != '\0' || v <= 0 || v > INT_MAX)
        return -1;
    *out = (int)v;
    return 0;
}

/* "a" or "a:b" or "a:b:step" -> values appended to l. */
static int parse_token(const char *tok, OptIntList *l)
{
    char *s = strdup(tok);
    if (!s)
        return -1;
    int rc = -1;
    char *c1 = strchr(s, ':');
    if (!c1) {
        int x;
        rc = (opt_parse_positive_int(s, &x) == 0 && opt_int_list_append(l, x) == 0) ? 0 : -1;
        free(s);
        return rc;
    }
    *c1 = '\0';
    char *c2 = strchr(c1 + 1, ':');
    if (c2)
        *c2 = '\0';
    int a, b, step = 1;
    if (opt_parse_positive_int(s, &a) == 0 && opt_parse_positive_int(c1 + 1, &b) == 0 &&
        (!c2 || opt_parse_positive_int(c2 + 1, &step) == 0) && a <= b) {
        rc = 0;
        for (long long x = a; x <= b; x += step) {
            if (opt_int_list_append(l, (int)x) != 0) {
                rc = -1;
                break;
            }
            if (x > (long long)INT_MAX - step)
                break;
        }
    }
    free(s);
    return rc;
}

static char *trim_ws(char *t)
{
    while (isspace((unsigned char)*t))
        t++;
    size_t n = strlen(t);
    while (n > 0 && isspace((unsigned char)t[n - 1]))
        t[--n] = '\0';
    return t;
}

int opt_parse_range_list(const char *spec, OptIntList *l, const char *label)
{
    if (!spec || !l)
        return -1;
    const char *what = label ? label : "value";
    char *copy = strdup(spec);
    if (!copy)
        return -1;
    char *save = NULL;
    char *tok = strtok_r(copy, ",", &save);
    if (!tok) {
        fprintf(stderr, "Invalid %s specification: '%s'\n", what, spec);
        free(copy);
        return -1;
    }
    for (; tok; tok = strtok_r(NULL, ",", &save)) {
        char *t = trim_ws(tok);
        if (!*t || parse_token(t, l) != 0) {
            fprintf(stderr, "Invalid %s specification near '%s'\n", what, t);
            free(copy);
            return -1;
        }
    }
    free(copy);
    if (l->size == 0) {
        fprintf(stderr, "No %s provided.\n", label ? label : "values");
        return -1;
    }
    opt_int_list_sort_unique(l);
    return 0;
}

/* ------------------------------------------------------ results writer */

int results_writer_ensure_directory(const char *path)
{
    if (!path || !*path)
        return 0;
    char buf[PATH_MAX];
    size_t n = strlen(path);
    if (n >= sizeof(buf)) {
        errno = ENAMETOOLONG;
        return -1;
    }
    memcpy(buf, path, n + 1);
    while (n > 1 && buf[n - 1] == '/')
        buf[--n] = '\0';
    for (char *p = buf + 1; *p; ++p) {
        if (*p != '/')
            continue;
        *p = '\0';
        int bad = mkdir(buf, 0755) != 0 && errno != EEXIST;
        *p = '/';
        if (bad)
            return -1;
    }
    if (mkdir(buf, 0755) != 0 && errno != EEXIST)
        return -1;
    return 0;
}

int results_writer_join_path(char *dest, size_t size, const char *dir, const char *file)
{
    if (!dest || !dir || !file) {
        errno = EINVAL;
        return -1;
    }
    size_t dl = strlen(dir);
    int w = snprintf(dest, size, (dl > 0 && dir[dl - 1] != '/') ? "%s/%s" : "%s%s", dir, file);
    if (w < 0 || (size_t)w >= size) {
        errno = ENAMETOOLONG;
        return -1;
    }
    return 0;
}

int results_writer_matrix_stem(const char *matrix_path, char *dest, size_t size)
{
    if (!dest || size == 0) {
        errno = EINVAL;
        return -1;
    }
    dest[0] = '\0';
    const char *p = matrix_path ? matrix_path : "";
    const char *slash = strrchr(p, '/');
    const char *base = slash ? slash + 1 : p;
    if (!*base)
        base = "graph";
    size_t n = strlen(base);
    if (n + 1 > size) {
        errno = ENAMETOOLONG;
        return -1;
    }
    memcpy(dest, base, n + 1);
    char *dot = strrchr(dest, '.');
    if (dot && dot != dest)
        *dot = '\0';
    if (!dest[0]) {
        if (size < 6) {
            errno = ENAMETOOLONG;
            return -1;
        }
        strcpy(dest, "graph");
    }
    return 0;
}

int results_writer_build_results_path(char *dest, size_t size, const char *output_dir,
                                      const char *prefix, const char *matrix_path)
{
    if (!dest || size == 0 || !output_dir || !prefix) {
        errno = EINVAL;
        return -1;
    }
    char stem[PATH_MAX];
    if (results_writer_matrix_stem(matrix_path, stem, sizeof(stem)) != 0)
        return -1;
    char file[PATH_MAX];
    int w = snprintf(file, sizeof(file), "%s_%s.csv", prefix, stem);
    if (w < 0 || (size_t)w >= sizeof(file)) {
        errno = ENAMETOOLONG;
        return -1;
    }
    return results_writer_join_path(dest, size, output_dir, file);
}

/* A CSV held as rows of cells; every row has `ncols` cells. */
typedef struct {
    char **cells; /* row-major [rows][ncols] */
    size_t rows, ncols, cap_rows;
    char **head;
} table;

static char *dup_s(const char *s)
{
    size_t n = strlen(s);
    char *d = (char *)malloc(n + 1);
    if (d)
        memcpy(d, s, n + 1);
    return d;
}

static void table_free(table *t)
{
    for (size_t i = 0; i < t->rows * t->ncols; ++i)
        free(t->cells[i]);
    free(t->cells);
    for (size_t c = 0; c < t->ncols; ++c)
        free(t->head[c]);
    free(t->head);
}

/* Splits a line on commas (no quoting, as the reference). */
static char **split_line(const char *line, size_t *count)
{
    size_t n = 1;
    for (const char *p = line; *p; ++p)
        n += (*p == ',');
    char **f = (char **)calloc(n, sizeof(char *));
    if (!f)
        return NULL;
    const char *start = line;
    size_t k = 0;
    for (const char *p = line;; ++p) {
        if (*p == ',' || *p == '\0') {
            size_t len = (size_t)(p - start);
            f[k] = (char *)malloc(len + 1);
            if (!f[k]) {
                for (size_t i = 0; i < k; ++i)
                    free(f[i]);
                free(f);
                return NULL;
            }
            memcpy(f[k], start, len);
            f[k][len] = '\0';
            k++;
            if (*p == '\0')
                break;
            start = p + 1;
        }
    }
    *count = k;
    return f;
}

static int table_add_row(table *t, char **fields, size_t nf)
{
    if (t->rows == t->cap_rows) {
        size_t nc = t->cap_rows ? t->cap_rows * 2 : 16;
        char **p = (char **)realloc(t->cells, nc * t->ncols * sizeof(char *));
        if (!p)
            return -1;
        t->cells = p;
        t->cap_rows = nc;
    }
    for (size_t c = 0; c < t->ncols; ++c) {
        char *cell = c < nf ? fields[c] : dup_s("");
        if (c < nf)
            fields[c] = NULL;
        if (!cell)
            return -1;
        t->cells[t->rows * t->ncols + c] = cell;
    }
    t->rows++;
    return 0;
}

static void chomp(char *s)
{
    size_t n = strlen(s);
    while (n > 0 && (s[n - 1] == '\n' || s[n - 1] == '\r'))
        s[--n] = '\0';
}

static results_writer_status write_fresh(const char *filename, const char *column,
                                         const double *values, size_t count)
{
    FILE *f = fopen(filename, "w");
    if (!f)
        return RESULTS_WRITER_IO_ERROR;
    int bad = fprintf(f, "%s\n", column) < 0;
    for (size_t i = 0; i < count && !bad; ++i)
        bad = fprintf(f, "%.6f\n", values[i]) < 0;
    bad |= fclose(f) != 0;
    return bad ? RESULTS_WRITER_IO_ERROR : RESULTS_WRITER_OK;
}

results_writer_status append_times_column(const char *filename, const char *column,
                                          const double *values, size_t count)
{
    if (!filename || !column || (!values && count > 0))
        return RESULTS_WRITER_INVALID_ARGS;
    FILE *f = fopen(filename, "r");
    if (!f)
        return errno == ENOENT ? write_fresh(filename, column, values, count)
                               : RESULTS_WRITER_IO_ERROR;
    char *line = NULL;
    size_t cap = 0;
    if (getline(&line, &cap, f) < 0) {
        free(line);
        fclose(f);
        return write_fresh(filename, column, values, count);
    }
    chomp(line);
    table t;
    memset(&t, 0, sizeof(t));
    t.head = split_line(line, &t.ncols);
    results_writer_status st = RESULTS_WRITER_OK;
    if (!t.head) {
        st = RESULTS_WRITER_MEMORY_ERROR;
        goto done;
    }
    while (getline(&line, &cap, f) >= 0) {
        chomp(line);
        size_t nf = 0;
        char **fields = split_line(line, &nf);
        if (!fields || table_add_row(&t, fields, nf) != 0) {
            if (fields) {
                for (size_t i = 0; i < nf; ++i)
                    free(fields[i]);
                free(fields);
            }
            st = RESULTS_WRITER_MEMORY_ERROR;
            goto done;
        }
        for (size_t i = 0; i < nf; ++i)
            free(fields[i]);
        free(fields);
    }
    fclose(f);
    f = NULL;
    {
        size_t target = t.ncols;
        for (size_t c = 0; c < t.ncols; ++c)
            if (strcmp(t.head[c], column) == 0) {
                target = c;
                break;
            }
        size_t total_rows = t.rows;
        size_t first_value_row = 0;
        if (target < t.ncols) { /* existing column: new rows below the table */
            first_value_row = t.rows;
            total_rows = t.rows + count;
        } else if (count > t.rows) {
            total_rows = count;
        }
        FILE *o = fopen(filename, "w");
        if (!o) {
            st = RESULTS_WRITER_IO_ERROR;
            goto done;
        }
        int bad = 0;
        const size_t out_cols = t.ncols + (target == t.ncols ? 1 : 0);
        for (size_t c = 0; c < out_cols && !bad; ++c)
            bad = fprintf(o, "%s%s", c < t.ncols ? t.head[c] : column,
                          c + 1 < out_cols ? "," : "") < 0;
        bad |= fprintf(o, "\n") < 0;
        for (size_t r = 0; r < total_rows && !bad; ++r) {
            for (size_t c = 0; c < out_cols && !bad; ++c) {
                char buf[64];
                const char *cell = "";
                if (c == target && r >= first_value_row && r - first_value_row < count) {
                    snprintf(buf, sizeof(buf), "%.6f", values[r - first_value_row]);
                    cell = buf;
                } else if (c < t.ncols && r < t.rows) {
                    cell = t.cells[r * t.ncols + c];
                }
                bad = fprintf(o, "%s%s", cell, c + 1 < out_cols ? "," : "") < 0;
            }
            bad |= fprintf(o, "\n") < 0;
        }
        bad |= fclose(o) != 0;
        if (bad)
            st = RESULTS_WRITER_IO_ERROR;
    }
done:
    if (f)
        fclose(f);
    free(line);
    table_free(&t);
    return st;
}
