/*
 * Minimal .npy (format 1.0/2.0) reader and writer for the oracle and the
 * reference harness.  TEST INFRASTRUCTURE: nothing in the product links this.
 *
 * The reference reads its datasets through cnpy (benchmark/bench_util.hpp:250-263),
 * whose submodule is empty, so the harness needs its own .npy I/O.  Only
 * little-endian, C-ordered, 1-D or 2-D arrays are supported, which is all the
 * harness and the tests exchange.
 */
#ifndef PK_ORACLE_NPY_H
#define PK_ORACLE_NPY_H

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    char kind;        /* 'f', 'i' or 'u' */
    int word;         /* bytes per element */
    int ndim;         /* 1 or 2 */
    int64_t shape[2]; /* shape[1] == 1 for 1-D arrays */
    void *data;       /* malloc'd, caller frees */
} pk_npy;

static inline int pk_npy_read(const char *path, pk_npy *out) {
    memset(out, 0, sizeof(*out));
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    unsigned char pre[10];
    if (fread(pre, 1, 10, f) != 10 || memcmp(pre, "\x93NUMPY", 6) != 0) { fclose(f); return -2; }
    uint32_t hlen;
    if (pre[6] == 1) {
        hlen = (uint32_t)pre[8] | ((uint32_t)pre[9] << 8);
    } else {
        unsigned char b2[2];
        if (fread(b2, 1, 2, f) != 2) { fclose(f); return -2; }
        hlen = (uint32_t)pre[8] | ((uint32_t)pre[9] << 8) | ((uint32_t)b2[0] << 16) | ((uint32_t)b2[1] << 24);
    }
    char *hdr = (char *)malloc(hlen + 1);
    if (!hdr || fread(hdr, 1, hlen, f) != hlen) { free(hdr); fclose(f); return -2; }
    hdr[hlen] = 0;
    const char *d = strstr(hdr, "'descr'");
    const char *fo = strstr(hdr, "'fortran_order'");
    const char *sh = strstr(hdr, "'shape'");
    if (!d || !fo || !sh) { free(hdr); fclose(f); return -3; }
    d = strchr(d + 7, '\'');
    if (!d) { free(hdr); fclose(f); return -3; }
    /* d -> '<f4' */
    char endian = d[1];
    out->kind = d[2];
    out->word = atoi(d + 3);
    const char *fv = fo + strlen("'fortran_order'");
    while (*fv == ':' || *fv == ' ') fv++;
    if (endian == '>' || strncmp(fv, "True", 4) == 0) {
        free(hdr); fclose(f); return -4;
    }
    const char *p = strchr(sh, '(');
    if (!p) { free(hdr); fclose(f); return -3; }
    p++;
    out->ndim = 0;
    out->shape[0] = 0; out->shape[1] = 1;
    while (*p && *p != ')') {
        while (*p == ' ' || *p == ',') p++;
        if (*p == ')') break;
        if (out->ndim >= 2) { free(hdr); fclose(f); return -5; }
        out->shape[out->ndim++] = strtoll(p, (char **)&p, 10);
    }
    if (out->ndim == 0) { out->ndim = 1; out->shape[0] = 1; }
    free(hdr);
    size_t n = (size_t)out->shape[0] * (size_t)out->shape[1] * (size_t)out->word;
    out->data = malloc(n ? n : 1);
    if (!out->data) { fclose(f); return -6; }
    if (n && fread(out->data, 1, n, f) != n) { free(out->data); out->data = NULL; fclose(f); return -7; }
    fclose(f);
    return 0;
}

static inline int pk_npy_write(const char *path, const char *descr, int ndim, const int64_t *shape,
                               const void *data) {
    char hdr[256];
    int len;
    if (ndim == 1)
        len = snprintf(hdr, sizeof(hdr), "{'descr': '%s', 'fortran_order': False, 'shape': (%lld,), }", descr,
                       (long long)shape[0]);
    else
        len = snprintf(hdr, sizeof(hdr), "{'descr': '%s', 'fortran_order': False, 'shape': (%lld, %lld), }",
                       descr, (long long)shape[0], (long long)shape[1]);
    int total = 10 + len + 1;
    int pad = (64 - total % 64) % 64;
    FILE *f = fopen(path, "wb");
    if (!f) return -1;
    unsigned char pre[10] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0, 0, 0};
    uint16_t hl = (uint16_t)(len + pad + 1);
    pre[8] = (unsigned char)(hl & 0xff);
    pre[9] = (unsigned char)(hl >> 8);
    fwrite(pre, 1, 10, f);
    fwrite(hdr, 1, (size_t)len, f);
    for (int i = 0; i < pad; i++) fputc(' ', f);
    fputc('\n', f);
    int word = atoi(descr + 2);
    size_t n = (size_t)shape[0] * (size_t)(ndim == 2 ? shape[1] : 1) * (size_t)word;
    if (n && fwrite(data, 1, n, f) != n) { fclose(f); return -2; }
    fclose(f);
    return 0;
}

#endif
