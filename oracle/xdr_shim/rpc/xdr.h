/* A minimal XDR (RFC 4506) for the reference's gauge-file reader and writer, which the
 * image has no library for: 32-bit integers, IEEE single and double precision, big-endian
 * on file, through a stdio stream.  TEST INFRASTRUCTURE ONLY (oracle/build_ref.sh); written
 * from the RFC, covering exactly the calls of starters/ReadStartGaugeConfiguration.cpp and
 * io/OutputSweep.cpp.  Each call returns 1 when its item was transferred, else 0. */
#ifndef LYM_XDR_SHIM_H
#define LYM_XDR_SHIM_H
#include <stdio.h>
#include <string.h>

typedef int bool_t;
#ifndef TRUE
#define TRUE 1
#define FALSE 0
#endif

enum xdr_op { XDR_ENCODE = 0, XDR_DECODE = 1, XDR_FREE = 2 };

typedef struct {
    FILE *file;
    enum xdr_op op;
} XDR;

static inline void xdrstdio_create(XDR *x, FILE *f, enum xdr_op op)
{
    x->file = f;
    x->op = op;
}

static inline void xdr_destroy(XDR *x)
{
    if (x->file) fflush(x->file);
}

/* n bytes of a native value, most significant byte first on file */
static inline bool_t lym_xdr_bytes(XDR *x, void *native, int n)
{
    unsigned char b[8], *v = (unsigned char *)native;
    const int little = 1;
    const int swap = *(const char *)&little == 1;
    if (x->op == XDR_ENCODE) {
        for (int i = 0; i < n; ++i) b[i] = swap ? v[n - 1 - i] : v[i];
        return fwrite(b, 1, (size_t)n, x->file) == (size_t)n;
    }
    if (x->op == XDR_DECODE) {
        if (fread(b, 1, (size_t)n, x->file) != (size_t)n) return FALSE;
        for (int i = 0; i < n; ++i) v[i] = swap ? b[n - 1 - i] : b[i];
        return TRUE;
    }
    return TRUE;
}

static inline bool_t xdr_int(XDR *x, int *v) { return lym_xdr_bytes(x, v, 4); }
static inline bool_t xdr_float(XDR *x, float *v) { return lym_xdr_bytes(x, v, 4); }
static inline bool_t xdr_double(XDR *x, double *v) { return lym_xdr_bytes(x, v, 8); }

#endif
