/*
 * CPU ORACLE — test infrastructure only (see spv_oracle.h).  Restates the
 * reference SparsePauliVector path; instantiates spv_oracle_body.h for the
 * two word types of _word_type (src/type_SparsePauliVector.jl:23-26).
 * Build: oracle/Makefile (gcc -O3 -ffp-contract=off, single thread).
 */
#include "spv_oracle.h"
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

struct orc_spv {
    int N, nw;
    void *z, *x; double *c; int64_t n, cap;     /* live (sorted, dup-free) */
    void *az, *ax; double *ac; int64_t an, acap; /* append */
    void *sz, *sx; double *sc;                   /* scratch (cap) */
    void *ws; int64_t wscap;                     /* merge workspace triples */
    void *ws2; int64_t ws2cap;                   /* unshuffle ping-pong */
};

static __thread char g_err[256];
static void orc_set_error(const char *m) { snprintf(g_err, sizeof g_err, "%s", m); }
const char *orc_last_error(void) { return g_err; }

/* Compensated binary powering for Float64^Int (the algorithm of Julia Base's
 * `^(::Float64, ::Integer)`: square-and-multiply carrying the low parts of
 * each product as a double-double, with x*x*x for n == 3). */
double orc_jl_pow(double x, int64_t n) {
    if (n == 0) return 1.0;
    double y = 1.0, xnlo = 0.0, ynlo = 0.0;
    if (n == 3) return x * x * x;
    if (n < 0) {
        double rx = 1.0 / x;
        if (n == -2) return rx * rx;
        if (isfinite(x)) xnlo = -fma(x, rx, -1.0) * rx;
        x = rx;
        n = -n;
    }
    while (n > 1) {
        if (n & 1) {
            double err = fma(y, xnlo, x * ynlo);
            double p = x * y;
            ynlo = fma(x, y, -p);
            y = p;
            ynlo += err;
        }
        double err = x * 2.0 * xnlo;
        double p = x * x;
        xnlo = fma(x, x, -p);
        x = p;
        xnlo += err;
        n >>= 1;
    }
    if (!isfinite(x)) return x * y;
    return fma(x, y, fma(y, xnlo, x * ynlo));
}

#define W_T uint64_t
#define W_BITS 64
#define SFX _w64
#include "spv_oracle_body.h"
#undef W_T
#undef W_BITS
#undef SFX

#define W_T unsigned __int128
#define W_BITS 128
#define SFX _w128
#include "spv_oracle_body.h"
#undef W_T
#undef W_BITS
#undef SFX

static size_t wbytes(const orc_spv *v) { return v->nw == 1 ? 8 : 16; }
static size_t tbytes(const orc_spv *v) {
    return v->nw == 1 ? sizeof(trip_w64) : sizeof(trip_w128);
}

orc_spv *orc_create(int N, int64_t live_cap, int64_t append_cap) {
    if (N < 0 || N > 128) { orc_set_error("N > 128 requires a multi-word type"); return NULL; }
    if (live_cap < 1) live_cap = 1;
    if (append_cap < 1) append_cap = 1;
    orc_spv *v = (orc_spv *)calloc(1, sizeof(orc_spv));
    if (!v) return NULL;
    v->N = N;
    v->nw = N <= 64 ? 1 : 2;
    size_t wb = wbytes(v);
    v->cap = live_cap; v->acap = append_cap;
    v->z = calloc(live_cap, wb); v->x = calloc(live_cap, wb); v->c = calloc(live_cap, 8);
    v->sz = calloc(live_cap, wb); v->sx = calloc(live_cap, wb); v->sc = calloc(live_cap, 8);
    v->az = calloc(append_cap, wb); v->ax = calloc(append_cap, wb); v->ac = calloc(append_cap, 8);
    v->wscap = live_cap > append_cap ? live_cap : append_cap;
    v->ws = calloc(v->wscap, tbytes(v));
    v->ws2 = NULL; v->ws2cap = 0;
    if (!v->z || !v->x || !v->c || !v->sz || !v->sx || !v->sc || !v->az || !v->ax || !v->ac || !v->ws) {
        orc_destroy(v);
        return NULL;
    }
    return v;
}

void orc_destroy(orc_spv *v) {
    if (!v) return;
    free(v->z); free(v->x); free(v->c); free(v->sz); free(v->sx); free(v->sc);
    free(v->az); free(v->ax); free(v->ac); free(v->ws); free(v->ws2);
    free(v);
}

int orc_nwords(const orc_spv *v) { return v->nw; }
int64_t orc_len(const orc_spv *v) { return v->n; }
int64_t orc_live_cap(const orc_spv *v) { return v->cap; }
int64_t orc_append_cap(const orc_spv *v) { return v->acap; }

/* Constructor fill + _sort_live! (type_SparsePauliVector.jl:167-188). */
int orc_upload(orc_spv *v, const void *z, const void *x, const double *c, int64_t n) {
    if (n > v->cap) {
        int e = v->nw == 1 ? grow_live_w64(v, n) : grow_live_w128(v, n);
        if (e) return e;
    }
    if (n > v->wscap) {
        void *p = realloc(v->ws, n * tbytes(v));
        if (!p) return ORC_OOM;
        v->ws = p; v->wscap = n;
    }
    size_t wb = wbytes(v);
    memcpy(v->z, z, n * wb); memcpy(v->x, x, n * wb); memcpy(v->c, c, n * 8);
    v->n = n; v->an = 0;
    if (v->nw == 1) sort_live_w64(v); else sort_live_w128(v);
    return ORC_OK;
}

int64_t orc_download(const orc_spv *v, void *z, void *x, double *c, int64_t cap) {
    int64_t n = v->n < cap ? v->n : cap;
    size_t wb = wbytes(v);
    if (z) memcpy(z, v->z, n * wb);
    if (x) memcpy(x, v->x, n * wb);
    if (c) memcpy(c, v->c, n * 8);
    return v->n;
}

orc_spv *orc_copy(const orc_spv *v) {
    orc_spv *w = orc_create(v->N, v->cap, v->acap);
    if (!w) return NULL;
    size_t wb = wbytes(v);
    memcpy(w->z, v->z, v->n * wb); memcpy(w->x, v->x, v->n * wb); memcpy(w->c, v->c, v->n * 8);
    memcpy(w->az, v->az, v->an * wb); memcpy(w->ax, v->ax, v->an * wb); memcpy(w->ac, v->ac, v->an * 8);
    w->n = v->n; w->an = v->an;
    return w;
}

static unsigned __int128 load_w(const void *p, int nw) {
    if (!p) return 0;
    uint64_t q[2] = {0, 0};
    memcpy(q, p, nw * 8);
    return (unsigned __int128)q[0] | (((unsigned __int128)q[1]) << 64);
}

int orc_evolve1(orc_spv *v, const void *gz, const void *gx, double cosv, double sinv) {
    if (v->nw == 1)
        return evolve1_w64(v, *(const uint64_t *)gz, *(const uint64_t *)gx, cosv, sinv);
    return evolve1_w128(v, load_w(gz, 2), load_w(gx, 2), cosv, sinv);
}

int orc_evolve(orc_spv *v, const void *gz, const void *gx, const double *cosv, const double *sinv,
               int64_t L, orc_evolve_params *p) {
    if (v->nw == 1)
        return evolve_seq_w64(v, (const uint64_t *)gz, (const uint64_t *)gx, cosv, sinv, L, p);
    /* copy into 16-byte-aligned storage: caller buffers need only 8-byte alignment */
    unsigned __int128 *az = (unsigned __int128 *)malloc((L > 0 ? L : 1) * 16);
    unsigned __int128 *ax = (unsigned __int128 *)malloc((L > 0 ? L : 1) * 16);
    if (!az || !ax) { free(az); free(ax); return ORC_OOM; }
    memcpy(az, gz, L * 16); memcpy(ax, gx, L * 16);
    int e = evolve_seq_w128(v, az, ax, cosv, sinv, L, p);
    free(az); free(ax);
    return e;
}

int orc_compact(orc_spv *v, const orc_filter *f) {
    if (v->nw == 1) compact_w64(v, f); else compact_w128(v, f);
    return ORC_OK;
}

int orc_adaptive(orc_spv *v, int64_t max_terms, double min_thresh) {
    return v->nw == 1 ? adaptive_w64(v, max_terms, min_thresh) : adaptive_w128(v, max_terms, min_thresh);
}

/* Argument validation of channels.jl:206-207, 225-226, 236, 247, 258. */
int orc_channel(orc_spv *v, int kind, const double *prm, const void *mask) {
    if (kind < 0 || kind > 4) { orc_set_error("unknown channel kind"); return ORC_ARGUMENT_ERROR; }
    if (kind == 4) {
        if (!(prm[0] >= 0 && prm[1] >= 0 && prm[2] >= 0)) {
            orc_set_error("probabilities must be non-negative"); return ORC_ARGUMENT_ERROR;
        }
        if (!(prm[0] + prm[1] + prm[2] <= 1.0 + 4.0 * 2.220446049250313e-16)) {
            orc_set_error("pX+pY+pZ must be <= 1"); return ORC_ARGUMENT_ERROR;
        }
    } else if (!(prm[0] >= 0.0 && prm[0] <= 1.0)) {
        orc_set_error("channel parameter p must be in [0,1]"); return ORC_ARGUMENT_ERROR;
    }
    unsigned __int128 all = v->N == 128 ? ~(unsigned __int128)0
                          : (((unsigned __int128)1) << v->N) - 1;
    unsigned __int128 M = mask ? load_w(mask, v->nw) : all;
    if (v->nw == 1) channel_w64(v, kind, prm, (uint64_t)M);
    else channel_w128(v, kind, prm, M);
    return ORC_OK;
}

double orc_expect(const orc_spv *v, const void *ket) {
    unsigned __int128 k = load_w(ket, v->nw);
    return v->nw == 1 ? expect_w64(v, (uint64_t)k) : expect_w128(v, k);
}

double orc_expect_neumaier(const orc_spv *v, const void *ket) {
    unsigned __int128 k = load_w(ket, v->nw);
    return v->nw == 1 ? expect_neumaier_w64(v, (uint64_t)k) : expect_neumaier_w128(v, k);
}

int orc_check(const orc_spv *v) { return v->nw == 1 ? check_w64(v) : check_w128(v); }
