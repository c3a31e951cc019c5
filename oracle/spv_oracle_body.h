/*
 * CPU ORACLE body (test infrastructure only), instantiated twice by
 * spv_oracle.c: W_T = uint64_t (SFX _w64) and W_T = unsigned __int128
 * (SFX _w128), mirroring the reference's _word_type
 * (src/type_SparsePauliVector.jl:23-26).  Every function restates the
 * reference function named in its comment, in the same loop order, so that
 * floating-point results agree term for term.
 */
#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)

typedef struct { W_T z, x; double c; } FN(trip);

#if W_BITS == 64
static inline int FN(popc)(W_T v) { return __builtin_popcountll(v); }
#else
static inline int FN(popc)(W_T v) {
    return __builtin_popcountll((uint64_t)v) + __builtin_popcountll((uint64_t)(v >> 64));
}
#endif

/* _key_lt on (z, x) tuples: z-major lexicographic, unsigned (spv_kernels.jl:14-15). */
static inline int FN(key_lt)(W_T az, W_T ax, W_T bz, W_T bx) {
    return (az < bz) | ((az == bz) & (ax < bx));
}

/* _majorana_weight_bits (spv_kernels.jl:51-62): suffix-parity shift cascade. */
static inline int64_t FN(majorana)(W_T z, W_T x) {
    W_T zonly = z & ~x;
    W_T S = x;
    for (int shift = 1; shift < W_BITS; shift <<= 1) S ^= S >> shift;
    W_T ctrl = ~(S ^ x);
    return (int64_t)FN(popc)(x) + 2 * (int64_t)FN(popc)(zonly & ctrl) +
           2 * (int64_t)FN(popc)(~(z | x) & ~ctrl);
}

/* should_drop (spv_kernels.jl:64-79). */
static inline int FN(should_drop)(const orc_filter *f, W_T z, W_T x, double absc) {
    if (absc <= f->thresh) return 1;
    int64_t w = FN(popc)(z | x);
    if (w > f->wmax) return 1;
    if ((int64_t)FN(popc)(x) > f->xwmax) return 1;
    if (f->mwmax != INT64_MAX) {
        if (FN(majorana)(z, x) > f->mwmax) return 1;
    }
    if (f->dthresh_w >= 0.0) {
        if (absc * exp(-f->alpha_w * (double)w) <= f->dthresh_w) return 1;
    }
    if (f->dthresh_xw >= 0.0) {
        if (absc * exp(-f->alpha_xw * (double)FN(popc)(x)) <= f->dthresh_xw) return 1;
    }
    return 0;
}

/* _rotate_range! (spv_kernels.jl:146-177); lo/hi are 0-based, half-open. */
static int64_t FN(rotate_range)(W_T *z, W_T *x, double *c, int64_t lo, int64_t hi,
                                W_T gz, W_T gx, int64_t n_g, double cosv, double sinv,
                                W_T *dz, W_T *dx, double *dc, int64_t *cur, int64_t cap_end,
                                const orc_filter *f, int *overflowed) {
    int64_t created = 0;
    for (int64_t i = lo; i < hi; i++) {
        W_T zi = z[i], xi = x[i];
        int64_t m1 = FN(popc)(gx & zi);
        int64_t m2 = FN(popc)(gz & xi);
        if (((m1 - m2) & 1) == 0) continue;
        W_T zp = gz ^ zi, xp = gx ^ xi;
        int64_t k = (FN(popc)(zp & xp) - n_g - FN(popc)(zi & xi) + 2 * m1) & 3;
        double cnew = ((double)(k - 2) * sinv) * c[i];
        c[i] *= cosv;
        if (FN(should_drop)(f, zp, xp, fabs(cnew))) continue;
        if (*cur >= cap_end) { *overflowed = 1; continue; }
        dz[*cur] = zp; dx[*cur] = xp; dc[*cur] = cnew;
        (*cur)++;
        created++;
    }
    return created;
}

/* _grow_live! (type_SparsePauliVector.jl:107-117). */
static int FN(grow_live)(orc_spv *v, int64_t need) {
    int64_t newcap = 2 * v->cap > need ? 2 * v->cap : need;
    size_t wb = sizeof(W_T);
    void *p;
    if (!(p = realloc(v->z, newcap * wb))) return ORC_OOM;
    v->z = p;
    if (!(p = realloc(v->x, newcap * wb))) return ORC_OOM;
    v->x = p;
    if (!(p = realloc(v->c, newcap * sizeof(double)))) return ORC_OOM;
    v->c = p;
    if (!(p = realloc(v->sz, newcap * wb))) return ORC_OOM;
    v->sz = p;
    if (!(p = realloc(v->sx, newcap * wb))) return ORC_OOM;
    v->sx = p;
    if (!(p = realloc(v->sc, newcap * sizeof(double)))) return ORC_OOM;
    v->sc = p;
    v->cap = newcap;
    if (v->wscap < newcap) {
        if (!(p = realloc(v->ws, newcap * sizeof(FN(trip))))) return ORC_OOM;
        v->ws = p; v->wscap = newcap;
    }
    return ORC_OK;
}

/* _grow_append! (type_SparsePauliVector.jl:119-126). */
static int FN(grow_append)(orc_spv *v, int64_t need) {
    int64_t newcap = 2 * v->acap > need ? 2 * v->acap : need;
    size_t wb = sizeof(W_T);
    void *p;
    if (!(p = realloc(v->az, newcap * wb))) return ORC_OOM;
    v->az = p;
    if (!(p = realloc(v->ax, newcap * wb))) return ORC_OOM;
    v->ax = p;
    if (!(p = realloc(v->ac, newcap * sizeof(double)))) return ORC_OOM;
    v->ac = p;
    v->acap = newcap;
    if (v->wscap < newcap) {
        if (!(p = realloc(v->ws, newcap * sizeof(FN(trip))))) return ORC_OOM;
        v->ws = p; v->wscap = newcap;
    }
    return ORC_OK;
}

/* _gather_append! (spv_kernels.jl:187-193). */
static int64_t FN(gather_append)(orc_spv *v) {
    FN(trip) *ws = (FN(trip) *)v->ws;
    W_T *az = (W_T *)v->az, *ax = (W_T *)v->ax;
    for (int64_t i = 0; i < v->an; i++) {
        ws[i].z = az[i]; ws[i].x = ax[i]; ws[i].c = v->ac[i];
    }
    return v->an;
}

#define TLT(a, b) FN(key_lt)((a).z, (a).x, (b).z, (b).x)

/* _sort_ws! (spv_kernels.jl:202-247): median-of-3 quicksort, insertion sort
 * below 24, recurse on the smaller side.  ws1 is indexed 1-based (ws1 = ws-1)
 * so that the pivot choice mid = (lo+hi)>>>1 is the reference's. */
static void FN(sort_ws)(FN(trip) *ws1, int64_t lo, int64_t hi) {
    FN(trip) t;
    while (hi - lo >= 24) {
        int64_t mid = (int64_t)(((uint64_t)lo + (uint64_t)hi) >> 1);
        if (TLT(ws1[mid], ws1[lo])) { t = ws1[mid]; ws1[mid] = ws1[lo]; ws1[lo] = t; }
        if (TLT(ws1[hi], ws1[mid])) {
            t = ws1[hi]; ws1[hi] = ws1[mid]; ws1[mid] = t;
            if (TLT(ws1[mid], ws1[lo])) { t = ws1[mid]; ws1[mid] = ws1[lo]; ws1[lo] = t; }
        }
        FN(trip) pivot = ws1[mid];
        int64_t i = lo, j = hi;
        while (i <= j) {
            while (TLT(ws1[i], pivot)) i++;
            while (TLT(pivot, ws1[j])) j--;
            if (i <= j) { t = ws1[i]; ws1[i] = ws1[j]; ws1[j] = t; i++; j--; }
        }
        if (j - lo < hi - i) { FN(sort_ws)(ws1, lo, j); lo = i; }
        else { FN(sort_ws)(ws1, i, hi); hi = j; }
    }
    for (int64_t k = lo + 1; k <= hi; k++) {
        FN(trip) val = ws1[k];
        int64_t m = k - 1;
        while (m >= lo && TLT(val, ws1[m])) { ws1[m + 1] = ws1[m]; m--; }
        ws1[m + 1] = val;
    }
}

/* _unshuffle_pass! (spv_kernels.jl:262-286); word 1 = z, word 2 = x. */
static void FN(unshuffle_pass)(const FN(trip) *src, FN(trip) *dst, int64_t m, int b, int word) {
    W_T one = 1;
    /* bits above b; 0 for the top bit (Julia's << by the full width yields 0) */
    W_T hb = (b + 1 == W_BITS) ? (W_T)0 : ~((one << (b + 1)) - one);
    int64_t i = 0;
    while (i < m) {
        W_T hpz = word == 1 ? (src[i].z & hb) : src[i].z;
        W_T hpx = word == 1 ? (W_T)0 : (src[i].x & hb);
        int64_t j = i;
        while (j + 1 < m) {
            W_T qz = word == 1 ? (src[j + 1].z & hb) : src[j + 1].z;
            W_T qx = word == 1 ? (W_T)0 : (src[j + 1].x & hb);
            if (qz != hpz || qx != hpx) break;
            j++;
        }
        int64_t f = i;
        while (f <= j && (((word == 1 ? src[f].z : src[f].x) >> b) & one) == one) f++;
        int64_t k = i;
        for (int64_t s = f; s <= j; s++) dst[k++] = src[s];
        for (int64_t s = i; s < f; s++) dst[k++] = src[s];
        i = j + 1;
    }
}

/* _unshuffle_ws! (spv_kernels.jl:300-320). */
static int FN(unshuffle_ws)(orc_spv *v, int64_t m, W_T gz, W_T gx) {
    if (m <= 1) return ORC_OK;
    if (FN(popc)(gz) + FN(popc)(gx) == 0) return ORC_OK;
    if (v->ws2cap < m) {
        void *p = realloc(v->ws2, v->wscap * sizeof(FN(trip)));
        if (!p) return ORC_OOM;
        v->ws2 = p; v->ws2cap = v->wscap;
    }
    FN(trip) *src = (FN(trip) *)v->ws, *dst = (FN(trip) *)v->ws2, *t;
    int flips = 0;
    for (int b = W_BITS - 1; b >= 0; b--) {
        if (((gz >> b) & 1) != 1) continue;
        FN(unshuffle_pass)(src, dst, m, b, 1);
        t = src; src = dst; dst = t; flips++;
    }
    for (int b = W_BITS - 1; b >= 0; b--) {
        if (((gx >> b) & 1) != 1) continue;
        FN(unshuffle_pass)(src, dst, m, b, 2);
        t = src; src = dst; dst = t; flips++;
    }
    if (flips & 1) memcpy(v->ws, v->ws2, m * sizeof(FN(trip)));
    return ORC_OK;
}

/* _try_merge! (spv_kernels.jl:326-363).  Returns out; *ovf set on overflow
 * (nothing swapped, live untouched). */
static int64_t FN(try_merge)(orc_spv *v, int64_t m, const orc_filter *f, int *ovf) {
    int64_t n = v->n;
    W_T *z = (W_T *)v->z, *x = (W_T *)v->x; double *c = v->c;
    W_T *sz = (W_T *)v->sz, *sx = (W_T *)v->sx; double *sc = v->sc;
    const FN(trip) *ws = (const FN(trip) *)v->ws;
    int64_t cap = v->cap, out = 0, i = 0, j = 0;
    *ovf = 0;
    while (i < n || j < m) {
        W_T kz, kx; double acc;
        if (j >= m || (i < n && !FN(key_lt)(ws[j].z, ws[j].x, z[i], x[i]))) {
            kz = z[i]; kx = x[i]; acc = c[i]; i++;
        } else {
            kz = ws[j].z; kx = ws[j].x; acc = ws[j].c; j++;
        }
        while (j < m && ws[j].z == kz && ws[j].x == kx) { acc += ws[j].c; j++; }
        if (FN(should_drop)(f, kz, kx, fabs(acc))) continue;
        out++;
        if (out > cap) { *ovf = 1; return out; }
        sz[out - 1] = kz; sx[out - 1] = kx; sc[out - 1] = acc;
    }
    void *t;
    t = v->z; v->z = v->sz; v->sz = t;
    t = v->x; v->x = v->sx; v->sx = t;
    double *tc = v->c; v->c = v->sc; v->sc = tc;
    v->n = out;
    return out;
}

/* _merge_spv! (spv_kernels.jl:377-386). */
static int FN(merge_spv)(orc_spv *v, int64_t m, const orc_filter *f, int64_t *n_in, int64_t *n_out) {
    *n_in = v->n + m;
    int ovf;
    int64_t out = FN(try_merge)(v, m, f, &ovf);
    while (ovf) {
        int e = FN(grow_live)(v, v->n + m);
        if (e) return e;
        out = FN(try_merge)(v, m, f, &ovf);
    }
    v->an = 0;
    *n_out = out;
    return ORC_OK;
}

/* _compact_spv! (spv_kernels.jl:395-408). */
static void FN(compact)(orc_spv *v, const orc_filter *f) {
    W_T *z = (W_T *)v->z, *x = (W_T *)v->x; double *c = v->c;
    int64_t out = 0;
    for (int64_t i = 0; i < v->n; i++) {
        if (FN(should_drop)(f, z[i], x[i], fabs(c[i]))) continue;
        out++;
        if (out - 1 != i) { z[out - 1] = z[i]; x[out - 1] = x[i]; c[out - 1] = c[i]; }
    }
    v->n = out;
}

/* _expectation_spv (spv_kernels.jl:441-452): live then pending appends, in index order. */
static double FN(expect)(const orc_spv *v, W_T kv) {
    const W_T *z = (const W_T *)v->z, *x = (const W_T *)v->x;
    const W_T *az = (const W_T *)v->az, *ax = (const W_T *)v->ax;
    double acc = 0.0;
    for (int64_t i = 0; i < v->n; i++) {
        if (x[i] != 0) continue;
        acc += (double)(1 - 2 * (FN(popc)(z[i] & kv) & 1)) * v->c[i];
    }
    for (int64_t i = 0; i < v->an; i++) {
        if (ax[i] != 0) continue;
        acc += (double)(1 - 2 * (FN(popc)(az[i] & kv) & 1)) * v->ac[i];
    }
    return acc;
}

/* Neumaier-compensated variant of the same sum (accuracy reference for the GPU). */
static double FN(expect_neumaier)(const orc_spv *v, W_T kv) {
    const W_T *z = (const W_T *)v->z, *x = (const W_T *)v->x;
    double s = 0.0, comp = 0.0;
    for (int64_t i = 0; i < v->n; i++) {
        if (x[i] != 0) continue;
        double t = (double)(1 - 2 * (FN(popc)(z[i] & kv) & 1)) * v->c[i];
        double u = s + t;
        if (fabs(s) >= fabs(t)) comp += (s - u) + t; else comp += (t - u) + s;
        s = u;
    }
    return s + comp;
}

/* _rotate_spv! (spv_evolve.jl:207-218). */
static int64_t FN(rotate_spv)(orc_spv *v, W_T gz, W_T gx, int64_t ng, double cosv, double sinv,
                              const orc_filter *f, int *ovf) {
    int64_t hi = v->an;
    int64_t cur = v->an;
    int o1 = 0, o2 = 0;
    int64_t cr1 = FN(rotate_range)((W_T *)v->z, (W_T *)v->x, v->c, 0, v->n, gz, gx, ng, cosv, sinv,
                                   (W_T *)v->az, (W_T *)v->ax, v->ac, &cur, v->acap, f, &o1);
    int64_t cr2 = FN(rotate_range)((W_T *)v->az, (W_T *)v->ax, v->ac, 0, hi, gz, gx, ng, cosv, sinv,
                                   (W_T *)v->az, (W_T *)v->ax, v->ac, &cur, v->acap, f, &o2);
    v->an = cur;
    *ovf = o1 | o2;
    return cr1 + cr2;
}

/* _sort_pending! (spv_evolve.jl:194-202). */
static int FN(sort_pending)(orc_spv *v, int64_t m, int have_mask, W_T mz, W_T mx) {
    if (!have_mask) { FN(sort_ws)((FN(trip) *)v->ws - 1, 1, m); return ORC_OK; }
    return FN(unshuffle_ws)(v, m, mz, mx);
}

/* evolve!(O, G, θ) single rotation (spv_evolve.jl:228-236) with merge_pending!
 * (spv_evolve.jl:185-190). */
static int FN(evolve1)(orc_spv *v, W_T gz, W_T gx, double cosv, double sinv) {
    static const orc_filter NOF = {INT64_MAX, INT64_MAX, INT64_MAX, -1.0, 0.0, -1.0, 0.0, -1.0};
    int64_t ng = FN(popc)(gz & gx);
    if (v->n + 2 * v->an > v->acap) { int e = FN(grow_append)(v, v->n + 2 * v->an); if (e) return e; }
    int ovf;
    FN(rotate_spv)(v, gz, gx, ng, cosv, sinv, &NOF, &ovf);
    if (ovf) { orc_set_error("append overflow despite precheck"); return ORC_ERROR_EXCEPTION; }
    int64_t m = FN(gather_append)(v);
    int e = FN(unshuffle_ws)(v, m, gz, gx);
    if (e) return e;
    int64_t a, b;
    return FN(merge_spv)(v, m, &NOF, &a, &b);
}

/* _measure for NoCorrection / EnergyCorrection (truncation.jl:285-289). */
static double FN(measure)(const orc_spv *v, const orc_evolve_params *p) {
    if (p->corr_kind != 1) return 0.0;
    W_T kv = (W_T)p->ket[0];
#if W_BITS == 128
    kv |= ((W_T)p->ket[1]) << 64;
#endif
    return FN(expect)(v, kv);
}

/* _apply!(v, ::AdaptiveTruncation) (spv_evolve.jl:103-114). */
static int FN(cmp_dbl)(const void *a, const void *b) {
    double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}
static int FN(adaptive)(orc_spv *v, int64_t max_terms, double min_thresh) {
    orc_filter f = {INT64_MAX, INT64_MAX, INT64_MAX, -1.0, 0.0, -1.0, 0.0, -1.0};
    if (v->n > max_terms) {
        double *coeffs = (double *)malloc((v->n > 0 ? v->n : 1) * sizeof(double));
        if (!coeffs) return ORC_OOM;
        for (int64_t i = 0; i < v->n; i++) coeffs[i] = fabs(v->c[i]);
        qsort(coeffs, v->n, sizeof(double), FN(cmp_dbl));
        if (v->n > max_terms) {
            f.thresh = coeffs[v->n - max_terms - 1];
            FN(compact)(v, &f);
        }
        free(coeffs);
    } else {
        f.thresh = min_thresh;
        FN(compact)(v, &f);
    }
    return ORC_OK;
}

/* _boundary! (spv_evolve.jl:258-284) for NoCorrection / EnergyCorrection
 * (both take the "measure on pre-merge state" branch, _needs_merged_measure = false). */
static int FN(boundary)(orc_spv *v, const orc_filter *f, orc_evolve_params *p, int64_t w,
                        int have_mask, W_T mz, W_T mx) {
    double before = FN(measure)(v, p);
    int64_t m = FN(gather_append)(v);
    int e = FN(sort_pending)(v, m, have_mask, mz, mx);
    if (e) return e;
    int64_t n_in, n_out;
    e = FN(merge_spv)(v, m, f, &n_in, &n_out);
    if (e) return e;
    if (!p->strict_compiled) { e = FN(adaptive)(v, p->adapt_max_terms, p->adapt_min_thresh); if (e) return e; }
    double after = FN(measure)(v, p);
    if (p->corr_kind == 1) p->corr_energy += after - before;
    if (p->nwin > 0 && w >= 1 && w <= p->nwin) {
        if (p->merge_in) p->merge_in[w - 1] += n_in;
        if (p->merge_out) p->merge_out[w - 1] += n_out;
    }
    return ORC_OK;
}

/* Sequence evolve! driver (spv_evolve.jl:312-387). gens are packed words. */
static int FN(evolve_seq)(orc_spv *v, const W_T *gz, const W_T *gx, const double *cosv,
                          const double *sinv, int64_t L, orc_evolve_params *p) {
    static const orc_filter NOF = {INT64_MAX, INT64_MAX, INT64_MAX, -1.0, 0.0, -1.0, 0.0, -1.0};
    if (p->window < 1) { orc_set_error("window must be >= 1"); return ORC_ARGUMENT_ERROR; }
    if (L == 0) return ORC_OK;
    const orc_filter *f = p->strict_compiled ? &p->strict : &NOF;
    const orc_filter *flocal = &p->local;
    int64_t since = 0;
    W_T lz = 0, lx = 0;
    for (int64_t i = 1; i <= L; i++) {
        int64_t w = (i + p->window - 1) / p->window;
        if (2 * v->an + v->n > v->acap) {
            int e = FN(boundary)(v, f, p, w, since == 1, lz, lx);
            if (e) return e;
            since = 0;
            if (p->nwin > 0 && w <= p->nwin && p->early_merges) p->early_merges[w - 1] += 1;
            if (v->n > v->acap) { e = FN(grow_append)(v, v->n); if (e) return e; }
        }
        W_T g_z = gz[i - 1], g_x = gx[i - 1];
        int64_t ng = FN(popc)(g_z & g_x);
        int ovf;
        int64_t created = FN(rotate_spv)(v, g_z, g_x, ng, cosv[i - 1], sinv[i - 1], flocal, &ovf);
        if (ovf) { orc_set_error("append overflow despite precheck"); return ORC_ERROR_EXCEPTION; }
        lz = g_z; lx = g_x;
        since++;
        if (p->nwin > 0 && w <= p->nwin && p->terms_created) p->terms_created[w - 1] += created;
        if (i % p->window == 0 || i == L) {
            int e = FN(boundary)(v, f, p, w, since == 1, lz, lx);
            if (e) return e;
            since = 0;
        }
    }
    return ORC_OK;
}

/* SPV channel fast paths (channels.jl:203-265); λ^k via the compensated
 * integer power (the reference's Float64^Int). */
static void FN(channel)(orc_spv *v, int kind, const double *prm, W_T M) {
    W_T *z = (W_T *)v->z, *x = (W_T *)v->x; double *c = v->c;
    if (kind == 4) {
        double pX = prm[0], pY = prm[1], pZ = prm[2];
        double lX = 1.0 - 2.0 * (pY + pZ), lY = 1.0 - 2.0 * (pX + pZ), lZ = 1.0 - 2.0 * (pX + pY);
        for (int64_t i = 0; i < v->n; i++) {
            W_T xM = x[i] & M, zM = z[i] & M;
            int64_t nX = FN(popc)(xM & ~z[i]);
            int64_t nY = FN(popc)(xM & z[i]);
            int64_t nZ = FN(popc)(zM & ~x[i]);
            c[i] *= orc_jl_pow(lX, nX) * orc_jl_pow(lY, nY) * orc_jl_pow(lZ, nZ);
        }
        return;
    }
    double p = prm[0];
    double lam = kind == 0 ? 1.0 - 4.0 * p / 3.0 : 1.0 - 2.0 * p;
    for (int64_t i = 0; i < v->n; i++) {
        W_T sel = kind == 0 ? ((z[i] | x[i]) & M) : kind == 1 ? (x[i] & M)
                : kind == 2 ? (z[i] & M) : ((x[i] ^ z[i]) & M);
        c[i] *= orc_jl_pow(lam, FN(popc)(sel));
    }
}

/* check_spv (type_SparsePauliVector.jl:263-278): strictly increasing live keys. */
static int FN(check)(const orc_spv *v) {
    const W_T *z = (const W_T *)v->z, *x = (const W_T *)v->x;
    if (v->n > v->cap || v->an > v->acap) return 0;
    for (int64_t i = 1; i < v->n; i++)
        if (!FN(key_lt)(z[i - 1], x[i - 1], z[i], x[i])) return 0;
    return 1;
}

/* _sort_live! (type_SparsePauliVector.jl:195-204). */
static void FN(sort_live)(orc_spv *v) {
    FN(trip) *ws = (FN(trip) *)v->ws;
    W_T *z = (W_T *)v->z, *x = (W_T *)v->x;
    for (int64_t i = 0; i < v->n; i++) { ws[i].z = z[i]; ws[i].x = x[i]; ws[i].c = v->c[i]; }
    FN(sort_ws)(ws - 1, 1, v->n);
    for (int64_t i = 0; i < v->n; i++) { z[i] = ws[i].z; x[i] = ws[i].x; v->c[i] = ws[i].c; }
}

#undef TLT
#undef FN
#undef CAT
#undef CAT2
