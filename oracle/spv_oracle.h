/*
 * CPU ORACLE — test infrastructure only. Nothing in the product library links,
 * loads or calls this code; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py use it, as the checker.
 *
 * A plain-C restatement of PauliOperators.jl's SparsePauliVector propagation
 * path (src/spv_kernels.jl, src/spv_evolve.jl, src/channels.jl SPV methods,
 * src/truncation.jl, src/type_SparsePauliVector.jl).  Each function in
 * spv_oracle_body.h cites the reference line it restates.
 *
 * Parity pinning: the reference is Julia and no Julia toolchain exists here,
 * so the oracle is pinned (tests/test_oracle_*.py) against
 *   - the reference's hand-literal known-answer tests (test_truncation.jl,
 *     test_channels.jl closed forms) transcribed into tests/golden/,
 *   - dense-matrix conjugation exp(iθ/2 G) O exp(-iθ/2 G) (numpy, N <= 5),
 *   - brute-force Kraus sums for the channels (numpy, N <= 3),
 *   - an independent Dict-path restatement (src/evolve.jl:226-240,
 *     evolve.jl:305-315, clip.jl) written with per-qubit Pauli products.
 * It is NOT pinned against outputs of the Julia reference itself.
 */
#ifndef SPV_ORACLE_H
#define SPV_ORACLE_H
#include <stdint.h>

/* Byte-identical to the reference's isbits MergeFilter (spv_kernels.jl:33-42). */
typedef struct {
    int64_t wmax, xwmax, mwmax;
    double thresh, alpha_w, dthresh_w, alpha_xw, dthresh_xw;
} orc_filter;

typedef struct orc_spv orc_spv;

typedef struct {
    int64_t window;
    orc_filter strict;          /* used when strict_compiled != 0 */
    int32_t strict_compiled;    /* 1: MergeFilter strategy; 0: AdaptiveTruncation */
    int32_t corr_kind;          /* 0 NoCorrection, 1 EnergyCorrection */
    int64_t adapt_max_terms;    /* AdaptiveTruncation(max_terms, min_thresh) */
    double adapt_min_thresh;
    orc_filter local;           /* local_truncation (always compiled) */
    uint64_t ket[2];            /* EnergyCorrection ket bits (lo, hi) */
    double corr_energy;         /* in/out: accumulated_energy */
    int64_t nwin;               /* length of the counter arrays below (0: none) */
    int64_t *terms_created, *merge_in, *merge_out, *early_merges;
} orc_evolve_params;

/* Construction: live_cap / append_cap as _alloc_spv (type_SparsePauliVector.jl:94-104). */
orc_spv *orc_create(int N, int64_t live_cap, int64_t append_cap);
void orc_destroy(orc_spv *v);
int orc_nwords(const orc_spv *v);                 /* 1 (UInt64) or 2 (UInt128) */
int64_t orc_len(const orc_spv *v);
int64_t orc_live_cap(const orc_spv *v);
int64_t orc_append_cap(const orc_spv *v);
/* z, x: n words of the word type (UInt128 = 16 B little-endian). */
int orc_upload(orc_spv *v, const void *z, const void *x, const double *c, int64_t n);
int64_t orc_download(const orc_spv *v, void *z, void *x, double *c, int64_t cap);
orc_spv *orc_copy(const orc_spv *v);

int orc_evolve1(orc_spv *v, const void *gz, const void *gx, double cosv, double sinv);
int orc_evolve(orc_spv *v, const void *gz, const void *gx, const double *cosv,
               const double *sinv, int64_t L, orc_evolve_params *p);
int orc_compact(orc_spv *v, const orc_filter *f);
int orc_adaptive(orc_spv *v, int64_t max_terms, double min_thresh);
/* kind: 0 depolarizing, 1 dephasing, 2 bit_flip, 3 bit_phase_flip, 4 pauli.
 * prm: p (kinds 0-3) or pX,pY,pZ (kind 4). mask: qubit mask words (NULL = all). */
int orc_channel(orc_spv *v, int kind, const double *prm, const void *mask);
double orc_expect(const orc_spv *v, const void *ket);          /* reference order */
double orc_expect_neumaier(const orc_spv *v, const void *ket); /* compensated */
int orc_check(const orc_spv *v);
double orc_jl_pow(double x, int64_t n);
const char *orc_last_error(void);

/* Error codes (mirror include/pauliprop.h). */
#define ORC_OK 0
#define ORC_ARGUMENT_ERROR 1
#define ORC_DIMENSION_MISMATCH 2
#define ORC_ERROR_EXCEPTION 3
#define ORC_OOM 4

#endif
