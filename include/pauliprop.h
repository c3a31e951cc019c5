/*
 * pauliprop — B200-native (sm_100a) SparsePauliVector propagation engine.
 *
 * C ABI of libpauliprop.so.  Every entry point is a drop-in for one method of
 * PauliOperators.jl's SparsePauliVector propagation path; the comment above
 * each declaration names the reference interface it replaces (file:line in
 * the PauliOperators.jl source tree).  Plain pointers and sizes only: a Julia
 * `ccall`, a Python `ctypes` or a C caller binds it directly.
 *
 * Word layout: z and x are arrays of the reference's packed word type
 * (_word_type, src/type_SparsePauliVector.jl:23-26): one uint64 per term for
 * N <= 64, one 16-byte little-endian UInt128 (low word first) per term for
 * 65 <= N <= 128 — byte-identical to Julia's Vector{UInt64}/Vector{UInt128}.
 * Coefficients are Float64 (T = Float64, the engine's real coefficient type).
 * Term arrays stay in device memory between calls; host buffers are touched
 * only by pp_upload / pp_download / the small argument arrays.
 *
 * Threading: one CUDA stream per handle; a handle is not re-entrant, distinct
 * handles are independent.  Calls that return data synchronize.
 * All entry points return a pp_status; pp_last_error() gives the message
 * (thread-local).
 */
#ifndef PAULIPROP_H
#define PAULIPROP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PP_OK = 0,
    PP_ARGUMENT_ERROR = 1,      /* Julia ArgumentError (channels.jl:16-27, 225-226; spv_evolve.jl:321, 327-330) */
    PP_DIMENSION_MISMATCH = 2,  /* Julia DimensionMismatch (spv_evolve.jl:319-320) */
    PP_ERROR_EXCEPTION = 3,     /* Julia ErrorException (type_SparsePauliVector.jl:25, 145-147; check_spv) */
    PP_OUT_OF_MEMORY = 4,
    PP_DEVICE_ERROR = 5,        /* CUDA runtime error */
    PP_TIMEOUT = 6,             /* a bounded device-side wait gave up */
    PP_NOT_IMPLEMENTED = 7      /* strategy without a GPU path (no CPU fallback exists) */
} pp_status;

typedef struct pp_spv pp_spv;

/* Byte-identical to the isbits MergeFilter (spv_kernels.jl:33-42); sentinels
 * INT64_MAX for disabled weight caps and negative thresholds for disabled
 * coefficient criteria, as in NOFILTER (spv_kernels.jl:44-45). */
typedef struct {
    int64_t wmax, xwmax, mwmax;
    double thresh, alpha_w, dthresh_w, alpha_xw, dthresh_xw;
} pp_filter;

/* WindowCounters (spv_evolve.jl:149-161); arrays of length nwin, caller-owned.
 * t_rotate / t_merge are device time in seconds (CUDA events). */
typedef struct {
    int64_t nwin;
    int64_t *terms_created, *merge_in, *merge_out, *early_merges;
    double *t_rotate, *t_merge;
} pp_counters;

/* Keyword arguments of the sequence evolve! (spv_evolve.jl:312-318). */
typedef struct {
    int64_t window;               /* window = 1 (default) */
    const pp_filter *strict;      /* truncation (compiled); NULL = NoTruncation */
    const pp_filter *local;       /* local_truncation; NULL = NoTruncation */
    int32_t strict_kind;          /* 0 compiled MergeFilter, 1 AdaptiveTruncation (adapt_max_terms,
                                     adapt_min_thresh), 2 StochasticCoeffTruncation (epsilon in
                                     adapt_min_thresh), 3 StochasticSamplingTruncation (n_keep in
                                     adapt_max_terms); 1-3 run after every unfiltered merge */
    int32_t corr_kind;            /* 0 NoCorrection, 1 EnergyCorrection (truncation.jl:255-266),
                                     2 EnergyVarianceCorrection (truncation.jl:269-278) */
    int64_t adapt_max_terms;
    double adapt_min_thresh;
    const void *ket;              /* EnergyCorrection ket: one word (type as z/x) */
    double *corr_energy;          /* in/out: accumulated_energy (EnergyCorrection) */
    pp_counters *counters;        /* nullable */
    int32_t chan_kind;            /* -1: none. 0..4: channel applied after the last rotation,
                                     fused into its merge (see pp_channel) */
    int32_t pad;
    double chan_prm[3];
    const void *chan_mask;        /* NULL: all qubits */
    double *expect_out;           /* nullable: <0...0|O|0...0> of the final state (fused reduction) */
    int64_t chan_every;           /* > 0: apply the channel after every chan_every-th rotation
                                     (a layer loop "evolve!(v, layer...); channel!(v, p)" in one call) */
    double *stats_out;            /* nullable, PP_STATS_LEN doubles: see PP_STAT_* */
    int32_t profile;              /* 1: time the rotate and merge kernels with CUDA events (stats) */
    int32_t pad2;
    double *corr_variance;        /* in/out: EnergyVarianceCorrection.accumulated_variance (corr_kind 2) */
    uint64_t seed;                /* strict_kind 2, 3: random stream (application k uses its own substream) */
} pp_evolve_opts;

/* stats_out layout (sums over the call's rotations). */
#define PP_STAT_TERMS_IN 0        /* live terms entering each rotation (terms/s numerator) */
#define PP_STAT_CREATED 1         /* sin branches appended */
#define PP_STAT_MERGE_IN 2        /* merge inputs (live + appended) */
#define PP_STAT_MERGE_OUT 3       /* merge survivors */
#define PP_STAT_PEAK 4            /* largest live count after a merge */
#define PP_STAT_EARLY 5           /* early (capacity-forced) merges */
#define PP_STAT_T_ROTATE 6        /* seconds in classify/scan/permute kernels (profile = 1) */
#define PP_STAT_T_MERGE 7         /* seconds in the merge kernel alone (profile = 1) */
#define PP_STAT_LAUNCHES 8        /* kernels launched by the call */
#define PP_STAT_T_PARTITION 9     /* seconds in partition + commit kernels (profile = 1) */
#define PP_STAT_BUCKET_ROT 10     /* rotations run by the bucketed kernel (k_bk_rotate) */
#define PP_STAT_BUCKET_BYTES 11   /* algorithmic bytes of those rotations: B * (terms in + terms out) */
#define PP_STATS_LEN 16

/* _alloc_spv (type_SparsePauliVector.jl:94-104) / SparsePauliVector(N, T; capacity)
 * (type_SparsePauliVector.jl:138-141).  append_cap is the reference's logical
 * append capacity, which drives the early-merge rule (spv_evolve.jl:356-362).
 * N > 128 -> PP_ERROR_EXCEPTION (type_SparsePauliVector.jl:25). */
int pp_create(int32_t N, int64_t live_cap, int64_t append_cap, pp_spv **out);
/* Finalizer of the Julia shim. */
int pp_destroy(pp_spv *h);
/* Constructor fill + _sort_live! (type_SparsePauliVector.jl:167-188).  sorted != 0:
 * input already strictly increasing (skip the device sort).  Keys must be unique. */
int pp_upload(pp_spv *h, const void *z, const void *x, const double *c, int64_t n, int32_t sorted);
/* PauliSum(v) gather (type_SparsePauliVector.jl:212-221): copies min(n, cap) terms
 * to the caller's buffers (host or device pointers) and returns n. */
int pp_download(pp_spv *h, void *z, void *x, double *c, int64_t cap, int64_t *n);
/* length(v) (type_SparsePauliVector.jl:363). */
int pp_length(pp_spv *h, int64_t *n);
/* copy(v) (type_SparsePauliVector.jl:249-254). */
int pp_copy(pp_spv *h, pp_spv **out);
/* evolve!(O, G, θ) (spv_evolve.jl:228-236): one rotation, NOFILTER. */
int pp_evolve1(pp_spv *h, const void *gz, const void *gx, double cos_theta, double sin_theta);
/* evolve!(O, generators, angles; window, truncation, local_truncation, correction,
 * counters) (spv_evolve.jl:312-387).  gz/gx: L packed generator words; cosv/sinv:
 * host-computed cos(θ_i), sin(θ_i) (spv_evolve.jl:341-342). */
int pp_evolve(pp_spv *h, const void *gz, const void *gx, const double *cosv, const double *sinv,
              int64_t L, const pp_evolve_opts *opts);
/* Batched instances for pp_evolve_batch.  Instance i's terms are 128-bit words
 * (the handle is created with N > 64): bits 0..63 of z / x are the instance's own
 * nq-qubit word (as a UInt64 SparsePauliVector of N = nq would hold it), bits
 * 64..127 of z hold i, bits 64..127 of x are zero. */
typedef struct {
    int64_t ninst;                /* instances */
    int32_t nq;                   /* qubits of every instance (1..64) */
    int32_t ncol;                 /* angle columns */
    const int32_t *acol;          /* [L] angle column of each rotation */
    const double *cosv, *sinv;    /* [ninst * ncol] cos / sin of instance i's column j at [i * ncol + j] */
    const int64_t *rot_end;       /* [ninst] rotations instance i runs: the first rot_end[i] of the L */
    int32_t keep_finished;        /* 0: an instance's terms leave the vector when it finishes */
    int32_t pad;
    double *expect_out;           /* [ninst] <ket|O_i|ket> after its last rotation (nullable) */
    double *t_done;               /* [ninst] device seconds from the call's start to that result (nullable) */
    int64_t *n_final;             /* [ninst] terms of instance i after its last rotation (nullable) */
} pp_batch;

/* The sequence evolve! (spv_evolve.jl:312-387) of many independent vectors in one
 * pass: equivalent, instance by instance, to evolve!(v_i, gens[1:rot_end[i]],
 * angles_i; truncation) at window = 1 with an append capacity large enough that no
 * early merge happens (spv_evolve.jl:356-362), plus opts->chan_kind applied after
 * every chan_every-th rotation the instance runs (the channel acts on the nq
 * instance qubits, or on opts->chan_mask's word 0).  gz/gx: L generators as
 * 128-bit words acting on bits 0..nq-1 only.  The strict filter's weights count
 * word 0 only.  opts may be NULL; window must be 1; local truncation, adaptive
 * truncation and corrections are rejected.  No counterpart in the reference (its
 * vectors evolve one at a time). */
int pp_evolve_batch(pp_spv *h, const void *gz, const void *gx, int64_t L, const pp_batch *b,
                    const pp_evolve_opts *opts);
/* ---- Learned truncation.  No counterpart in the reference (which truncates by
 * coefficient and weight only).  A 16 -> 64 -> 64 -> 1 GELU network predicts
 * log10 |contribution of a term to the final expectation value| from 16 term
 * features; a budget truncation keeps the `budget` terms of largest prediction
 * (ties: the smaller (z, x) key).  Matrices are BF16 on the tensor cores with
 * FP32 accumulation; parameters are an FP32 vector of PP_MLP_NPARAM values laid
 * out W1[64][16], b1[64], W2[64][64], b2[64], w3[64], b3. */
#define PP_MLP_NPARAM 5313
typedef struct pp_mlp pp_mlp;

/* Position of a vector in its circuit and the lattice geometry the features use
 * (N <= 64 qubits; qubit q is bit q-1). */
typedef struct {
    int32_t nq;                   /* qubits */
    int32_t pad;
    uint64_t nbr[64];             /* neighbour mask of each qubit */
    uint64_t light_cone;          /* qubits in the remaining circuit's light cone */
    uint64_t boundary;            /* qubits on the lattice boundary */
    uint8_t row[64], col[64];     /* lattice coordinates of each qubit */
    float layer_frac;             /* layers done / total layers */
    float remaining_frac;         /* layers to go / total layers */
    float theta_j, theta_h;       /* the circuit's angles */
} pp_feature_ctx;

int pp_mlp_create(pp_mlp **out);
int pp_mlp_destroy(pp_mlp *m);
/* Sets / reads the FP32 parameters (host or device pointers); set resets Adam. */
int pp_mlp_set_params(pp_mlp *m, const float *params);
int pp_mlp_get_params(pp_mlp *m, float *params);
/* out[i] = network(feat[i][0..15]) for i < n (host or device pointers). */
int pp_mlp_forward(pp_mlp *m, const float *feat, int64_t n, float *out);
/* Gradient of mean_i (network(feat[i]) - target[i])^2 over all n rows with respect to
 * the parameters (PP_MLP_NPARAM floats) and the loss. */
int pp_mlp_grad(pp_mlp *m, const float *feat, const float *target, int64_t n, float *grad, float *loss);
/* Copies a training set (n rows of 16 features and a target) to the device. */
int pp_mlp_load_data(pp_mlp *m, const float *feat, const float *target, int64_t n);
/* `steps` Adam steps (lr; betas 0.9, 0.999) on minibatches of `batch` rows drawn
 * without replacement per epoch (seeded shuffle); loss_out[steps] gets each step's
 * minibatch loss (nullable). */
int pp_mlp_train(pp_mlp *m, int64_t steps, int64_t batch, float lr, uint64_t seed, float *loss_out);
/* The 16 features of each live term (n x 16 FP32, host or device; at most cap rows);
 * *n_out = live count. */
int pp_features(pp_spv *h, const pp_feature_ctx *ctx, float *out, int64_t cap, int64_t *n_out);
/* Stratified random sample of the live terms (N <= 64), for building training
 * sets: nbins equal-width bins of log10 |c| over [lg_lo, lg_hi) (outside values
 * fall into the end bins), about 0.9 per_bin terms from each bin (all of a bin
 * with fewer), chosen by a hash of (seed, index); at most cap rows, in no
 * particular order. */
int pp_sample_terms(pp_spv *h, int32_t nbins, double lg_lo, double lg_hi, int64_t per_bin, uint64_t seed,
                    void *z, void *x, double *c, int64_t cap, int64_t *n_out);
/* Uniform sample of the terms a budget truncation drops (for auditing the cut):
 * up to cap terms (word 0 of z / x, coefficient), each dropped term taken with
 * probability 0.9 cap / n_dropped by a hash of (seed, its index). */
typedef struct {
    int64_t cap;                  /* in: buffer rows (0: no sample) */
    uint64_t seed;                /* in */
    void *z, *x;                  /* out: host or device, cap words each */
    double *c;                    /* out: cap coefficients */
    int64_t n;                    /* out: rows written */
    int64_t n_dropped;            /* out: terms the cut dropped */
} pp_drop_sample;
/* Budget truncation: when more than `budget` terms are live, keeps exactly the
 * `budget` of largest network output (computed from the live terms in one fused
 * pass), in key order.  *cut_score: the smallest kept output (-inf when nothing
 * was dropped).  sample: nullable. */
int pp_learned_truncate(pp_spv *h, pp_mlp *m, const pp_feature_ctx *ctx, int64_t budget, float *cut_score,
                        pp_drop_sample *sample);

/* coeff_clip! / weight_clip! / x_weight_clip! / majorana_weight_clip! /
 * weight_damped_clip! / x_weight_damped_clip! and the compilable truncate!
 * (spv_evolve.jl:13-26, 59-65) -> _compact_spv! (spv_kernels.jl:395-408). */
int pp_compact(pp_spv *h, const pp_filter *f);
/* Largest term count pp_compact_static accepts: the size its static scratch covers. */
#define PP_COMPACT_STATIC_MAX_TERMS (1 << 25)
/* No counterpart in the reference.  The clip / compaction of pp_compact for a
 * caller that cannot allocate device memory — one whose device memory is owned by
 * another allocator, or that calls from a phase where allocating is not allowed —
 * and so cannot hold a pp_spv handle.  Reads n terms (z, x, c: device arrays in
 * the word layout above), writes the terms that filter f keeps, in order, to
 * z_out / x_out / c_out (device arrays with room for n terms), and stores their
 * count in *n_out (host).  Allocates nothing: its look-back scratch is a static
 * device array of 8 + PP_COMPACT_STATIC_MAX_TERMS/1024 words that every GPU loading
 * the library holds until exit.  The first call in each CUDA context on a device looks
 * up that array's address, so make it before any stream capture.  All calls share
 * the scratch: calls whose work overlaps on the GPU race on it.
 * n > PP_COMPACT_STATIC_MAX_TERMS gives PP_ARGUMENT_ERROR.  stream: a cudaStream_t
 * (NULL: the default stream); every call synchronizes it before returning, because
 * the survivor count is read back to *n_out. */
int pp_compact_static(int32_t N, const void *z, const void *x, const double *c, int64_t n, const pp_filter *f,
                      void *z_out, void *x_out, double *c_out, int64_t *n_out, void *stream);
/* _apply!(v, ::AdaptiveTruncation) (spv_evolve.jl:103-114). */
int pp_adaptive(pp_spv *h, int64_t max_terms, double min_thresh);
/* stochastic_clip!(v, epsilon) (spv_evolve.jl:35-52) and _apply!(v,
 * ::StochasticSamplingTruncation) (spv_evolve.jl:69-99).  Random numbers come from a
 * counter-based generator keyed by seed and term index (the reference's Julia RNG
 * stream cannot be reproduced; results agree in distribution). */
int pp_stochastic_clip(pp_spv *h, double epsilon, uint64_t seed);
int pp_stochastic_sample(pp_spv *h, int64_t n_keep, uint64_t seed);
/* depolarizing_channel! (channels.jl:223-232, kind 0), dephasing_channel! (234-243, 1),
 * bit_flip_channel! (245-254, 2), bit_phase_flip_channel! (256-265, 3),
 * pauli_channel! (203-221, 4).  prm: p, or pX,pY,pZ for kind 4.  qubit_mask: one
 * word (NULL = all qubits) as _spv_mask (channels.jl:200-201). */
int pp_channel(pp_spv *h, int32_t kind, const double *prm, const void *qubit_mask);
/* ---- SparsePauliVector algebra (spv_ops.jl) for real (Float64) coefficients. */
/* mul!(v, a) (spv_ops.jl:12-17); with pp_copy it gives -v and v * a (:19-30). */
int pp_scale(pp_spv *h, double a);
/* norm(v, p) (spv_ops.jl:57-86): p = 2, 1, INFINITY, or any other p > 0. */
int pp_norm(pp_spv *h, double p, double *out);
/* tr(v) (spv_ops.jl:52-55): the identity coefficient times 2^N, where 2^N is the
 * reference's Int64 power (it wraps: 0 for N >= 64). */
int pp_trace(pp_spv *h, double *out);
/* sum!(h, o) (spv_ops.jl:182-190) for sign = +1; h += -o for sign = -1 (with pp_copy:
 * v1 + v2, v1 - v2, spv_ops.jl:131-167).  Unfiltered merge: zero sums are kept.
 * o may be h. */
int pp_sum(pp_spv *h, pp_spv *o, double sign);
/* inner_product(a, b) (spv_ops.jl:378-399): sum over shared keys of c_a c_b. */
int pp_inner_product(pp_spv *a, pp_spv *b, double *out);
/* out = a * b (kind 0, spv_ops.jl:257-284), anticommutator!(out, a, b) (kind 1,
 * :460-470) or commutator!(out, a, b) (kind 2, :446-458).  A real-typed product with
 * an imaginary coefficient and every real commutator raise PP_ERROR_EXCEPTION, as the
 * reference does.  out may be a or b; its previous contents are replaced. */
int pp_product(pp_spv *out, pp_spv *a, pp_spv *b, int32_t kind);
/* variance(v, ::Ket) (statistics.jl:6-22): <psi|O^2|psi> - <psi|O|psi>^2.  ket: one word. */
int pp_variance(pp_spv *h, const void *ket, double *out);
/* expectation_value(v, ::Ket) (spv_evolve.jl:133-134) -> _expectation_spv
 * (spv_kernels.jl:441-452).  ket: one word. */
int pp_expect_ket(pp_spv *h, const void *ket, double *out);
/* check_spv (type_SparsePauliVector.jl:263-278): *ok = 1 if live keys are strictly
 * increasing and within capacity. */
int pp_check(pp_spv *h, int32_t *ok);
/* The handle's CUDA stream (cudaStream_t), for callers that time with events. */
int pp_stream(pp_spv *h, void **stream);
/* Bytes of device memory held by the handle. */
int pp_device_bytes(pp_spv *h, int64_t *bytes);
/* lambda^k for k = 0..kmax with the compensated integer power used by the channel
 * tables (the algorithm of Julia's Float64^Integer). Host-only helper. */
int pp_power_table(double lambda, int32_t kmax, double *out);
/* Message of the last failing call on this thread. */
const char *pp_last_error(void);

/* Launch configuration of the bucketed window-1 rotations (no counterpart in the
 * reference; results do not depend on it).  (bucket_cap, items_per_thread) must be
 * a compiled variant: (128, 4), (256, 4), (512, 4), (256, 8), (512, 8) or
 * (1024, 8); a CTA of 256 threads has two staging areas of 256 * items_per_thread
 * terms (a group of bucket pairs in one, the next group's terms in the other).
 * load_div (3..16): bucketing aims at a mean load of at most bucket_cap /
 * load_div.  chunk (8..256): rotations launched between host checks.
 * pauliprop's autotuner (pauliprop/tune.py) measures the variants on the device
 * and caches the fastest per (word count, SM count); a new handle starts with
 * (512, 4, 6, 128). */
typedef struct {
    int32_t bucket_cap, items_per_thread, load_div, chunk;
} pp_tuning;
int pp_set_tuning(pp_spv *h, const pp_tuning *t);
int pp_get_tuning(pp_spv *h, pp_tuning *t);
/* The handle's device: multiprocessor count and compute capability (the key of the
 * tuning cache). */
int pp_device_info(pp_spv *h, int32_t *sm_count, int32_t *cc_major, int32_t *cc_minor);

/* Key-sharded window-1 evolution over 2^rank_bits ranks (no counterpart in the
 * reference, whose evolve! runs in one process; spv_kernels.jl:3-5 names a
 * multi-device engine as future work).  Rank r holds the keys P with owner(P) = r,
 * owner being rank_bits GF(2)-linear parities of P (pp_shard_owner, host-side);
 * the sin branch P xor M then belongs to rank r xor owner(M), so each rotation
 * exchanges terms with one partner rank.  Per rotation r, on every rank:
 *   pp_shard_send   packs into device buffers the local terms that anticommute
 *                   with G_r and survive the early-merge pre-filter (pref), and
 *                   names the partner rank (itself when nothing is to be sent);
 *   the caller moves them to the partner (NCCL, peer copies, ...);
 *   pp_shard_recv   takes the partner's terms (device buffers) as foreign terms;
 *   pp_shard_rotate runs the rotation: stats5 = local {terms in, terms out, sin
 *                   branches created, pre-filter survivors, largest bucket}.
 * The caller sums the counts over ranks for the early-merge rule
 * (spv_evolve.jl:356-362: pref = global n > append capacity) and, when the
 * largest bucket of any rank passes bucket_cap / 2, calls pp_shard_regrid with
 * one more bucket bit on every rank.  pp_shard_begin takes the call's options
 * (window 1, a compiled truncation, no correction, no WindowCounters) and the
 * bucket bits every rank uses; pp_shard_end returns the local set to the dense
 * sorted layout and gives this shard's part of <ket|O|ket>. */
int pp_shard_owner(int32_t nw, const void *z, const void *x, int64_t n, int32_t rank_bits, int32_t *owner);
int pp_shard_begin(pp_spv *h, int32_t rank_bits, int32_t rank, const void *gz, const void *gx, const double *cosv,
                   const double *sinv, int64_t L, const pp_evolve_opts *opts, int32_t bits, int32_t *maxcnt);
int pp_shard_send(pp_spv *h, int64_t r, int32_t pref, void *z_out, void *x_out, double *c_out, int64_t cap,
                  int64_t *n_out, int32_t *partner);
int pp_shard_recv(pp_spv *h, const void *z, const void *x, const double *c, int64_t n);
int pp_shard_rotate(pp_spv *h, int64_t r, int32_t pref, int64_t *stats5);
int pp_shard_regrid(pp_spv *h, int32_t bits, int32_t *maxcnt);
int pp_shard_end(pp_spv *h, double *expect_partial, double *stats_out);

/* Test hooks for failure detection (no counterpart in the reference, which has no
 * device).  pp_debug_fail_alloc: the after-th next device allocation of any handle
 * fails with PP_OUT_OF_MEMORY, once (after <= 0 disarms); every growth is
 * transactional, so the handle keeps its previous live set.
 * pp_debug_lookback_timeout: runs one look-back wait on a status that nothing
 * publishes, bounded by limit polls (1..2^22); returns PP_TIMEOUT when the wait
 * gives up as it must, and the device stays usable.
 * pp_debug_bucket_limit: bucket layouts of more than `slots` term slots count as
 * not fitting in device memory (slots <= 0: only the real free memory limits
 * them); a sequence whose live set outgrows the layout that fits continues on the
 * sorted-merge kernels with the same result. */
int pp_debug_fail_alloc(int64_t after);
int pp_debug_lookback_timeout(int64_t limit);
int pp_debug_bucket_limit(int64_t slots);

#ifdef __cplusplus
}
#endif

#endif /* PAULIPROP_H */
