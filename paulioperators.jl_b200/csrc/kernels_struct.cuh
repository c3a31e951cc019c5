// Window-1 rotation as a sort-free pass structure (the GPU counterpart of
// _rotate_range! + _gather_append! + _unshuffle_ws! + _try_merge!,
// spv_kernels.jl:146-177, 187-193, 262-363, driven as in spv_evolve.jl:352-385).
//
// The sin branches of one rotation are the keys P xor M (M = (gz, gx)) of the
// anticommuting live terms P.  Since live is sorted, the appended keys are
// sorted by key xor M; their sorted position is the rank identity
//   rank(P xor M) = rank(P) + sum_{b in M} ([P_b = 0] - [P_b = 1]) * sib_b(P),
// where sib_b(P) counts emitted terms that share P's bits above level b and
// differ at b.  sib_b comes from the positions where the "highest differing
// bit" h between consecutive emitted keys crosses b and b+1, i.e. from
// forward/backward max/min scans.  Kernels:
//   k_classify  (A1) per-segment compaction of emitting terms, h, tile aggregates
//   k_tilescan  (A2) one CTA: tile offsets and cross-tile scan carries
//   k_permute   (A3) final ranks -> src[rank] = physical live index (no key traffic)
//   k_partition (P)  merge-path split of (live, virtual sorted appends)
//   k_merge     (B)  merge + reduce-by-key + filter + channel epilogue
//   k_commit         segment table of the output, counters, partial reductions
// The appended keys are never materialised: B gathers live[src[k]] and applies
// the xor and the phase on the fly.
//
// Live layout: a segment table.  Segment k (all non-empty) holds the terms of
// dense indices [soff[k], soff[k+1]) at physical positions sphys[k] + j of the
// live set `cur`.  A window-1 merge writes each output tile to its own SEG-term
// slot (no cross-tile offset wait) and k_commit lists the non-empty slots; a
// dense live set is the table with sphys[k] = soff[k] = k * SEG.
#pragma once
#include "blockscan.cuh"

// Optional per-phase cycle counters of the merge kernel (thread 0 of each CTA;
// compiled only with -DPP_PHASE_TIMERS, for tuning experiments).
#ifdef PP_PHASE_TIMERS
__device__ unsigned long long pp_phase_cycles[8];
#define PHASE_MARK(i)                                                              \
    do {                                                                           \
        if (threadIdx.x == 0) {                                                    \
            long long now_ = clock64();                                            \
            atomicAdd(&pp_phase_cycles[i], (unsigned long long)(now_ - ph_t_));    \
            ph_t_ = now_;                                                          \
        }                                                                          \
    } while (0)
#define PHASE_START() long long ph_t_ = clock64()
#else
#define PHASE_MARK(i) do {} while (0)
#define PHASE_START() do {} while (0)
#endif

namespace pp {

struct Bufs {
    u64 *z[2], *x[2];
    double *c[2];
    long long cap;
    // structured path
    int *srcidx;
    unsigned *meta;
    int *src;
    TileAggA *aggA;
    int *offA, *hfirstA, *fwdA, *bwdA;
    // merge
    int *split_i, *split_j, *split_k;
    u64 *tstat;
    double *part;
    // general path (direct V = sorted appends)
    u64 *az, *ax;
    double *ac;
    long long acap;
    long long *rec;               // nullable: per-rotation counters [rot][4] (window 1)
    int *sphys, *soff;            // live segment table: physical base / dense start [nseg + 1]
    int *kcnt;                    // survivors per merge tile (window-1 merge)
    // batched instances (NW = 2 only): the instance index of a term is its z word 1
    const double *bcos, *bsin;    // [ninst * ncol] cos / sin of each instance's angle columns
    const long long *bend;        // [ninst] rotations each instance runs
    long long ninst;
    int ncol;
    int batch;                    // 1: the live set holds batched instances
    u64 *vz, *vx;
    double *vc;
    u64 *gstat;
    DevState *S;
    const DevParams *P;
    const GenRec *gens;
};

constexpr int TAUV = 8;   // scan thresholds sharing one vector block scan

__device__ __forceinline__ int tau_value(const GenRec &g, int tau) {
    return (int)g.level[tau >> 1] + (tau & 1);
}

// Rotation angle of a term at rotation `rot`: the generator's own cos/sin, or for
// batched instances the term's instance's angle column; false when the instance
// has finished (it no longer rotates, creates no sin branch and gets no channel).
template <int NW>
__device__ __forceinline__ bool term_angle(const Bufs &B, const GenRec &g, long long rot, const Key<NW> &k,
                                           double *cv, double *sv) {
    if constexpr (NW == 2) {
        if (B.batch) {
            const u64 t = k.z[1];
            if (t >= (u64)B.ninst) { atomicOr(&B.S->err, ERR_BOUNDS); return false; }
            if (rot >= B.bend[t]) return false;
            const long long i = (long long)t * B.ncol + g.acol;
            *cv = B.bcos[i];
            *sv = B.bsin[i];
            return true;
        }
    }
    *cv = g.cosv;
    *sv = g.sinv;
    return true;
}

// A batched term whose instance ran its last rotation before `rot`.
template <int NW>
__device__ __forceinline__ bool term_finished(const Bufs &B, long long rot, const Key<NW> &k) {
    if constexpr (NW == 2) {
        if (B.batch) {
            const u64 t = k.z[1];
            return t >= (u64)B.ninst || rot >= B.bend[t];
        }
    }
    return false;
}

// ---------------------------------------------------------------- A1 classify
// One tile per live segment: anticommutation, tile-local compaction of the terms
// that emit a sin branch, their h levels and the tile aggregates.  srcidx holds
// the physical index of each emitting term (used by the merge's gather).
template <int NW>
__global__ void __launch_bounds__(A_THREADS, 2) k_classify(Bufs B) {
    DevState *S = B.S;
    if (S->err) return;
    const long long rot = S->rot;
    if (rot >= S->rot_end) return;
    __shared__ GenRec g;
    __shared__ int wtot[A_ITEMS * (A_THREADS / 32)];
    __shared__ int s_total;
    __shared__ int s_first[TAU_MAX], s_last[TAU_MAX];
    extern __shared__ u64 sm[];
    u64 *skz = sm;                    // [NW][A_TILE]
    u64 *skx = sm + NW * A_TILE;      // [NW][A_TILE]
    unsigned char *sh = reinterpret_cast<unsigned char *>(sm + 2 * NW * A_TILE);  // [A_TILE]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) g = B.gens[rot];
    __syncthreads();
    const DevParams &P = *B.P;
    const long long n = S->n;
    const int cur = S->cur;
    const bool pref = n > S->acap_logical;
    const bool local_on = P.local_active != 0;
    const u64 *Z = B.z[cur], *X = B.x[cur];
    const double *C = B.c[cur];
    const int ntiles = (int)S->nseg;
    const int ntau = 2 * g.k;
    const bool need_c = pref || local_on;

    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long long pbase = B.sphys[t];
        const int tcnt = B.soff[t + 1] - B.soff[t];
        bool emit[A_ITEMS];
        Key<NW> key[A_ITEMS];
#pragma unroll
        for (int it = 0; it < A_ITEMS; ++it) {
            const int idx = it * A_THREADS + tid;
            emit[it] = false;
            if (idx < tcnt) {
                key[it] = load_key<NW>(Z, X, pbase + idx);
                double c = 0.0;
                if (need_c) c = C[pbase + idx];
                Key<NW> q;
                double sg, cv, sv;
                if (rotate_term<NW>(key[it], g, &q, &sg) && term_angle<NW>(B, g, rot, key[it], &cv, &sv)) {
                    bool ok = true;
                    if (pref && should_drop<NW>(P.strict, key[it], fabs(c))) ok = false;
                    if (ok && local_on) {
                        const double cn = __dmul_rn(sg * sv, c);
                        if (should_drop<NW>(P.local, q, fabs(cn))) ok = false;
                    }
                    emit[it] = ok;
                }
            }
        }
        int lpre[A_ITEMS];
#pragma unroll
        for (int it = 0; it < A_ITEMS; ++it) {
            unsigned m = __ballot_sync(0xffffffffu, emit[it]);
            lpre[it] = __popc(m & lanemask_lt());
            if (lane == 0) wtot[it * (A_THREADS / 32) + warp] = __popc(m);
        }
        __syncthreads();
        if (warp == 0) {
            // exclusive scan of the A_ITEMS x NWARPS row-major warp counts
            constexpr int NE = A_ITEMS * (A_THREADS / 32);
            constexpr int PER = (NE + 31) / 32;
            int v[PER];
            int s = 0;
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                const int e = lane * PER + q;
                v[q] = e < NE ? wtot[e] : 0;
                s += v[q];
            }
            int incl = warp_incl_scan(s, OpSum());
            int ex = incl - s;
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                const int e = lane * PER + q;
                if (e < NE) wtot[e] = ex;
                ex += v[q];
            }
            if (lane == 31) s_total = incl;
        }
        if (tid < TAU_MAX) { s_first[tid] = 0x7fff; s_last[tid] = -1; }
        __syncthreads();
        const int total = s_total;
#pragma unroll
        for (int it = 0; it < A_ITEMS; ++it) {
            if (emit[it]) {
                const int j = wtot[it * (A_THREADS / 32) + warp] + lpre[it];
#pragma unroll
                for (int w = 0; w < NW; ++w) { skz[w * A_TILE + j] = key[it].z[w]; skx[w * A_TILE + j] = key[it].x[w]; }
                B.srcidx[pbase + j] = (int)(pbase + it * A_THREADS + tid);
            }
        }
        __syncthreads();
        for (int j = tid; j < total; j += A_THREADS) {
            Key<NW> kj;
#pragma unroll
            for (int w = 0; w < NW; ++w) { kj.z[w] = skz[w * A_TILE + j]; kj.x[w] = skx[w * A_TILE + j]; }
            int h = 0xff;
            if (j > 0) {
                Key<NW> kp;
#pragma unroll
                for (int w = 0; w < NW; ++w) { kp.z[w] = skz[w * A_TILE + j - 1]; kp.x[w] = skx[w * A_TILE + j - 1]; }
                h = hdiff<NW>(kp, kj);
            }
            unsigned cls = 0;
            for (int i = 0; i < g.k; ++i) cls |= (unsigned)key_bit<NW>(kj, g.level[i]) << i;
            sh[j] = (unsigned char)h;
            B.meta[pbase + j] = (unsigned)h | (cls << 8);
        }
        __syncthreads();
        for (int tau = 0; tau < ntau; ++tau) {
            const int thr = tau_value(g, tau);
            int mn = 0x7fff, mx = -1;
            for (int j = tid; j < total; j += A_THREADS) {
                if (j > 0 && (int)sh[j] >= thr) { mn = min(mn, j); mx = max(mx, j); }
            }
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) {
                mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, d));
                mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, d));
            }
            if (lane == 0 && mx >= 0) { atomicMin(&s_first[tau], mn); atomicMax(&s_last[tau], mx); }
        }
        __syncthreads();
        if (tid == 0) {
            TileAggA *A = B.aggA + t;
            A->count = total;
            if (total > 0) {
#pragma unroll
                for (int w = 0; w < NW; ++w) {
                    A->first[w] = skz[w * A_TILE];
                    A->first[2 + w] = skx[w * A_TILE];
                    A->last[w] = skz[w * A_TILE + total - 1];
                    A->last[2 + w] = skx[w * A_TILE + total - 1];
                }
            }
        }
        if (tid < TAU_MAX) {
            B.aggA[t].firstpos[tid] = (short)s_first[tid];
            B.aggA[t].lastpos[tid] = (short)s_last[tid];
        }
        __syncthreads();
    }
}

template <int NW>
__device__ __forceinline__ Key<NW> agg_key(const u64 *w4) {
    Key<NW> k;
#pragma unroll
    for (int w = 0; w < NW; ++w) { k.z[w] = w4[w]; k.x[w] = w4[2 + w]; }
    return k;
}

// ---------------------------------------------------------------- A2 tilescan
constexpr int S_THREADS = 1024;
// Rotations with at most TS_CAP tiles and TS_TAU thresholds (every rotation of a
// one- or two-qubit generator up to ~5M live terms) stage the tile aggregates in
// shared memory with one coalesced pass; the scans then read shared memory only.
constexpr int TS_CAP = 2048;
constexpr int TS_TAU = 8;

template <int NW>
constexpr size_t tilescan_smem() {
    return (size_t)TS_CAP * (4 * NW * 8 + 3 * 4 + 2 * TS_TAU * 2);
}

template <int NW>
__device__ __forceinline__ Key<NW> ts_key(const u64 *k) {
    Key<NW> r;
#pragma unroll
    for (int w = 0; w < NW; ++w) { r.z[w] = k[w]; r.x[w] = k[NW + w]; }
    return r;
}

// The tile scan of k_tilescan below, from shared-memory copies of the aggregates.
template <int NW>
__device__ void tilescan_cached(const Bufs &B, const GenRec &g, int ntiles, long long n, long long *sml, int *smi,
                                int *svec) {
    DevState *S = B.S;
    extern __shared__ u64 tsm[];
    u64 *skey = tsm;                                                  // [TS_CAP][4 NW]: first (z, x), last (z, x)
    int *scnt = reinterpret_cast<int *>(tsm + (size_t)TS_CAP * 4 * NW);
    int *soffa = scnt + TS_CAP;
    int *shf = soffa + TS_CAP;
    short *sfp = reinterpret_cast<short *>(shf + TS_CAP);             // [TS_CAP][TS_TAU]
    short *slp = sfp + TS_CAP * TS_TAU;
    const int tid = threadIdx.x;
    const int ntau = 2 * g.k;
    for (int t = tid; t < ntiles; t += S_THREADS) {
        const TileAggA &A = B.aggA[t];
        const int c = A.count;
        scnt[t] = c;
        if (c > 0) {
#pragma unroll
            for (int w = 0; w < NW; ++w) {
                skey[t * 4 * NW + w] = A.first[w];
                skey[t * 4 * NW + NW + w] = A.first[2 + w];
                skey[t * 4 * NW + 2 * NW + w] = A.last[w];
                skey[t * 4 * NW + 3 * NW + w] = A.last[2 + w];
            }
        }
        for (int tau = 0; tau < ntau; ++tau) {
            sfp[t * TS_TAU + tau] = A.firstpos[tau];
            slp[t * TS_TAU + tau] = A.lastpos[tau];
        }
    }
    __syncthreads();
    const int tpt = (ntiles + S_THREADS - 1) / S_THREADS;
    const int t0 = min(tid * tpt, ntiles), t1 = min(t0 + tpt, ntiles);
    long long loc = 0;
    for (int t = t0; t < t1; ++t) loc += scnt[t];
    long long total;
    long long run = block_excl_scan<S_THREADS>(loc, 0ll, OpSum(), sml, &total);
    for (int t = t0; t < t1; ++t) { soffa[t] = (int)run; B.offA[t] = (int)run; run += scnt[t]; }
    const long long slots = max(1ll, (n + total + B_D - 1) / B_D);
    if (slots * SEG > B.cap || n + total > B.cap) {
        if (tid == 0) { S->err |= ERR_OVERFLOW; S->need = slots * SEG + SEG; }
        return;
    }
    if (tid == 0) S->a = total;
    int lastne = -1;
    for (int t = t0; t < t1; ++t) if (scnt[t] > 0) lastne = t;
    int tot_i;
    int carry = block_excl_scan<S_THREADS>(lastne, -1, OpMax(), smi, &tot_i);
    for (int t = t0; t < t1; ++t) {
        int hf = -1;
        if (scnt[t] > 0) {
            hf = carry >= 0 ? hdiff<NW>(ts_key<NW>(skey + carry * 4 * NW + 2 * NW), ts_key<NW>(skey + t * 4 * NW))
                            : H_INF;
            carry = t;
        }
        shf[t] = hf;
        B.hfirstA[t] = hf;
    }
    const int itotal = (int)total;
    auto tileL = [&](int t, int tau, int thr) {
        int L = shf[t] >= thr ? soffa[t] : -1;
        const int lp = slp[t * TS_TAU + tau];
        if (lp >= 0) L = max(L, soffa[t] + lp);
        return L;
    };
    auto tileF = [&](int t, int tau, int thr) {
        if (shf[t] >= thr) return soffa[t];
        const int fp = sfp[t * TS_TAU + tau];
        return fp != 0x7fff ? soffa[t] + fp : 0x7fffffff;
    };
    for (int g0 = 0; g0 < ntau; g0 += TAUV) {
        const int na = min(TAUV, ntau - g0);
        int lm[TAUV], fm[TAUV];
#pragma unroll
        for (int c = 0; c < TAUV; ++c) { lm[c] = -1; fm[c] = 0x7fffffff; }
        for (int t = t0; t < t1; ++t) {
            if (scnt[t] == 0) continue;
#pragma unroll
            for (int c = 0; c < TAUV; ++c) {
                if (c < na) {
                    const int thr = tau_value(g, g0 + c);
                    lm[c] = max(lm[c], tileL(t, g0 + c, thr));
                    fm[c] = min(fm[c], tileF(t, g0 + c, thr));
                }
            }
        }
        block_excl_scan_vec<S_THREADS, TAUV>(lm, -1, OpMax(), svec, na);
        block_excl_suffix_vec<S_THREADS, TAUV>(fm, 0x7fffffff, OpMin(), svec, na);
        for (int t = t0; t < t1; ++t) {
            const bool ne = scnt[t] > 0;
#pragma unroll
            for (int c = 0; c < TAUV; ++c) {
                if (c < na) {
                    B.fwdA[(long long)t * TAU_MAX + g0 + c] = lm[c];
                    if (ne) lm[c] = max(lm[c], tileL(t, g0 + c, tau_value(g, g0 + c)));
                }
            }
        }
        for (int t = t1 - 1; t >= t0; --t) {
            const bool ne = scnt[t] > 0;
#pragma unroll
            for (int c = 0; c < TAUV; ++c) {
                if (c < na) {
                    B.bwdA[(long long)t * TAU_MAX + g0 + c] = min(fm[c], itotal);
                    if (ne) fm[c] = min(fm[c], tileF(t, g0 + c, tau_value(g, g0 + c)));
                }
            }
        }
    }
}

template <int NW>
__global__ void __launch_bounds__(S_THREADS) k_tilescan(Bufs B) {
    DevState *S = B.S;
    if (S->err) return;
    const long long rot = S->rot;
    if (rot >= S->rot_end) return;
    __shared__ GenRec g;
    __shared__ long long sml[S_THREADS / 32 + 1];
    __shared__ int smi[S_THREADS / 32 + 1];
    __shared__ int svec[TAUV * (S_THREADS / 32)];
    const int tid = threadIdx.x;
    if (tid == 0) g = B.gens[rot];
    __syncthreads();
    const long long n = S->n;
    const int ntiles = (int)S->nseg;
    if (ntiles <= TS_CAP && 2 * g.k <= TS_TAU) {
        tilescan_cached<NW>(B, g, ntiles, n, sml, smi, svec);
        return;
    }
    const int tpt = (ntiles + S_THREADS - 1) / S_THREADS;
    const int t0 = min(tid * tpt, ntiles), t1 = min(t0 + tpt, ntiles);
    // tile offsets
    long long loc = 0;
    for (int t = t0; t < t1; ++t) loc += B.aggA[t].count;
    long long total;
    long long run = block_excl_scan<S_THREADS>(loc, 0ll, OpSum(), sml, &total);
    for (int t = t0; t < t1; ++t) { B.offA[t] = (int)run; run += B.aggA[t].count; }
    // the merge writes its tiles to fixed SEG-term slots: ceil((n + a) / B_D) of them
    const long long slots = max(1ll, (n + total + B_D - 1) / B_D);
    if (slots * SEG > B.cap || n + total > B.cap) {
        if (tid == 0) { S->err |= ERR_OVERFLOW; S->need = slots * SEG + SEG; }
        return;
    }
    if (tid == 0) S->a = total;
    // first-element h of every tile: against the last key of the previous non-empty tile
    int lastne = -1;
    for (int t = t0; t < t1; ++t) if (B.aggA[t].count > 0) lastne = t;
    int tot_i;
    int carry = block_excl_scan<S_THREADS>(lastne, -1, OpMax(), smi, &tot_i);
    for (int t = t0; t < t1; ++t) {
        int hf = -1;
        if (B.aggA[t].count > 0) {
            hf = carry >= 0 ? hdiff<NW>(agg_key<NW>(B.aggA[carry].last), agg_key<NW>(B.aggA[t].first)) : H_INF;
            carry = t;
        }
        B.hfirstA[t] = hf;
    }
    __syncthreads();
    const int ntau = 2 * g.k;
    const int itotal = (int)total;
    // Per threshold tau: forward = last global position with h >= tau strictly
    // before each tile; backward = first such position strictly after it.  The
    // thresholds of a group share one vector scan in each direction.
    auto tileL = [&](int t, int tau, int thr) {
        int L = B.hfirstA[t] >= thr ? B.offA[t] : -1;
        const int lp = B.aggA[t].lastpos[tau];
        if (lp >= 0) L = max(L, B.offA[t] + lp);
        return L;
    };
    auto tileF = [&](int t, int tau, int thr) {
        if (B.hfirstA[t] >= thr) return B.offA[t];
        const int fp = B.aggA[t].firstpos[tau];
        return fp != 0x7fff ? B.offA[t] + fp : 0x7fffffff;
    };
    for (int g0 = 0; g0 < ntau; g0 += TAUV) {
        const int na = min(TAUV, ntau - g0);
        int lm[TAUV], fm[TAUV];
#pragma unroll
        for (int c = 0; c < TAUV; ++c) { lm[c] = -1; fm[c] = 0x7fffffff; }
        for (int t = t0; t < t1; ++t) {
            if (B.aggA[t].count == 0) continue;
#pragma unroll
            for (int c = 0; c < TAUV; ++c) {
                if (c < na) {
                    const int thr = tau_value(g, g0 + c);
                    lm[c] = max(lm[c], tileL(t, g0 + c, thr));
                    fm[c] = min(fm[c], tileF(t, g0 + c, thr));
                }
            }
        }
        block_excl_scan_vec<S_THREADS, TAUV>(lm, -1, OpMax(), svec, na);
        block_excl_suffix_vec<S_THREADS, TAUV>(fm, 0x7fffffff, OpMin(), svec, na);
        for (int t = t0; t < t1; ++t) {
            const bool ne = B.aggA[t].count > 0;
#pragma unroll
            for (int c = 0; c < TAUV; ++c) {
                if (c < na) {
                    B.fwdA[(long long)t * TAU_MAX + g0 + c] = lm[c];
                    if (ne) lm[c] = max(lm[c], tileL(t, g0 + c, tau_value(g, g0 + c)));
                }
            }
        }
        for (int t = t1 - 1; t >= t0; --t) {
            const bool ne = B.aggA[t].count > 0;
#pragma unroll
            for (int c = 0; c < TAUV; ++c) {
                if (c < na) {
                    B.bwdA[(long long)t * TAU_MAX + g0 + c] = min(fm[c], itotal);
                    if (ne) fm[c] = min(fm[c], tileF(t, g0 + c, tau_value(g, g0 + c)));
                }
            }
        }
    }
}

// ---------------------------------------------------------------- A3 permute

// ---------------------------------------------------------------- A3 permute
// Thresholds are processed in groups of TAUV: per group one vector forward
// max-scan and one vector backward min-scan of per-thread aggregates, then each
// thread re-scans its A_ITEMS items in registers.

// Tiles with at most PW_CAP emitting terms (most of them: a rotation emits from
// a small fraction of the live terms) are permuted by one warp each, lane l
// owning items l*PW_ITEMS .. +PW_ITEMS-1, with the scans done by shuffles (no
// block barriers); larger tiles take the block path below.
constexpr int PW_ITEMS = 8;
constexpr int PW_CAP = 32 * PW_ITEMS;

template <int NW>
__device__ __forceinline__ void permute_warp_tile(const Bufs &B, const GenRec &g, int t, int cnt, long long atot,
                                                  int lane) {
    const int off = B.offA[t];
    const long long base = B.sphys[t];
    const int j0 = lane * PW_ITEMS;
    const int ntau = 2 * g.k;
    int h[PW_ITEMS];
    unsigned cls[PW_ITEMS];
    int delta[PW_ITEMS];
#pragma unroll
    for (int q = 0; q < PW_ITEMS; ++q) {
        const int j = j0 + q;
        const bool valid = j < cnt;
        const unsigned m = valid ? B.meta[base + j] : 0u;
        h[q] = valid ? (j == 0 ? B.hfirstA[t] : (int)(m & 0xffu)) : -1;
        cls[q] = m >> 8;
        delta[q] = 0;
    }
    for (int g0 = 0; g0 < ntau; g0 += TAUV) {
        const int na = min(TAUV, ntau - g0);
        int fw[TAUV], bw[TAUV];
#pragma unroll
        for (int c = 0; c < TAUV; ++c) {
            fw[c] = -1;
            bw[c] = 0x7fffffff;
            if (c < na) {
                const int thr = tau_value(g, g0 + c);
#pragma unroll
                for (int q = 0; q < PW_ITEMS; ++q)
                    if (h[q] >= thr) { fw[c] = off + j0 + q; bw[c] = min(bw[c], off + j0 + q); }
            }
        }
        // exclusive max-scan of fw over lower lanes, exclusive min-scan of bw over higher lanes,
        // then the carries from the other tiles
#pragma unroll
        for (int c = 0; c < TAUV; ++c) {
            if (c < na) {
                int v = fw[c], u = bw[c];
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const int o = __shfl_up_sync(0xffffffffu, v, d);
                    if (lane >= d) v = max(v, o);
                    const int p = __shfl_down_sync(0xffffffffu, u, d);
                    if (lane + d < 32) u = min(u, p);
                }
                int ev = __shfl_up_sync(0xffffffffu, v, 1);
                int eu = __shfl_down_sync(0xffffffffu, u, 1);
                if (lane == 0) ev = -1;
                if (lane == 31) eu = 0x7fffffff;
                fw[c] = max(ev, B.fwdA[(long long)t * TAU_MAX + g0 + c]);
                bw[c] = min(eu, B.bwdA[(long long)t * TAU_MAX + g0 + c]);
            }
        }
#pragma unroll
        for (int c = 0; c < TAUV; c += 2) {
            if (c + 1 >= na) continue;
            const int i = (g0 + c) >> 1;
            const int thr_ge = tau_value(g, g0 + c), thr_gt = tau_value(g, g0 + c + 1);
            int last_ge = fw[c], last_gt = fw[c + 1];
            int nxt_ge[PW_ITEMS], nxt_gt[PW_ITEMS];
            int run_ge = bw[c], run_gt = bw[c + 1];
#pragma unroll
            for (int q = PW_ITEMS - 1; q >= 0; --q) {
                nxt_ge[q] = run_ge;
                nxt_gt[q] = run_gt;
                if (h[q] >= thr_ge) run_ge = off + j0 + q;
                if (h[q] >= thr_gt) run_gt = off + j0 + q;
            }
#pragma unroll
            for (int q = 0; q < PW_ITEMS; ++q) {
                if (h[q] >= thr_ge) last_ge = off + j0 + q;
                if (h[q] >= thr_gt) last_gt = off + j0 + q;
                if ((cls[q] >> i) & 1u) delta[q] -= last_ge - last_gt;
                else delta[q] += nxt_gt[q] - nxt_ge[q];
            }
        }
    }
#pragma unroll
    for (int q = 0; q < PW_ITEMS; ++q) {
        const int j = j0 + q;
        if (j < cnt) {
            const long long pos = (long long)off + j + delta[q];
            if (pos >= 0 && pos < atot) B.src[pos] = B.srcidx[base + j];
            else atomicOr(&B.S->err, ERR_BOUNDS);
        }
    }
}

template <int NW>
__global__ void __launch_bounds__(A_THREADS, 2) k_permute(Bufs B) {
    DevState *S = B.S;
    if (S->err) return;
    const long long rot = S->rot;
    if (rot >= S->rot_end) return;
    __shared__ GenRec g;
    __shared__ unsigned smeta[A_TILE];
    __shared__ int ssrc[A_TILE];
    __shared__ int sscan[TAUV * (A_THREADS / 32)];
    const int tid = threadIdx.x;
    if (tid == 0) g = B.gens[rot];
    __syncthreads();
    const long long atot = S->a;
    const int ntiles = (int)S->nseg;
    const int ntau = 2 * g.k;
    {
        const int lane = tid & 31;
        const long long w0 = (long long)blockIdx.x * (A_THREADS / 32) + (tid >> 5);
        const long long nw = (long long)gridDim.x * (A_THREADS / 32);
        for (long long t = w0; t < ntiles; t += nw) {
            const int cnt = B.aggA[t].count;
            if (cnt == 0 || cnt > PW_CAP) continue;
            permute_warp_tile<NW>(B, g, (int)t, cnt, atot, lane);
        }
    }
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int cnt = B.aggA[t].count;
        if (cnt <= PW_CAP) continue;   // empty, or done by a warp above
        const int off = B.offA[t];
        const long long base = B.sphys[t];
        for (int j = tid; j < cnt; j += A_THREADS) { smeta[j] = B.meta[base + j]; ssrc[j] = B.srcidx[base + j]; }
        __syncthreads();
        const int j0 = tid * A_ITEMS;
        int h[A_ITEMS];
        unsigned cls[A_ITEMS];
        int delta[A_ITEMS];
#pragma unroll
        for (int q = 0; q < A_ITEMS; ++q) {
            const int j = j0 + q;
            const bool valid = j < cnt;
            h[q] = valid ? (j == 0 ? B.hfirstA[t] : (int)(smeta[j] & 0xffu)) : -1;
            cls[q] = valid ? (smeta[j] >> 8) : 0u;
            delta[q] = 0;
        }
        for (int g0 = 0; g0 < ntau; g0 += TAUV) {
            const int na = min(TAUV, ntau - g0);
            int fw[TAUV], bw[TAUV];
#pragma unroll
            for (int c = 0; c < TAUV; ++c) {
                fw[c] = -1;
                bw[c] = 0x7fffffff;
                if (c < na) {
                    const int thr = tau_value(g, g0 + c);
#pragma unroll
                    for (int q = 0; q < A_ITEMS; ++q)
                        if (h[q] >= thr) { fw[c] = off + j0 + q; bw[c] = min(bw[c], off + j0 + q); }
                }
            }
            block_excl_scan_vec<A_THREADS, TAUV>(fw, -1, OpMax(), sscan, na);
            block_excl_suffix_vec<A_THREADS, TAUV>(bw, 0x7fffffff, OpMin(), sscan, na);
#pragma unroll
            for (int c = 0; c < TAUV; ++c) {
                if (c < na) {
                    fw[c] = max(fw[c], B.fwdA[(long long)t * TAU_MAX + g0 + c]);
                    bw[c] = min(bw[c], B.bwdA[(long long)t * TAU_MAX + g0 + c]);
                }
            }
            // each mask level's two thresholds (b and b+1) lie in the same group
#pragma unroll
            for (int c = 0; c < TAUV; c += 2) {
                if (c + 1 >= na) continue;
                const int i = (g0 + c) >> 1;
                const int thr_ge = tau_value(g, g0 + c), thr_gt = tau_value(g, g0 + c + 1);
                int last_ge = fw[c], last_gt = fw[c + 1];
                int nxt_ge[A_ITEMS], nxt_gt[A_ITEMS];
                int run_ge = bw[c], run_gt = bw[c + 1];
#pragma unroll
                for (int q = A_ITEMS - 1; q >= 0; --q) {
                    nxt_ge[q] = run_ge;
                    nxt_gt[q] = run_gt;
                    if (h[q] >= thr_ge) run_ge = off + j0 + q;
                    if (h[q] >= thr_gt) run_gt = off + j0 + q;
                }
#pragma unroll
                for (int q = 0; q < A_ITEMS; ++q) {
                    if (h[q] >= thr_ge) last_ge = off + j0 + q;
                    if (h[q] >= thr_gt) last_gt = off + j0 + q;
                    if ((cls[q] >> i) & 1u) delta[q] -= last_ge - last_gt;
                    else delta[q] += nxt_gt[q] - nxt_ge[q];
                }
            }
        }
#pragma unroll
        for (int q = 0; q < A_ITEMS; ++q) {
            const int j = j0 + q;
            if (j < cnt) {
                const long long pos = (long long)off + j + delta[q];
                if (pos >= 0 && pos < atot) B.src[pos] = ssrc[j];
                else atomicOr(&S->err, ERR_BOUNDS);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- merge inputs
// MODE 0: structured window-1 rotation (V = live[src[k]] xor M, sin branch on the fly,
//         live cos branch applied on load).
// MODE 1: direct (V = sorted materialised appends; live already rotated).
// MODE 2: filter only (no V): the order-preserving compaction of the clip family.
template <int NW, int MODE>
__device__ __forceinline__ Key<NW> v_key(const Bufs &B, const GenRec &g, const u64 *Z, const u64 *X, long long k) {
    if constexpr (MODE == 0) {
        int p = B.src[k];
        if (p < 0 || p >= B.cap) { atomicOr(&B.S->err, ERR_BOUNDS); p = 0; }
        Key<NW> P = load_key<NW>(Z, X, p);
#pragma unroll
        for (int w = 0; w < NW; ++w) { P.z[w] ^= g.gz[w]; P.x[w] ^= g.gx[w]; }
        return P;
    } else {
        return load_key<NW>(B.vz, B.vx, k);
    }
}

template <int MODE>
__device__ __forceinline__ long long v_count(const DevState *S) {
    return MODE == 0 ? S->a : MODE == 1 ? S->an : 0ll;
}

// ---------------------------------------------------------------- P partition
// Merge-path split of (live, appended) at every multiple of B_D, one warp per
// split: 33-ary searches (each round the 32 lanes probe 32 interior points), so a
// split costs a few rounds of dependent loads instead of log_2(n).  For the
// window-1 rotation the live set is a segment table: the search first finds the
// segment by probing segment starts, then the position inside it, and records
// the segment (split_k) for the merge.
constexpr int P_THREADS = 256;

template <int NW, int MODE>
__global__ void __launch_bounds__(P_THREADS) k_partition(Bufs B) {
    DevState *S = B.S;
    if (S->err) return;
    if (MODE == 0 && S->rot >= S->rot_end) return;
    __shared__ GenRec gs;
    if constexpr (MODE == 0) {
        if (threadIdx.x == 0) gs = B.gens[S->rot];
        __syncthreads();
    }
    const GenRec &g = gs;
    const long long n = S->n, a = v_count<MODE>(S), tot = n + a;
    const int cur = S->cur;
    const u64 *Z = B.z[cur], *X = B.x[cur];
    const long long nsplit = max(1ll, (tot + B_D - 1) / B_D);
    const int nseg = MODE == 0 ? (int)S->nseg : 0;
    const int lane = threadIdx.x & 31;
    const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    // pred(i): live element i (at physical position p) precedes appended[d-i-1]
    auto pred = [&](long long d, long long i, long long p) {
        return !key_lt<NW>(v_key<NW, MODE>(B, g, Z, X, d - i - 1), load_key<NW>(Z, X, p));
    };
    for (long long s = warp0; s <= nsplit; s += nwarps) {
        const long long d = min(s * (long long)B_D, tot);
        long long lo = max(0ll, d - a), hi = min(d, n);
        long long seg_lo = 0, pbase = 0;          // dense start / physical base of the segment searched
        int kseg = 0;
        if constexpr (MODE == 0) {
            // level 1: first segment k whose start is not below the split (Q(k) false)
            auto Q = [&](int k) {
                const long long sk = B.soff[k];
                if (sk < lo) return true;
                if (sk >= hi) return false;
                return pred(d, sk, B.sphys[k]);
            };
            int klo = 0, khi = nseg;
            while (khi - klo > 32) {
                const long long span = khi - klo;
                const int p = klo + (int)((span * (lane + 1)) / 33);
                const unsigned m = __ballot_sync(0xffffffffu, !Q(p));
                if (m == 0) {
                    klo = __shfl_sync(0xffffffffu, p, 31) + 1;
                } else {
                    const int fl = __ffs(m) - 1;
                    const int pf = __shfl_sync(0xffffffffu, p, fl);
                    const int pprev = __shfl_sync(0xffffffffu, p, fl > 0 ? fl - 1 : 0);
                    khi = pf;
                    if (fl > 0) klo = pprev + 1;
                }
            }
            {
                const int p = klo + lane;
                const unsigned m = __ballot_sync(0xffffffffu, p < khi && !Q(p));
                klo = m ? klo + (__ffs(m) - 1) : khi;
            }
            const int K = klo - 1;                 // last segment whose start precedes the split
            if (K < 0) {
                hi = lo;                           // the split is at dense index 0
            } else {
                seg_lo = B.soff[K];
                pbase = B.sphys[K];
                lo = max(lo, seg_lo + 1);
                hi = min(hi, (long long)B.soff[K + 1]);
            }
            kseg = K < 0 ? 0 : K;
        }
        // level 2 (or the whole search for dense live): first i in [lo, hi) with pred false
        while (hi - lo > 32) {
            const long long span = hi - lo;
            const long long p = lo + (span * (lane + 1)) / 33;
            const bool f = !pred(d, p, pbase + p - seg_lo);
            const unsigned m = __ballot_sync(0xffffffffu, f);
            if (m == 0) {
                lo = __shfl_sync(0xffffffffu, p, 31) + 1;
            } else {
                const int fl = __ffs(m) - 1;
                const long long pf = __shfl_sync(0xffffffffu, p, fl);
                const long long pprev = __shfl_sync(0xffffffffu, p, fl > 0 ? fl - 1 : 0);
                hi = pf;
                if (fl > 0) lo = pprev + 1;
            }
        }
        {
            const long long p = lo + lane;
            const bool f = p < hi && !pred(d, p, pbase + p - seg_lo);
            const unsigned m = __ballot_sync(0xffffffffu, f);
            lo = m ? lo + (__ffs(m) - 1) : hi;
        }
        if (lane == 0) {
            long long i = lo, j = d - lo;
            if constexpr (MODE == 0) {
                // segment holding dense index i (nseg when i == n)
                if (i >= n) kseg = nseg;
                else if (nseg > 0 && i >= B.soff[kseg + 1]) kseg = kseg + 1;
            }
            // keep an equal-key run (live element followed by its appends) in one tile
            if (j < a && (i > 0 || j > 0)) {
                Key<NW> last;
                const long long pim1 = pbase + (i - 1) - seg_lo;   // live i-1 lies in the segment searched
                if (j > 0 && i > 0) {
                    const Key<NW> lv = load_key<NW>(Z, X, pim1);
                    const Key<NW> vv = v_key<NW, MODE>(B, g, Z, X, j - 1);
                    last = key_lt<NW>(vv, lv) ? lv : vv;
                } else if (j > 0) {
                    last = v_key<NW, MODE>(B, g, Z, X, j - 1);
                } else {
                    last = load_key<NW>(Z, X, pim1);
                }
                while (j < a && key_eq<NW>(v_key<NW, MODE>(B, g, Z, X, j), last)) ++j;
            }
            B.split_i[s] = (int)i;
            B.split_j[s] = (int)j;
            if constexpr (MODE == 0) B.split_k[s] = kseg;
        }
    }
}

// ---------------------------------------------------------------- B merge
constexpr int B_VPT = B_CAP / B_THREADS;   // staged inputs per thread (5)
constexpr int B_HALF = B_VPT;              // loads issued in one batch per tile
constexpr int B_SEGL = 256;                // live segments of a tile held in shared memory

template <int NW>
constexpr size_t merge_smem_bytes() {
    return (size_t)B_CAP * (2 * NW * 8 + 8 + 2 + 1) + 64;
}

// MODE 2 (clip family) filters with DevParams::clip; evolve modes with ::strict.
template <int MODE>
__device__ __forceinline__ const DevFilter &merge_filter(const DevParams &P) {
    if constexpr (MODE == 2) return P.clip; else return P.strict;
}

// Filter parameters held in registers for the merge epilogue; the damped
// exponential tables live in shared memory when a damped criterion is active.
struct FLite {
    long long wmax, xwmax, mwmax;
    double thresh, dthresh_w, dthresh_xw;
    int use_mw, use_dw, use_dxw, wlow;
};

__device__ __forceinline__ FLite flite(const DevFilter &f) {
    FLite r;
    r.wmax = f.wmax; r.xwmax = f.xwmax; r.mwmax = f.mwmax;
    r.thresh = f.thresh; r.dthresh_w = f.dthresh_w; r.dthresh_xw = f.dthresh_xw;
    r.use_mw = f.use_mw; r.use_dw = f.use_dw; r.use_dxw = f.use_dxw; r.wlow = f.wlow;
    return r;
}

// should_drop (spv_kernels.jl:64-79) with register parameters.
template <int NW>
__device__ __forceinline__ bool drop_lite(const FLite &f, const double *sexpw, const double *sexpxw, const Key<NW> &k,
                                          double absc) {
    if (absc <= f.thresh) return true;
    u64 o[NW], xx[NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) { o[w] = k.z[w] | k.x[w]; xx[w] = k.x[w]; }
    if constexpr (NW == 2) {
        if (f.wlow) { o[1] = 0; xx[1] = 0; }
    }
    const int wt = popc_w<NW>(o);
    if (wt > f.wmax) return true;
    const int xw = popc_w<NW>(xx);
    if (xw > f.xwmax) return true;
    if (f.use_mw && majorana_f<NW>(k, f.wlow) > f.mwmax) return true;
    if (f.use_dw && __dmul_rn(absc, sexpw[wt]) <= f.dthresh_w) return true;
    if (f.use_dxw && __dmul_rn(absc, sexpxw[xw]) <= f.dthresh_xw) return true;
    return false;
}

template <int NW>
__device__ __forceinline__ double chan_lite(int kind, const u64 *mask, const double *tX, const double *tY,
                                           const double *tZ, const Key<NW> &k) {
    if (kind == 4) {
        int nX = 0, nY = 0, nZ = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            const u64 xM = k.x[w] & mask[w], zM = k.z[w] & mask[w];
            nX += __popcll(xM & ~k.z[w]);
            nY += __popcll(xM & k.z[w]);
            nZ += __popcll(zM & ~k.x[w]);
        }
        return __dmul_rn(__dmul_rn(tX[nX], tY[nY]), tZ[nZ]);
    }
    int cnt = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        const u64 s = kind == 0 ? (k.z[w] | k.x[w]) : kind == 1 ? k.x[w] : kind == 2 ? k.z[w] : (k.x[w] ^ k.z[w]);
        cnt += __popcll(s & mask[w]);
    }
    return tX[cnt];
}

// One merge tile: the merge-path diagonal range [split[t], split[t+1]) of
// (live, appended).  Each CTA loops over tiles taken in order from a counter.
// A window-1 merge (MODE 0) writes each tile to its own SEG-term slot; the
// general merges (MODE 1, 2) find the tile's output offset by decoupled look-back
// in warp 0.

template <int NW, int MODE>
__global__ void __launch_bounds__(B_THREADS, 2) k_merge(Bufs B, int argflags) {
    DevState *S = B.S;
    if (S->err) return;
    if (MODE == 0 && S->rot >= S->rot_end) return;
    __shared__ GenRec g;
    __shared__ int s_next[2];
    __shared__ int s_sc[B_THREADS / 32 + 1];
    __shared__ double s_red[3][B_THREADS / 32];
    __shared__ unsigned s_base;
    __shared__ double s_expw[130], s_expxw[130];   // filter tables; the channel tables are read through L1
    __shared__ int s_so[B_SEGL], s_sp[B_SEGL];   // live segment list of the tile (MODE 0)
    extern __shared__ u64 sm[];
    u64 *skz = sm;                                                    // [NW][B_CAP]
    u64 *skx = skz + NW * B_CAP;                                      // [NW][B_CAP]
    double *sval = reinterpret_cast<double *>(skx + NW * B_CAP);      // [B_CAP] inputs, then outputs
    unsigned short *sperm = reinterpret_cast<unsigned short *>(sval + B_CAP);  // [B_CAP] merge order, then output slots
    unsigned char *sdead = reinterpret_cast<unsigned char *>(sperm + B_CAP);   // [B_CAP]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (MODE == 0 && tid == 0) g = B.gens[S->rot];
    if (tid == 0) s_next[0] = atomicAdd(&S->b_tile_ctr, 1);
    const DevParams &P = *B.P;
    const DevFilter &F = merge_filter<MODE>(P);
    const FLite fl = flite(F);
    for (int i = tid; i < 130; i += B_THREADS) {
        if (fl.use_dw) s_expw[i] = F.expw[i];
        if (fl.use_dxw) s_expxw[i] = F.expxw[i];
    }
    __syncthreads();
    const int flags = MODE == 0 ? g.flags : argflags;
    const bool do_chan = MODE != 2 && (flags & GEN_CHANNEL) != 0 && P.chan_kind >= 0;
    const bool do_corr = MODE != 2 && P.corr_kind == 1;
    const bool do_meas = (flags & GEN_MEASURE) != 0 || do_corr;
    const int chan_kind = P.chan_kind;
    const u64 chan_mask[2] = {P.chan_mask[0], P.chan_mask[1]};
    FLite fs;                       // early-merge pre-filter (the strict filter of the evolve call)
    if constexpr (MODE == 0) fs = flite(P.strict);
    const long long n = S->n, a = v_count<MODE>(S), tot = n + a;
    const int cur = S->cur;
    const u64 *Z = B.z[cur], *X = B.x[cur];
    const double *C = B.c[cur];
    u64 *OZ = B.z[cur ^ 1], *OX = B.x[cur ^ 1];
    double *OC = B.c[cur ^ 1];
    const int nsplit = (int)max(1ll, (tot + B_D - 1) / B_D);
    const int nseg = MODE == 0 ? (int)S->nseg : 0;
    const unsigned epoch = S->epoch;
    const bool pref = MODE == 0 && n > S->acap_logical;
    const u64 ket[2] = {P.ket[0], P.ket[1]};
    const long long rot = S->rot;
    const bool harvest = MODE == 2 && (flags & GEN_HARVEST) != 0;

    auto skey = [&](int slot) {
        Key<NW> k;
#pragma unroll
        for (int w = 0; w < NW; ++w) { k.z[w] = skz[w * B_CAP + slot]; k.x[w] = skx[w * B_CAP + slot]; }
        return k;
    };

    int it = 0;
    int t = s_next[0];
    while (t < nsplit) {
        if (tid == 0) s_next[(it + 1) & 1] = atomicAdd(&S->b_tile_ctr, 1);  // next tile index
        const int i0 = B.split_i[t], j0 = B.split_j[t];
        const int i1 = B.split_i[t + 1], j1 = B.split_j[t + 1];
        int nl = i1 - i0, nv = j1 - j0;
        bool tbad = (nl + nv > B_CAP) || nl < 0 || nv < 0 || i0 < 0 || j0 < 0 || i1 > n || j1 > a;
        if (tbad) { nl = 0; nv = 0; }
        int ks = 0, nsg = 1;
        const int *so = s_so, *sp = s_sp;
        if constexpr (MODE == 0) {
            // segments ks..ke hold the tile's live range [i0, i1): ks holds i0, ke
            // holds i1 (ke = nseg when i1 = n); every segment before ke holds one
            // of its terms, so nsg <= nl + 1
            ks = B.split_k[t];
            const int ke = B.split_k[t + 1];
            if (ks < 0 || ke > nseg || ke < ks) { tbad = true; nl = 0; nv = 0; ks = 0; }
            else nsg = ke - ks + 1;
            if (nsg <= B_SEGL) {
                for (int k = tid; k < nsg; k += B_THREADS) {
                    s_so[k] = B.soff[ks + k];
                    s_sp[k] = ks + k < nseg ? B.sphys[ks + k] : 0;
                }
            } else {
                so = B.soff + ks;
                sp = B.sphys + ks;
            }
            __syncthreads();
        }
        const int ntot = nl + nv;
        PHASE_START();
        // ---- stage the tile, two batches of loads each issued before its shared
        // stores: the live part gets the cos branch / early-merge pre-filter, the
        // appended part is the sin branch of live[src[k]] computed on the fly
        int nalive = 0;
#pragma unroll
        for (int hb = 0; hb < B_VPT / B_HALF; ++hb) {
            int srcp[B_HALF];
            Key<NW> kk[B_HALF];
            double cc[B_HALF];
#pragma unroll
            for (int q = 0; q < B_HALF; ++q) {
                const int e = tid + (hb * B_HALF + q) * B_THREADS;
                srcp[q] = 0;
                if constexpr (MODE == 0) {
                    if (e >= nl && e < ntot) {
                        int p = B.src[j0 + e - nl];
                        if (p < 0 || p >= B.cap) { atomicOr(&S->err, ERR_BOUNDS); p = 0; }
                        srcp[q] = p;
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < B_HALF; ++q) {
                const int e = tid + (hb * B_HALF + q) * B_THREADS;
                if (e < nl) {
                    long long p = i0 + e;
                    if constexpr (MODE == 0) {
                        // physical position: the last segment starting at or before i0 + e
                        int lo = 0, hi = nsg - 1;
                        while (lo < hi) {
                            const int mid = (lo + hi + 1) >> 1;
                            if (so[mid] <= i0 + e) lo = mid; else hi = mid - 1;
                        }
                        p = (long long)sp[lo] + (i0 + e - so[lo]);
                        if (p < 0 || p >= B.cap) { atomicOr(&S->err, ERR_BOUNDS); p = 0; }
                    }
                    kk[q] = load_key<NW>(Z, X, p);
                    cc[q] = C[p];
                } else if (e < ntot) {
                    if constexpr (MODE == 0) {
                        kk[q] = load_key<NW>(Z, X, srcp[q]);
                        cc[q] = C[srcp[q]];
                    } else {
                        kk[q] = load_key<NW>(B.vz, B.vx, j0 + e - nl);
                        cc[q] = B.vc[j0 + e - nl];
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < B_HALF; ++q) {
                const int e = tid + (hb * B_HALF + q) * B_THREADS;
                if (e >= ntot) continue;
                Key<NW> k = kk[q];
                double c = cc[q];
                unsigned char dead = 0;
                if constexpr (MODE == 0) {
                    Key<NW> qk;
                    double sg = 0.0, cv = 1.0, sv = 0.0;
                    const bool anti = rotate_term<NW>(k, g, &qk, &sg);
                    const bool act = term_angle<NW>(B, g, rot, k, &cv, &sv);
                    if (e < nl) {
                        if (pref && drop_lite<NW>(fs, F.expw, F.expxw, k, fabs(c))) dead = 1;
                        else if (anti && act) c = __dmul_rn(c, cv);
                        nalive += dead ? 0 : 1;
                    } else {
                        k = qk;
                        c = __dmul_rn(sg * sv, c);
                    }
                }
#pragma unroll
                for (int w = 0; w < NW; ++w) { skz[w * B_CAP + e] = k.z[w]; skx[w * B_CAP + e] = k.x[w]; }
                sval[e] = c;
                sdead[e] = dead;
            }
        }
        __syncthreads();
        PHASE_MARK(0);
        // ---- merge path inside the tile; each thread owns a contiguous output range
        // (live first on equal keys: spv_kernels.jl:338)
        const int ipt = (ntot + B_THREADS - 1) / B_THREADS;
        const int d0 = min(tid * ipt, ntot), dend = min(d0 + ipt, ntot);
        if (d0 < dend) {
            int lo = max(0, d0 - nv), hi = min(d0, nl);
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (!key_lt<NW>(skey(nl + d0 - mid - 1), skey(mid))) lo = mid + 1; else hi = mid;
            }
            int i = lo, j = d0 - lo;
            for (int d = d0; d < dend; ++d) {
                bool takeL;
                if (i >= nl) takeL = false;
                else if (j >= nv) takeL = true;
                else takeL = !key_lt<NW>(skey(nl + j), skey(i));
                sperm[d] = (unsigned short)(takeL ? i++ : nl + j++);
            }
        }
        __syncthreads();
        PHASE_MARK(1);
        // ---- reduce equal-key runs (live value first, then appends in order,
        // spv_kernels.jl:338-350), strict filter on the unscaled sum, channel epilogue
        double outq[B_VPT];
        unsigned short slotq[B_VPT];
        unsigned keepm = 0;
        Neu e_keep{0.0, 0.0}, e_drop{0.0, 0.0}, e_pre{0.0, 0.0};
        Key<NW> kprev;
        if (d0 > 0 && d0 < dend) kprev = skey(sperm[d0 - 1]);
#pragma unroll
        for (int q = 0; q < B_VPT; ++q) {
            const int p = d0 + q;
            outq[q] = 0.0;
            slotq[q] = 0;
            if (p >= dend) continue;
            const int sl = sperm[p];
            const Key<NW> kp = skey(sl);
            const bool head = !(p > 0 && key_eq<NW>(kprev, kp));
            kprev = kp;
            if (!head) continue;
            double acc = 0.0;
            bool have = false;
            const bool diag = is_diag<NW>(kp);
            const double sgn = diag ? ket_sign<NW>(kp, ket) : 0.0;
            for (int r = p; r < ntot; ++r) {
                const int sr = r == p ? sl : sperm[r];
                if (r > p && !key_eq<NW>(skey(sr), kp)) break;
                if (sdead[sr]) { if (diag && do_meas) e_pre.add(sgn * sval[sr]); continue; }
                acc = have ? __dadd_rn(acc, sval[sr]) : sval[sr];
                have = true;
            }
            if (!have) continue;
            // a finished batched instance is left as its last merge wrote it: no
            // filter, no channel (its terms passed its own last filter already)
            const bool fin = term_finished<NW>(B, rot, kp);
            if (!fin && drop_lite<NW>(fl, s_expw, s_expxw, kp, fabs(acc))) {
                if (diag && do_meas) e_drop.add(sgn * acc);
                continue;
            }
            if (harvest && fin) continue;
            const bool ch = do_chan && !fin;
            const double o = ch ? __dmul_rn(acc, chan_lite<NW>(chan_kind, chan_mask, P.chanX, P.chanY, P.chanZ, kp)) : acc;
            if (diag && do_meas) e_keep.add(sgn * o);
            outq[q] = o;
            slotq[q] = (unsigned short)sl;
            keepm |= 1u << q;
        }
        PHASE_MARK(2);
        const int kept = __popc(keepm);
        int tkept;
        const int loff = block_excl_scan<B_THREADS>(kept, 0, OpSum(), s_sc, &tkept);  // ends with a barrier
        PHASE_MARK(3);
        if constexpr (MODE == 0) {
            // window-1 merge: the tile's survivors go to its own SEG-term slot of
            // the other set (k_commit lists the non-empty slots), no look-back wait
            if (tid == 0) { s_base = (unsigned)((long long)t * SEG); B.kcnt[t] = tkept; }
        } else if (warp == 0) {
            const unsigned ex = lookback_warp(B.tstat, t, epoch, (unsigned)tkept, &S->err);
            if (lane == 0) s_base = ex;
        }
        PHASE_MARK(4);
        // outputs reuse the staging buffers (every read of sval / sperm is done)
        {
            int o = loff;
#pragma unroll
            for (int q = 0; q < B_VPT; ++q) if ((keepm >> q) & 1u) { sval[o] = outq[q]; sperm[o] = slotq[q]; ++o; }
        }
        const int tn = s_next[(it + 1) & 1];
        __syncthreads();
        PHASE_MARK(7);
        const long long obase = s_base;
        if (obase + tkept > B.cap) {
            if (tid == 0) atomicOr(&S->err, ERR_BOUNDS);
            tkept = 0;
        }
        for (int e = tid; e < tkept; e += B_THREADS) {
            store_key<NW>(OZ, OX, obase + e, skey(sperm[e]));
            OC[obase + e] = sval[e];
        }
        PHASE_MARK(5);
        if (tbad && tid == 0) atomicOr(&S->err, ERR_TILE);
        if (MODE == 0 && pref) {
            int na = nalive;
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) na += __shfl_xor_sync(0xffffffffu, na, d);
            if (lane == 0 && na) atomicAdd((unsigned long long *)&S->npref, (unsigned long long)na);
        }
        if (do_meas) {
            double v0 = e_keep.s + e_keep.c, v1 = e_drop.s + e_drop.c, v2 = e_pre.s + e_pre.c;
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) {
                v0 += __shfl_xor_sync(0xffffffffu, v0, d);
                v1 += __shfl_xor_sync(0xffffffffu, v1, d);
                v2 += __shfl_xor_sync(0xffffffffu, v2, d);
            }
            if (lane == 0) { s_red[0][warp] = v0; s_red[1][warp] = v1; s_red[2][warp] = v2; }
            __syncthreads();
            if (tid < 3) {
                double s = 0.0;
                for (int w = 0; w < B_THREADS / 32; ++w) s += s_red[tid][w];
                B.part[(long long)t * 4 + tid] = s;
            }
        }
        __syncthreads();
        PHASE_MARK(6);
        ++it;
        t = tn;
    }
}

// Commits a merge launch (one block, after k_merge): new live count and buffer
// parity, WindowCounters totals, the early-merge append-capacity rule
// (spv_evolve.jl:356-362), the ordered reduction of <ket|O|ket> and correction
// partials, and the reset of the tile dispenser.  Kept out of k_merge so that no
// CTA of a merge launch can observe a half-committed state.
template <int MODE>
__global__ void __launch_bounds__(256) k_commit(Bufs B, int argflags) {
    DevState *S = B.S;
    if (S->err & ~ERR_TIMEOUT) return;
    if (MODE == 0 && S->rot >= S->rot_end) return;
    __shared__ double s_p[3][256];
    const int tid = threadIdx.x;
    const DevParams &P = *B.P;
    const int flags = MODE == 0 ? B.gens[S->rot].flags : argflags;
    const bool do_corr = MODE != 2 && P.corr_kind == 1;
    const bool do_meas = (flags & GEN_MEASURE) != 0 || do_corr;
    const long long n = S->n, a = v_count<MODE>(S), tot = n + a;
    const int nsplit = (int)max(1ll, (tot + B_D - 1) / B_D);
    if (do_meas) {
        const int per = (nsplit + 255) / 256;
        Neu r0{0, 0}, r1{0, 0}, r2{0, 0};
        for (int tt = tid * per; tt < min(nsplit, (tid + 1) * per); ++tt) {
            r0.add(B.part[(long long)tt * 4 + 0]);
            r1.add(B.part[(long long)tt * 4 + 1]);
            r2.add(B.part[(long long)tt * 4 + 2]);
        }
        s_p[0][tid] = r0.s + r0.c; s_p[1][tid] = r1.s + r1.c; s_p[2][tid] = r2.s + r2.c;
        __syncthreads();
        if (tid == 0) {
            Neu f0{0, 0}, f1{0, 0}, f2{0, 0};
            for (int w = 0; w < 256; ++w) { f0.add(s_p[0][w]); f1.add(s_p[1][w]); f2.add(s_p[2][w]); }
            S->expect_val = f0.s + f0.c;
            S->measure_valid = 1;
            if (do_corr) S->corr_energy = __dsub_rn(S->corr_energy, __dadd_rn(f1.s + f1.c, f2.s + f2.c));
        }
    }
    __shared__ long long s_tot;
    __shared__ int s_nseg;
    __shared__ int s_scan[256 / 32 + 1];
    if constexpr (MODE == 0) {
        // window-1 merge: the segment table of the output, i.e. its non-empty tile
        // slots in tile order with the dense index of their first term
        const int per = (nsplit + 255) / 256;
        const int t0 = min(tid * per, nsplit), t1 = min(t0 + per, nsplit);
        int loc = 0, lne = 0;
        for (int tt = t0; tt < t1; ++tt) { const int k = B.kcnt[tt]; loc += k; lne += k > 0; }
        int all, nne;
        int run = block_excl_scan<256>(loc, 0, OpSum(), s_scan, &all);
        int pos = block_excl_scan<256>(lne, 0, OpSum(), s_scan, &nne);
        for (int tt = t0; tt < t1; ++tt) {
            const int k = B.kcnt[tt];
            if (k > 0) { B.sphys[pos] = tt * SEG; B.soff[pos] = run; ++pos; run += k; }
        }
        if (tid == 0) { B.soff[nne] = all; s_tot = all; s_nseg = nne; }
        __syncthreads();
    } else {
        if (tid == 0) s_tot = (long long)(unsigned)(st_load(B.tstat + (nsplit - 1)) & 0xffffffffu);
        __syncthreads();
    }
    if (tid == 0) {
        const bool pref = MODE == 0 && n > S->acap_logical;
        const long long total = s_tot;
        S->n = total;
        S->cur ^= 1;
        if (MODE == 0) {
            S->seg_dense = 0;
            S->nseg = s_nseg;
        } else {
            S->seg_dense = 1;   // dense output; the segment table is rebuilt before the next window-1 run
        }
        S->merge_in += tot;
        S->merge_out += total;
        if (total > S->peak) S->peak = total;
        if (MODE == 0) {
            S->live_in += n;
            S->created += a;
            const long long np = pref ? S->npref : n;
            if (B.rec) {
                // WindowCounters of this rotation (window = 1): an early boundary
                // merges n -> np first, the regular one np + a -> total
                long long *r = B.rec + 4 * S->rot;
                r[0] = a;
                r[1] = (pref ? n : 0) + np + a;
                r[2] = (pref ? np : 0) + total;
                r[3] = pref ? 1 : 0;
            }
            if (pref) {
                S->early += 1;
                if (np > S->acap_logical) S->acap_logical = max(2 * S->acap_logical, np);
                S->npref = 0;
            }
            S->rot += 1;
        }
        if (MODE == 1) S->an = 0;
        S->b_tile_ctr = 0;
        S->epoch += 1;
    }
}

// Segment table of a dense live set (set cur): segment k = terms [k SEG, (k+1) SEG).
__global__ void k_segdense(Bufs B) {
    DevState *S = B.S;
    if (!S->seg_dense) return;    // a segmented live set keeps the table its merge wrote
    const long long n = S->n;
    const int nseg = (int)((n + SEG - 1) / SEG);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k <= nseg; k += gridDim.x * blockDim.x) {
        if (k < nseg) B.sphys[k] = k * SEG;
        B.soff[k] = k < nseg ? k * SEG : (int)n;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) { S->nseg = nseg; S->seg_dense = 1; }
}

// Copies a segmented live set (set cur) densely into set cur^1; k_densify_commit
// then makes that the live set.
template <int NW>
__global__ void k_densify(Bufs B) {
    DevState *S = B.S;
    if (S->seg_dense) return;
    const int cur = S->cur;
    const int nseg = (int)S->nseg;
    const u64 *Zs = B.z[cur], *Xs = B.x[cur];
    const double *Cs = B.c[cur];
    u64 *Zd = B.z[cur ^ 1], *Xd = B.x[cur ^ 1];
    double *Cd = B.c[cur ^ 1];
    for (int k = blockIdx.x; k < nseg; k += gridDim.x) {
        const long long d0 = B.soff[k];
        const int cnt = B.soff[k + 1] - B.soff[k];
        const long long p0 = B.sphys[k];
        for (int e = threadIdx.x; e < cnt; e += blockDim.x) {
            store_key<NW>(Zd, Xd, d0 + e, load_key<NW>(Zs, Xs, p0 + e));
            Cd[d0 + e] = Cs[p0 + e];
        }
    }
}

__global__ void k_densify_commit(Bufs B) {
    DevState *S = B.S;
    if (threadIdx.x == 0 && blockIdx.x == 0 && !S->seg_dense) { S->cur ^= 1; S->seg_dense = 1; }
}

}  // namespace pp
