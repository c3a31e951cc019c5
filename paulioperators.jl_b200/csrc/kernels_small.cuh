// Window-1 rotations of a small live set in one CTA.  While the live set holds at
// most small_cap<NW>() terms, one launch runs rotation after rotation with the
// whole set in shared memory, instead of one grid-wide launch per rotation,
// whose fixed latency dominates small sets.  It is the same sequence
// (spv_evolve.jl:352-385, spv_kernels.jl:146-177, 326-386) with the same per-term
// arithmetic, so results are bit-identical to the other paths.  As in the
// bucketed kernel, an output key sums at most two terms (the live P and the sin
// branch of its partner P xor M), so no order is needed between rotations:
//   - early-merge pre-filter when n > acap (live terms failing the strict filter
//     emit nothing and are dropped, counted in the early-merge rule);
//   - the live terms that anticommute with G and survive the pre-filter are
//     indexed in a shared-memory hash table (only they can be a partner);
//   - per live term: cos branch, partner lookup, partner's sin branch added to
//     the live value (its phase is -sg: k(P) + k(P xor M) = 0 mod 4), strict
//     filter on the unscaled sum, channel; a sin branch whose partner is absent
//     becomes a new term;
//   - counters and WindowCounters records as the other paths write them.
// Three barriers per rotation.  The set is sorted once, when the launch ends
// (bitonic over an index array; keys are distinct), and <ket|O|ket> of a
// measured last rotation is reduced on the sorted set.  The launch stops when
// the set outgrows small_cap or the call's rotations are done, and leaves the
// live set dense and sorted in the other buffer set.  It does not handle local
// truncation, corrections or batched instances; the host launches it only
// without them.  No waits: every barrier is in uniform control flow, every loop
// is bounded by the rotation count, the set size or the table size.
#pragma once
#include "kernels_struct.cuh"
#include "kernels_bucket.cuh"

namespace pp {

constexpr int SM_THREADS = 256;                   // 1024 measured 9 % slower on chain20 (idle warps at barriers)

template <int NW>
__host__ __device__ constexpr int small_cap() { return NW == 1 ? 2048 : 1024; }

// two term sets of 2C (the live set and the next one; a rotation at most doubles
// the set), the key index (16-bit slots, 2C), pre-filter marks (2C) and the final
// sort's index array (2C)
template <int NW>
constexpr size_t small_smem() {
    constexpr size_t C = small_cap<NW>();
    return 2 * (2 * C) * (2 * NW * 8 + 8) + 2 * C * 2 + 2 * C + 2 * C * 2;
}

template <int NW>
__device__ __forceinline__ Key<NW> sm_key(const u64 *Z, const u64 *X, int stride, int i) {
    Key<NW> k;
#pragma unroll
    for (int w = 0; w < NW; ++w) { k.z[w] = Z[w * stride + i]; k.x[w] = X[w * stride + i]; }
    return k;
}

template <int NW>
__device__ __forceinline__ void sm_put(u64 *Z, u64 *X, int stride, int i, const Key<NW> &k) {
#pragma unroll
    for (int w = 0; w < NW; ++w) { Z[w * stride + i] = k.z[w]; X[w * stride + i] = k.x[w]; }
}

template <int NW>
__global__ void __launch_bounds__(SM_THREADS, 1) k_small_run(Bufs B) {
    constexpr int C = small_cap<NW>();
    constexpr int C2 = 2 * C;                      // capacity of each term set
    constexpr int TAB = 2 * C;                     // key index slots
    constexpr int T = SM_THREADS;
    DevState *S = B.S;
    __shared__ int s_go;
    __shared__ int s_cnt[2][3];                    // per rotation parity: outputs, sin branches, pre-filtered
    __shared__ double s_red[SM_THREADS / 32];
    __shared__ double s_expw[130], s_expxw[130];
    __shared__ __align__(16) GenRec gs[2];         // this rotation's generator and the next one (prefetched)
    static_assert(sizeof(GenRec) % 16 == 0, "generator records copy in 16-byte pieces");
    constexpr int GQ = (int)(sizeof(GenRec) / 16);
    extern __shared__ u64 sm[];
    // term sets t = 0, 1: keys (NW words, stride C2) and coefficients
    auto tz = [&](int t) { return sm + t * (2 * NW + 1) * C2; };
    auto tx = [&](int t) { return sm + t * (2 * NW + 1) * C2 + NW * C2; };
    auto tc = [&](int t) { return reinterpret_cast<double *>(sm + t * (2 * NW + 1) * C2 + 2 * NW * C2); };
    unsigned short *tab = reinterpret_cast<unsigned short *>(sm + 2 * (2 * NW + 1) * C2);   // [TAB]
    unsigned char *sdead = reinterpret_cast<unsigned char *>(tab + TAB);                   // [C2]
    unsigned short *sa = reinterpret_cast<unsigned short *>(sdead + C2);                   // [C2]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (tid == 0) s_go = (S->err == 0 && S->rot < S->rot_end && S->n <= C) ? 1 : 0;
    __syncthreads();
    if (!s_go) return;
    const DevParams &P = *B.P;
    const DevFilter &F = P.strict;
    const FLite fl = flite(F);
    for (int i = tid; i < 130; i += T) {
        s_expw[i] = fl.use_dw ? F.expw[i] : 0.0;
        s_expxw[i] = fl.use_dxw ? F.expxw[i] : 0.0;
    }
    const u64 ket[2] = {P.ket[0], P.ket[1]};
    const int chan_kind = P.chan_kind;
    const u64 chan_mask[2] = {P.chan_mask[0], P.chan_mask[1]};
    const int cur = S->cur;
    int n = (int)S->n;
    int li = 0;                                    // the term set holding the live set
    {
        // the live set: dense, or the segment table of the last multi-kernel merge
        const u64 *Z = B.z[cur], *X = B.x[cur];
        const double *Cc = B.c[cur];
        const bool dense = S->seg_dense != 0;
        const int nseg = (int)S->nseg;
        for (int i = tid; i < n; i += T) {
            long long p = i;
            if (!dense) {
                int lo = 0, hi = nseg - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (B.soff[mid] <= i) lo = mid; else hi = mid - 1;
                }
                p = (long long)B.sphys[lo] + (i - B.soff[lo]);
            }
            if (p < 0 || p >= B.cap) { atomicOr(&S->err, ERR_BOUNDS); p = 0; }
            sm_put<NW>(tz(0), tx(0), C2, i, load_key<NW>(Z, X, p));
            tc(0)[i] = Cc[p];
        }
    }
    for (int i = tid; i < TAB / 8; i += T) reinterpret_cast<uint4 *>(tab)[i] = make_uint4(0u, 0u, 0u, 0u);
    if (tid < 6) (&s_cnt[0][0])[tid] = 0;
    long long rot = S->rot;
    const long long rot_end = S->rot_end;
    // the first generator; later ones are copied in during the rotation before
    auto fetch_gen = [&](int slot, long long q) {
        if (tid < GQ) {
            cp_async16(reinterpret_cast<char *>(&gs[slot]) + 16 * tid, reinterpret_cast<const char *>(B.gens + q) + 16 * tid);
            cp_async_commit();
        }
    };
    fetch_gen(0, rot);
    if (tid < GQ) cp_async_wait_all();
    long long acap = S->acap_logical;
    long long created = 0, merge_in = 0, merge_out = 0, live_in = 0, early = 0, peak = S->peak;
    bool measure_last = false;

    for (int par = 0;; par ^= 1) {
        __syncthreads();
        const GenRec &g = gs[par];
        if (rot + 1 < rot_end) fetch_gen(par ^ 1, rot + 1);   // the previous readers of that slot passed the barrier
        // the next rotation's counters start from zero (their last readers passed this barrier)
        if (tid < 3) s_cnt[par ^ 1][tid] = 0;
        const bool pref = n > acap;
        const int flags = g.flags;
        const bool do_chan = (flags & GEN_CHANNEL) != 0 && chan_kind >= 0;
        measure_last = (flags & GEN_MEASURE) != 0;
        const u64 *LZ = tz(li), *LX = tx(li);
        const double *LC = tc(li);
        u64 *OZ = tz(li ^ 1), *OX = tx(li ^ 1);
        double *OC = tc(li ^ 1);
        // ---- pre-filter marks, and the index of the live anticommuting terms
        int nd = 0, na = 0;
        for (int i = tid; i < n; i += T) {
            const Key<NW> k = sm_key<NW>(LZ, LX, C2, i);
            const bool dead = pref && drop_lite<NW>(fl, s_expw, s_expxw, k, fabs(LC[i]));
            sdead[i] = dead ? 1 : 0;
            nd += dead ? 1 : 0;
            if (dead || !anticommutes<NW>(k, g)) continue;
            ++na;
            unsigned h = bk_slot<NW, TAB>(k);
            for (int probe = 0; probe < TAB; ++probe) {
                if (atomicCAS(&tab[h], (unsigned short)0, (unsigned short)(i + 1)) == (unsigned short)0) break;
                h = (h + 1) & (TAB - 1);
            }
        }
        if (nd) atomicAdd(&s_cnt[par][2], nd);
        if (na) atomicAdd(&s_cnt[par][1], na);
        __syncthreads();
        // ---- outputs: own term (cos branch plus the partner's sin branch), new sin branches
        const int rounds = (n + T - 1) / T;
        for (int rd = 0; rd < rounds; ++rd) {
            const int i = rd * T + tid;
            bool own = false, nw_ = false;
            double oval = 0.0, nval = 0.0;
            Key<NW> kk, qk;
            if (i < n && !sdead[i]) {
                kk = sm_key<NW>(LZ, LX, C2, i);
                const double c = LC[i];
                double v = c;
                double sg = 0.0;
                if (rotate_term<NW>(kk, g, &qk, &sg)) {
                    v = __dmul_rn(c, g.cosv);
                    const double sv = g.sinv;
                    // the partner P xor G in the index (live, anticommuting, not pre-filtered)
                    int j = -1;
                    unsigned h = bk_slot<NW, TAB>(qk);
                    for (int probe = 0; probe < TAB; ++probe) {
                        const int e = tab[h];
                        if (e == 0) break;
                        if (e - 1 < n && key_eq<NW>(sm_key<NW>(LZ, LX, C2, e - 1), qk)) { j = e - 1; break; }
                        h = (h + 1) & (TAB - 1);
                    }
                    if (j >= 0) {
                        // live value first, then the partner's sin branch (phase -sg)
                        v = __dadd_rn(v, __dmul_rn(-(sg * sv), LC[j]));
                    } else {
                        const double sbr = __dmul_rn(sg * sv, c);   // (k - 2) * sin(theta) * c, spv_kernels.jl:163
                        if (!drop_lite<NW>(fl, s_expw, s_expxw, qk, fabs(sbr))) {
                            nval = do_chan ? __dmul_rn(sbr, chan_lite<NW>(chan_kind, chan_mask, P.chanX, P.chanY,
                                                                           P.chanZ, qk))
                                           : sbr;
                            nw_ = true;
                        }
                    }
                }
                if (!drop_lite<NW>(fl, s_expw, s_expxw, kk, fabs(v))) {
                    oval = do_chan ? __dmul_rn(v, chan_lite<NW>(chan_kind, chan_mask, P.chanX, P.chanY, P.chanZ, kk))
                                   : v;
                    own = true;
                }
            }
            // slots: the warp's claiming lanes take consecutive slots from one atomic
            const unsigned w1 = __ballot_sync(0xffffffffu, own), w2 = __ballot_sync(0xffffffffu, nw_);
            const int c1 = __popc(w1);
            const int leader = __ffs(w1 | w2) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(&s_cnt[par][0], c1 + __popc(w2));
            base = __shfl_sync(0xffffffffu, base, leader < 0 ? 0 : leader);
            const unsigned lt = (1u << lane) - 1u;
            if (own) {
                const int o = base + __popc(w1 & lt);
                if (o < C2) { sm_put<NW>(OZ, OX, C2, o, kk); OC[o] = oval; }
            }
            if (nw_) {
                const int o = base + c1 + __popc(w2 & lt);
                if (o < C2) { sm_put<NW>(OZ, OX, C2, o, qk); OC[o] = nval; }
            }
        }
        __syncthreads();
        for (int q = tid; q < TAB / 8; q += T) reinterpret_cast<uint4 *>(tab)[q] = make_uint4(0u, 0u, 0u, 0u);
        // ---- commit (every thread keeps the same counts; thread 0 records)
        const int total = s_cnt[par][0], a = s_cnt[par][1], ndead = s_cnt[par][2];
        const long long np = pref ? (long long)(n - ndead) : (long long)n;
        if (tid == 0 && B.rec) {
            long long *r = B.rec + 4 * rot;
            r[0] = a;
            r[1] = (pref ? n : 0) + np + a;
            r[2] = (pref ? np : 0) + total;
            r[3] = pref ? 1 : 0;
        }
        if (total > C2 && tid == 0) atomicOr(&S->err, ERR_BOUNDS);   // n + a <= 2n <= C2: never
        created += a;
        merge_in += n + a;
        merge_out += total;
        live_in += n;
        if (total > peak) peak = total;
        if (pref) {
            early += 1;
            if (np > acap) acap = max(2 * acap, np);
        }
        n = min(total, C2);
        li ^= 1;
        ++rot;
        if (tid < GQ) cp_async_wait_all();   // the next generator has landed (published by the next barrier)
        if (rot >= rot_end || n > C) break;
    }
    __syncthreads();
    // ---- sort the survivors once (bitonic over an index array; keys are distinct)
    const u64 *LZ = tz(li), *LX = tx(li);
    const double *LC = tc(li);
    int pa = 1;
    while (pa < n) pa <<= 1;
    for (int j = tid; j < pa; j += T) sa[j] = (unsigned short)j;
    __syncthreads();
    for (int k = 2; k <= pa; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < pa; i += T) {
                const int l = i ^ j;
                if (l > i) {
                    const int u = sa[i], v = sa[l];
                    bool gt;   // element u after element v
                    if (u >= n) gt = v >= n ? u > v : true;
                    else if (v >= n) gt = false;
                    else gt = key_lt<NW>(sm_key<NW>(LZ, LX, C2, v), sm_key<NW>(LZ, LX, C2, u));
                    if (gt == ((i & k) == 0)) { sa[i] = (unsigned short)v; sa[l] = (unsigned short)u; }
                }
            }
            __syncthreads();
        }
    }
    // ---- the survivors, dense and sorted, into the other buffer set; <ket|O|ket>
    // of a measured last rotation over the sorted set (contiguous runs per thread,
    // compensated, then lanes and warps in a fixed order)
    u64 *Z = B.z[cur ^ 1], *X = B.x[cur ^ 1];
    double *Cc = B.c[cur ^ 1];
    if ((long long)n > B.cap) {
        if (tid == 0) atomicOr(&S->err, ERR_BOUNDS);
        return;
    }
    const int per = (n + T - 1) / T;
    const int i0 = min(tid * per, n), i1 = min(i0 + per, n);
    Neu acc{0.0, 0.0};
    for (int i = i0; i < i1; ++i) {
        const int src = sa[i];
        const Key<NW> k = sm_key<NW>(LZ, LX, C2, src);
        const double c = LC[src];
        store_key<NW>(Z, X, i, k);
        Cc[i] = c;
        if (measure_last && is_diag<NW>(k)) acc.add(ket_sign<NW>(k, ket) * c);
    }
    double expect = 0.0;
    if (measure_last) {
        double v = acc.s + acc.c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double y = __shfl_down_sync(0xffffffffu, v, d);
            if ((lane & (2 * d - 1)) == 0) v += y;
        }
        if (lane == 0) s_red[warp] = v;
        __syncthreads();
        Neu f{0.0, 0.0};
        for (int w = 0; w < T / 32; ++w) f.add(s_red[w]);
        expect = f.s + f.c;
    }
    if (tid == 0) {
        S->n = n;
        S->cur = cur ^ 1;
        S->seg_dense = 1;
        S->rot = rot;
        S->acap_logical = acap;
        S->created += created;
        S->merge_in += merge_in;
        S->merge_out += merge_out;
        S->live_in += live_in;
        S->early += early;
        S->peak = peak;
        S->npref = 0;
        if (measure_last) { S->expect_val = expect; S->measure_valid = 1; }
    }
}

}  // namespace pp
