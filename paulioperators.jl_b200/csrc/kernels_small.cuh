// Window-1 rotations of a small live set in one CTA.  While the live set holds at
// most small_cap<NW>() terms, one launch runs rotation after rotation with the
// whole set in shared memory, instead of the six dependent launches per rotation
// of k_classify ... k_commit, whose fixed latency dominates small sets.  It is
// the same sequence (spv_evolve.jl:352-385, spv_kernels.jl:146-177, 326-386) with
// the same per-term arithmetic, so results are bit-identical to the multi-kernel
// path:
//   - early-merge pre-filter when n > acap (live terms failing the strict filter
//     emit nothing and are dropped, counted in the early-merge rule);
//   - cos branch c * cos in place, sin branch (P xor G, (k - 2) * sin * c);
//   - sin branches sorted (bitonic sort of an index array; keys are distinct);
//   - merge with live first on equal keys, sum, strict filter on the unscaled sum,
//     channel epilogue, <ket|O|ket> partials on a measured rotation;
//   - counters and WindowCounters records as k_commit writes them.
// The launch stops when the set outgrows the shared-memory capacity or the call's
// rotations are done, and leaves the live set dense in the other buffer set.  It
// does not handle local truncation, corrections or batched instances; the host
// launches it only without them.  No waits: every barrier is in uniform control
// flow, every loop is bounded by the rotation count or the set size.
#pragma once
#include "kernels_struct.cuh"

namespace pp {

constexpr int SM_THREADS = 1024;

template <int NW>
__host__ __device__ constexpr int small_cap() { return NW == 1 ? 2048 : 1024; }

// live [C], sin branches [C], merged survivors [2C] (keys and values), the sorted
// order of the sin branches [C], the merged order [2C], pre-filter marks [C]
template <int NW>
constexpr size_t small_smem() {
    constexpr size_t C = small_cap<NW>();
    return C * (2 * NW * 8 + 8) * 4 + C * 2 + 2 * C * 2 + C;
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
    constexpr int IPT = 2 * C / SM_THREADS;        // merged positions per thread at most
    constexpr int LPT = C / SM_THREADS;            // live terms per thread at most
    DevState *S = B.S;
    __shared__ int s_go, s_ndead;
    __shared__ int s_scan[SM_THREADS / 32 + 1];
    __shared__ double s_red[3][SM_THREADS / 32];
    __shared__ double s_expw[130], s_expxw[130];
    __shared__ GenRec g;
    extern __shared__ u64 sm[];
    u64 *Lz = sm, *Lx = Lz + NW * C;                       // live, sorted
    u64 *Az = Lx + NW * C, *Ax = Az + NW * C;              // sin branches, emission order
    u64 *Oz = Ax + NW * C, *Ox = Oz + NW * 2 * C;          // merged survivors, sorted
    double *Lc = reinterpret_cast<double *>(Ox + NW * 2 * C);
    double *Ac = Lc + C;
    double *Oc = Ac + C;
    unsigned short *sa = reinterpret_cast<unsigned short *>(Oc + 2 * C);   // sorted order of A
    unsigned short *sperm = sa + C;                        // merged order: slot < C live, else C + sorted A index
    unsigned char *sdead = reinterpret_cast<unsigned char *>(sperm + 2 * C);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (tid == 0) s_go = (S->err == 0 && S->rot < S->rot_end && S->n <= C) ? 1 : 0;
    __syncthreads();
    if (!s_go) return;
    const DevParams &P = *B.P;
    const DevFilter &F = P.strict;
    const FLite fl = flite(F);
    for (int i = tid; i < 130; i += SM_THREADS) {
        s_expw[i] = fl.use_dw ? F.expw[i] : 0.0;
        s_expxw[i] = fl.use_dxw ? F.expxw[i] : 0.0;
    }
    const u64 ket[2] = {P.ket[0], P.ket[1]};
    const int chan_kind = P.chan_kind;
    const u64 chan_mask[2] = {P.chan_mask[0], P.chan_mask[1]};
    const int cur = S->cur;
    int n = (int)S->n;
    {
        // the live set: dense, or the segment table of the last multi-kernel merge
        const u64 *Z = B.z[cur], *X = B.x[cur];
        const double *Cc = B.c[cur];
        const bool dense = S->seg_dense != 0;
        const int nseg = (int)S->nseg;
        for (int i = tid; i < n; i += SM_THREADS) {
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
            sm_put<NW>(Lz, Lx, C, i, load_key<NW>(Z, X, p));
            Lc[i] = Cc[p];
        }
    }
    long long rot = S->rot;
    const long long rot_end = S->rot_end;
    long long acap = S->acap_logical;
    long long created = 0, merge_in = 0, merge_out = 0, live_in = 0, early = 0, peak = S->peak;
    bool measured = false;
    double expect = 0.0;
    __syncthreads();

    for (;;) {
        if (tid == 0) g = B.gens[rot];
        if (tid == 0) s_ndead = 0;
        __syncthreads();
        const bool pref = n > acap;
        const int flags = g.flags;
        const bool do_chan = (flags & GEN_CHANNEL) != 0 && chan_kind >= 0;
        const bool do_meas = (flags & GEN_MEASURE) != 0;
        // ---- live terms: pre-filter, cos branch in place, sin branches
        bool emit[LPT];
        Key<NW> qk[LPT];
        double qc[LPT];
        int ne = 0, nd = 0;
#pragma unroll
        for (int q = 0; q < LPT; ++q) {
            const int i = tid + q * SM_THREADS;
            emit[q] = false;
            if (i < n) {
                const Key<NW> k = sm_key<NW>(Lz, Lx, C, i);
                const double c = Lc[i];
                const bool dead = pref && drop_lite<NW>(fl, s_expw, s_expxw, k, fabs(c));
                sdead[i] = dead ? 1 : 0;
                nd += dead ? 1 : 0;
                double sg = 0.0;
                if (!dead && rotate_term<NW>(k, g, &qk[q], &sg)) {
                    emit[q] = true;
                    qc[q] = __dmul_rn(sg * g.sinv, c);
                    Lc[i] = __dmul_rn(c, g.cosv);
                    ++ne;
                }
            }
        }
        if (nd) atomicAdd(&s_ndead, nd);
        int a;
        int off = block_excl_scan<SM_THREADS>(ne, 0, OpSum(), s_scan, &a);
#pragma unroll
        for (int q = 0; q < LPT; ++q) {
            if (emit[q]) { sm_put<NW>(Az, Ax, C, off, qk[q]); Ac[off] = qc[q]; ++off; }
        }
        // ---- sort the sin branches: bitonic over the next power of two, indices
        // at or beyond a ordered last
        int pa = 1;
        while (pa < a) pa <<= 1;
        for (int j = tid; j < pa; j += SM_THREADS) sa[j] = (unsigned short)j;
        __syncthreads();
        if (a > 1) {
            for (int k = 2; k <= pa; k <<= 1) {
                for (int j = k >> 1; j > 0; j >>= 1) {
                    for (int i = tid; i < pa; i += SM_THREADS) {
                        const int l = i ^ j;
                        if (l > i) {
                            const int u = sa[i], v = sa[l];
                            bool gt;   // element u after element v
                            if (u >= a) gt = v >= a ? u > v : true;
                            else if (v >= a) gt = false;
                            else gt = key_lt<NW>(sm_key<NW>(Az, Ax, C, v), sm_key<NW>(Az, Ax, C, u));
                            if (gt == ((i & k) == 0)) { sa[i] = (unsigned short)v; sa[l] = (unsigned short)u; }
                        }
                    }
                    __syncthreads();
                }
            }
        }
        auto skey = [&](int slot) {
            return slot < C ? sm_key<NW>(Lz, Lx, C, slot) : sm_key<NW>(Az, Ax, C, sa[slot - C]);
        };
        auto sval = [&](int slot) { return slot < C ? Lc[slot] : Ac[sa[slot - C]]; };
        // ---- merge path: each thread owns merged positions [d0, dend) (live first
        // on equal keys: spv_kernels.jl:338)
        const int tot = n + a;
        const int ipt = (tot + SM_THREADS - 1) / SM_THREADS;
        const int d0 = min(tid * ipt, tot), dend = min(d0 + ipt, tot);
        if (d0 < dend) {
            int lo = max(0, d0 - a), hi = min(d0, n);
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (!key_lt<NW>(skey(C + d0 - mid - 1), skey(mid))) lo = mid + 1; else hi = mid;
            }
            int i = lo, j = d0 - lo;
            for (int d = d0; d < dend; ++d) {
                bool takeL;
                if (i >= n) takeL = false;
                else if (j >= a) takeL = true;
                else takeL = !key_lt<NW>(skey(C + j), skey(i));
                sperm[d] = (unsigned short)(takeL ? i++ : C + j++);
            }
        }
        __syncthreads();
        // ---- reduce equal-key runs, strict filter on the unscaled sum, channel
        double outq[IPT];
        unsigned short slotq[IPT];
        unsigned keepm = 0;
        Neu e_keep{0.0, 0.0}, e_drop{0.0, 0.0}, e_pre{0.0, 0.0};
        Key<NW> kprev;
        if (d0 > 0 && d0 < dend) kprev = skey(sperm[d0 - 1]);
#pragma unroll
        for (int q = 0; q < IPT; ++q) {
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
            for (int r = p; r < tot; ++r) {
                const int sr = r == p ? sl : sperm[r];
                if (r > p && !key_eq<NW>(skey(sr), kp)) break;
                if (sr < C && sdead[sr]) { if (diag && do_meas) e_pre.add(sgn * Lc[sr]); continue; }
                const double v = sval(sr);
                acc = have ? __dadd_rn(acc, v) : v;
                have = true;
            }
            if (!have) continue;
            if (drop_lite<NW>(fl, s_expw, s_expxw, kp, fabs(acc))) {
                if (diag && do_meas) e_drop.add(sgn * acc);
                continue;
            }
            const double o = do_chan ? __dmul_rn(acc, chan_lite<NW>(chan_kind, chan_mask, P.chanX, P.chanY, P.chanZ, kp))
                                     : acc;
            if (diag && do_meas) e_keep.add(sgn * o);
            outq[q] = o;
            slotq[q] = (unsigned short)sl;
            keepm |= 1u << q;
        }
        int total;
        int o = block_excl_scan<SM_THREADS>(__popc(keepm), 0, OpSum(), s_scan, &total);
#pragma unroll
        for (int q = 0; q < IPT; ++q) {
            if ((keepm >> q) & 1u) {
                sm_put<NW>(Oz, Ox, 2 * C, o, skey(slotq[q]));
                Oc[o] = outq[q];
                ++o;
            }
        }
        if (do_meas) {
            // per warp in lane order, then the warps in order
            double v0 = e_keep.s + e_keep.c, v1 = e_drop.s + e_drop.c, v2 = e_pre.s + e_pre.c;
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) {
                v0 += __shfl_xor_sync(0xffffffffu, v0, d);
                v1 += __shfl_xor_sync(0xffffffffu, v1, d);
                v2 += __shfl_xor_sync(0xffffffffu, v2, d);
            }
            if (lane == 0) { s_red[0][warp] = v0; s_red[1][warp] = v1; s_red[2][warp] = v2; }
        }
        __syncthreads();
        if (do_meas) {
            Neu f0{0.0, 0.0};
            for (int w = 0; w < SM_THREADS / 32; ++w) f0.add(s_red[0][w]);
            expect = f0.s + f0.c;
            measured = true;
        }
        // ---- commit (every thread keeps the same counts; thread 0 records)
        const int ndead = s_ndead;
        const long long np = pref ? (long long)(n - ndead) : (long long)n;
        if (tid == 0 && B.rec) {
            long long *r = B.rec + 4 * rot;
            r[0] = a;
            r[1] = (pref ? n : 0) + np + a;
            r[2] = (pref ? np : 0) + total;
            r[3] = pref ? 1 : 0;
        }
        created += a;
        merge_in += tot;
        merge_out += total;
        live_in += n;
        if (total > peak) peak = total;
        if (pref) {
            early += 1;
            if (np > acap) acap = max(2 * acap, np);
        }
        n = total;
        ++rot;
        if (rot >= rot_end || n > C) break;
        // the survivors become the live set of the next rotation
        for (int i = tid; i < n; i += SM_THREADS) {
            sm_put<NW>(Lz, Lx, C, i, sm_key<NW>(Oz, Ox, 2 * C, i));
            Lc[i] = Oc[i];
        }
        __syncthreads();
    }
    // ---- the survivors, dense, into the other buffer set
    {
        u64 *Z = B.z[cur ^ 1], *X = B.x[cur ^ 1];
        double *Cc = B.c[cur ^ 1];
        if ((long long)n > B.cap) {
            if (tid == 0) atomicOr(&S->err, ERR_BOUNDS);
            return;
        }
        for (int i = tid; i < n; i += SM_THREADS) {
            store_key<NW>(Z, X, i, sm_key<NW>(Oz, Ox, 2 * C, i));
            Cc[i] = Oc[i];
        }
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
        if (measured) { S->expect_val = expect; S->measure_valid = 1; }
    }
}

}  // namespace pp
