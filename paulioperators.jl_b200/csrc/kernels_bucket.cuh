// Window-1 rotations over a hash-bucketed live set: one kernel per rotation.
//
// A window-1 rotation (_rotate_range! + _merge_spv!, spv_kernels.jl:146-177,
// 326-386, driven as in spv_evolve.jl:352-385) maps the live set {P} to
// {P} ∪ {P xor M : P anticommutes with G}, M = (gz, gx), and sums each output
// key from at most two terms: the live P (cos branch, or unchanged) and the sin
// branch of P xor M, which is live and anticommutes whenever P does.  IEEE
// addition of two terms is commutative, so no order among the terms is needed
// to reproduce the reference's coefficients bit for bit; only the set of
// partners is.
//
// The live set is kept in 2^bits buckets of CAP slots.  A term's bucket is
// h(P), a GF(2)-linear hash: bit r of h(P) is the parity of P & R_r for fixed
// pseudo-random rows R_r.  Linearity gives h(P xor M) = h(P) xor h(M), so for
// the rotation's generator the partner of every term of bucket b lies in bucket
// b xor delta, delta = h(M), and the sin branch of a term of b belongs to
// b xor delta as well.  A CTA therefore owns whole bucket pairs {b, b xor delta}
// (two neighbouring buckets when delta = 0): it loads a group of pairs into
// shared memory, indexes their keys in a shared-memory hash table, finds each
// anticommuting term's partner there, and appends each output term to its
// bucket of the other bucket set (positions from shared-memory counters, so the
// order inside a bucket is arbitrary; nothing depends on it).  No cross-CTA
// scan, sort or wait is involved.
//
// Per rotation, per term: the early-merge pre-filter, the cos branch, the sum
// with the partner's sin branch (or a new term when the partner is absent or was
// pre-filtered), the local filter on sin branches, the strict filter on the
// unscaled sum, and the channel factor -- the same arithmetic, in the same
// rounding steps, as the sorted-merge kernels.  The live set goes back to a
// dense, sorted layout (gather + radix sort) when the call ends.
#pragma once
#include "blockscan.cuh"

namespace pp {

// Compiled (bucket capacity, items per thread) variants; the autotuner picks
// one per device.  A CTA of BK_THREADS threads stages up to BK_THREADS * ITEMS
// terms: a group of up to that many / CAP bucket pairs, processed in one pass
// when their terms fit (else in consecutive sub-groups; a single pair always
// fits, 2 * CAP <= BK_THREADS * ITEMS), with a shared-memory key index of twice
// as many slots.
constexpr int BK_ROWS = 26;                    // hash rows: at most 2^26 buckets
constexpr int BK_THREADS = 256;
constexpr int BK_DEFAULT_CAP = 256;
constexpr int BK_DEFAULT_ITEMS = 8;

// Per-rotation record: rec[r] describes the live set entering rotation r (the
// output of rotation r - 1); rotation r reads it and fills rec[r + 1].
struct BkRec {
    long long n_in;                 // live terms entering the rotation (written by CTA 0)
    long long acap;                 // the reference's append capacity in effect (CTA 0)
    unsigned long long n_out;       // survivors (sum over CTAs)
    unsigned long long np;          // survivors of the early-merge pre-filter (when pref)
    unsigned long long created;     // sin branches appended (after the local filter)
    int pref;                       // the rotation began with an early merge (CTA 0)
    int maxcnt;                     // largest output bucket
};

struct BkArgs {
    u64 *z[2], *x[2];               // bucket sets: slot j of bucket b at b * CAP + j (NW words per key)
    double *c[2];
    int *cnt[2];                    // terms per bucket
    int bits;                       // 2^bits buckets
    int group;                      // bucket pairs per CTA (a power of two)
    const u64 *rows;                // [BK_ROWS][4]: z words 0..1, x words 0..1 of each hash row
    BkRec *rec;
    DevState *S;
    const DevParams *P;
    const GenRec *gens;
};

// Bucket of a key: the low `bits` bits of the GF(2)-linear hash.
template <int NW>
__device__ __forceinline__ unsigned bk_hash(const u64 *kz, const u64 *kx, const u64 *rows, int bits) {
    unsigned h = 0;
    for (int r = 0; r < bits; ++r) {
        const u64 *R = rows + 4 * r;
        int p = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) p += __popcll(kz[w] & R[w]) + __popcll(kx[w] & R[2 + w]);
        h |= (unsigned)(p & 1) << r;
    }
    return h;
}

// Slot hash of the shared-memory key index (a mix of all key bits).
template <int NW, int TAB>
__device__ __forceinline__ unsigned bk_slot(const Key<NW> &k) {
    u64 h = k.z[0] * 0x9E3779B97F4A7C15ull ^ (k.x[0] + 0x632BE59BD9B4E019ull) * 0xC2B2AE3D27D4EB4Full;
    if constexpr (NW == 2) h ^= k.z[1] * 0xD6E8FEB86659FD93ull ^ (k.x[1] + 0x165667B19E3779F9ull) * 0x94D049BB133111EBull;
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    return (unsigned)(h >> 40) & (TAB - 1);
}

template <int NW, int CAP, int ITEMS>
__host__ __device__ constexpr size_t bk_smem_bytes() {
    return (size_t)(BK_THREADS * ITEMS) * (2 * NW * 8 + 8 + 1 + 1) + (size_t)(2 * BK_THREADS * ITEMS) * 4;
}
template <int CAP, int ITEMS>
__host__ __device__ constexpr int bk_group_max() { return BK_THREADS * ITEMS / CAP; }

// Position in output bucket lb for every lane that passes `want`: lanes of a warp
// with the same bucket take consecutive slots from one shared-memory atomic.
__device__ __forceinline__ int bk_claim(int *s_out, int lb, bool want) {
    const unsigned act = __ballot_sync(0xffffffffu, want);
    int pos = -1;
    if (want) {
        const unsigned peers = __match_any_sync(act, lb);
        const int leader = __ffs(peers) - 1;
        const int lane = threadIdx.x & 31;
        int base = 0;
        if (lane == leader) base = atomicAdd(&s_out[lb], __popc(peers));
        base = __shfl_sync(peers, base, leader);
        pos = base + __popc(peers & ((1u << lane) - 1u));
    }
    return pos;
}

// One window-1 rotation: CTA blockIdx.x owns bucket pairs
// [blockIdx.x * group, (blockIdx.x + 1) * group).  k is the rotation's index
// within the launched group of rotations (rotation S->bk_rot0 + k, input set
// (S->bk_cur0 + k) & 1).
template <int NW, int CAP, int ITEMS>
__global__ void __launch_bounds__(BK_THREADS, ITEMS >= 16 ? 1 : ITEMS >= 8 ? 3 : 4) k_bk_rotate(BkArgs A, int k) {
    constexpr int T = BK_THREADS;
    constexpr int SMI = T * ITEMS;                 // staged terms
    constexpr int TAB = 2 * SMI;                   // key index slots
    constexpr int GMAX = bk_group_max<CAP, ITEMS>();
    constexpr int NBK = 2 * GMAX;                  // buckets of a group
    static_assert(GMAX >= 2, "a pair of full buckets fits");
    DevState *S = A.S;
    if (S->err) return;
    const long long r = S->bk_rot0 + k;
    if (r >= S->rot_end) return;
    const int cur = (S->bk_cur0 + k) & 1;
    __shared__ GenRec g;
    __shared__ unsigned s_delta;
    __shared__ int s_b[NBK], s_n[NBK], s_out[NBK], s_off[NBK + 1];
    __shared__ int s_j1, s_bad;
    __shared__ int s_red[3][T / 32];
    extern __shared__ u64 bsm[];
    u64 *skz = bsm;                                                     // [NW][SMI]
    u64 *skx = skz + NW * SMI;                                          // [NW][SMI]
    double *sc = reinterpret_cast<double *>(skx + NW * SMI);            // [SMI]
    unsigned *tab = reinterpret_cast<unsigned *>(sc + SMI);             // [TAB]
    unsigned char *sdead = reinterpret_cast<unsigned char *>(tab + TAB);  // [SMI]
    unsigned char *sbk = sdead + SMI;                                   // [SMI] local bucket of each term
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        g = A.gens[r];
        s_delta = bk_hash<NW>(g.gz, g.gx, A.rows, A.bits);
        s_bad = 0;
    }
    // the state entering this rotation, from the previous rotation's record (the
    // early-merge rule of spv_evolve.jl:356-362)
    const BkRec &prev = A.rec[r];
    const long long n_r = (long long)prev.n_out;
    long long acap = prev.acap;
    if (prev.pref && (long long)prev.np > acap) acap = max(2 * acap, (long long)prev.np);
    const bool pref = n_r > acap;
    if (blockIdx.x == 0 && tid == 0) {
        BkRec &me = A.rec[r + 1];
        me.n_in = n_r;
        me.acap = acap;
        me.pref = pref ? 1 : 0;
    }
    __syncthreads();
    const unsigned delta = s_delta;
    const int nb = 1 << A.bits;
    const int G = A.group;
    if (G < 1 || G > GMAX) {
        if (tid == 0) atomicOr(&S->err, ERR_BOUNDS);
        return;
    }
    const int *CNT = A.cnt[cur];
    if (tid < G) {
        // pair p = blockIdx.x * G + tid: buckets (b0, b0 xor delta), or (2p, 2p + 1) when delta = 0
        const int p = blockIdx.x * G + tid;
        int b0, b1;
        if (delta == 0) {
            b0 = 2 * p;
            b1 = b0 + 1;
        } else {
            const int low = __ffs(delta) - 1;
            b0 = ((p >> low) << (low + 1)) | (p & ((1 << low) - 1));
            b1 = b0 ^ (int)delta;
        }
        int n0 = 0, n1 = 0;
        if (b0 >= nb || b1 >= nb) {
            s_bad = 1;
        } else {
            n0 = CNT[b0];
            n1 = CNT[b1];
            if (n0 < 0 || n1 < 0 || n0 > CAP || n1 > CAP) s_bad = 1;
        }
        s_b[2 * tid] = b0; s_b[2 * tid + 1] = b1;
        s_n[2 * tid] = s_bad ? 0 : n0; s_n[2 * tid + 1] = s_bad ? 0 : n1;
    }
    if (tid < NBK) s_out[tid] = 0;
    __syncthreads();
    if (s_bad) {
        if (tid == 0) atomicOr(&S->err, ERR_BOUNDS);
        return;
    }
    const u64 *Z = A.z[cur], *X = A.x[cur];
    const double *C = A.c[cur];
    u64 *OZ = A.z[cur ^ 1], *OX = A.x[cur ^ 1];
    double *OC = A.c[cur ^ 1];
    const DevParams &P = *A.P;
    const bool do_chan = (g.flags & GEN_CHANNEL) != 0 && P.chan_kind >= 0;
    const bool local_on = P.local_active != 0;
    const double cv = g.cosv, sv = g.sinv;
    const int flip = delta != 0 ? 1 : 0;
    auto skey = [&](int i) {
        Key<NW> kk;
#pragma unroll
        for (int w = 0; w < NW; ++w) { kk.z[w] = skz[w * SMI + i]; kk.x[w] = skx[w * SMI + i]; }
        return kk;
    };
    int cre = 0, alive = 0, kept = 0;
    bool over = false;
    // ---- sub-groups of consecutive pairs whose terms fit the staging area
    for (int j0 = 0; j0 < G;) {
        if (tid == 0) {
            int j = j0, tot = 0;
            while (j < G && tot + s_n[2 * j] + s_n[2 * j + 1] <= SMI) {
                s_off[2 * (j - j0)] = tot;
                tot += s_n[2 * j];
                s_off[2 * (j - j0) + 1] = tot;
                tot += s_n[2 * j + 1];
                ++j;
            }
            s_off[2 * (j - j0)] = tot;
            s_j1 = j;
        }
        __syncthreads();
        const int j1 = s_j1;
        const int nloc = 2 * (j1 - j0);            // buckets of this sub-group
        const int ntot = s_off[nloc];
        // stage: term i lies in local bucket lb with s_off[lb] <= i < s_off[lb + 1]
        for (int i = tid; i < ntot; i += T) {
            int lb = 0;
            while (lb + 1 < nloc && s_off[lb + 1] <= i) ++lb;
            const long long p = (long long)s_b[2 * j0 + lb] * CAP + (i - s_off[lb]);
            const Key<NW> kk = load_key<NW>(Z, X, p);
#pragma unroll
            for (int w = 0; w < NW; ++w) { skz[w * SMI + i] = kk.z[w]; skx[w * SMI + i] = kk.x[w]; }
            sc[i] = C[p];
            sbk[i] = (unsigned char)(2 * j0 + lb);
        }
        for (int s2 = tid; s2 < TAB; s2 += T) tab[s2] = 0u;
        __syncthreads();
        // index the keys; mark the terms the early merge drops
        for (int i = tid; i < ntot; i += T) {
            const Key<NW> kk = skey(i);
            unsigned h = bk_slot<NW, TAB>(kk);
            for (int probe = 0; probe < TAB; ++probe) {
                if (atomicCAS(&tab[h], 0u, (unsigned)(i + 1)) == 0u) break;
                h = (h + 1) & (TAB - 1);
            }
            sdead[i] = (pref && should_drop<NW>(P.strict, kk, fabs(sc[i]))) ? 1 : 0;
        }
        __syncthreads();
        auto find = [&](const Key<NW> &q) {
            unsigned h = bk_slot<NW, TAB>(q);
            for (int probe = 0; probe < TAB; ++probe) {
                const unsigned e = tab[h];
                if (e == 0u) return -1;
                const int j = (int)e - 1;
                if (key_eq<NW>(skey(j), q)) return j;
                h = (h + 1) & (TAB - 1);
            }
            return -1;
        };
        // each term: own output (in its bucket) and new sin-branch term (in the partner bucket)
        const int rounds = (ntot + T - 1) / T;
        for (int rd = 0; rd < rounds; ++rd) {
            const int i = rd * T + tid;
            const bool in = i < ntot && !sdead[i];
            bool own = false, nw_ = false;
            double oval = 0.0, nval = 0.0;
            int lb = 0;
            if (in) {
                ++alive;
                lb = sbk[i];
                const Key<NW> kk = skey(i);
                const double c = sc[i];
                double v = c;
                Key<NW> qk;
                double sg = 0.0;
                if (rotate_term<NW>(kk, g, &qk, &sg)) {
                    v = __dmul_rn(c, cv);
                    const double s = __dmul_rn(sg * sv, c);      // (k - 2) * sin(theta) * c, spv_kernels.jl:163
                    const bool s_ok = !(local_on && should_drop<NW>(P.local, qk, fabs(s)));
                    cre += s_ok ? 1 : 0;
                    const int j = find(qk);
                    if (j >= 0 && !sdead[j]) {
                        // the partner's sin branch lands on this key: live value first, then the append
                        const Key<NW> kj = skey(j);
                        Key<NW> back;
                        double sgj = 0.0;
                        rotate_term<NW>(kj, g, &back, &sgj);
                        const double t = __dmul_rn(sgj * sv, sc[j]);
                        if (!(local_on && should_drop<NW>(P.local, kk, fabs(t)))) v = __dadd_rn(v, t);
                    } else if (s_ok && !should_drop<NW>(P.strict, qk, fabs(s))) {
                        nval = do_chan ? __dmul_rn(s, channel_factor<NW>(P, qk)) : s;
                        nw_ = true;
                    }
                }
                if (!should_drop<NW>(P.strict, kk, fabs(v))) {
                    oval = do_chan ? __dmul_rn(v, channel_factor<NW>(P, kk)) : v;
                    own = true;
                }
            }
            kept += (own ? 1 : 0) + (nw_ ? 1 : 0);
            const int po = bk_claim(s_out, lb, own);
            if (own) {
                if (po < CAP) {
                    const long long o = (long long)s_b[lb] * CAP + po;
                    store_key<NW>(OZ, OX, o, skey(i));
                    OC[o] = oval;
                } else {
                    over = true;
                }
            }
            const int tb = lb ^ flip;
            const int pn = bk_claim(s_out, tb, nw_);
            if (nw_) {
                if (pn < CAP) {
                    const long long o = (long long)s_b[tb] * CAP + pn;
                    Key<NW> nk = skey(i);
#pragma unroll
                    for (int w = 0; w < NW; ++w) { nk.z[w] ^= g.gz[w]; nk.x[w] ^= g.gx[w]; }
                    store_key<NW>(OZ, OX, o, nk);
                    OC[o] = nval;
                } else {
                    over = true;
                }
            }
        }
        __syncthreads();      // the staging area and index are reused by the next sub-group
        j0 = j1;
    }
    // ---- counts and per-rotation totals
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        kept += __shfl_xor_sync(0xffffffffu, kept, d);
        cre += __shfl_xor_sync(0xffffffffu, cre, d);
        alive += __shfl_xor_sync(0xffffffffu, alive, d);
    }
    if (lane == 0) { s_red[0][warp] = kept; s_red[1][warp] = cre; s_red[2][warp] = alive; }
    if (over) atomicOr(&S->err, ERR_OVERFLOW);
    __syncthreads();
    int *OCNT = A.cnt[cur ^ 1];
    BkRec &me = A.rec[r + 1];
    if (tid < 2 * G) OCNT[s_b[tid]] = min(s_out[tid], CAP);
    if (tid == 0) {
        int kt = 0, ct = 0, at = 0, mx = 0;
        for (int w = 0; w < T / 32; ++w) { kt += s_red[0][w]; ct += s_red[1][w]; at += s_red[2][w]; }
        for (int b = 0; b < 2 * G; ++b) mx = max(mx, s_out[b]);
        atomicAdd(&me.n_out, (unsigned long long)kt);
        atomicAdd(&me.created, (unsigned long long)ct);
        if (pref) atomicAdd(&me.np, (unsigned long long)at);
        atomicMax(&me.maxcnt, mx);
        if (mx > CAP) {
            atomicOr(&S->err, ERR_OVERFLOW);
            atomicMin(&S->bk_fail, r);
        }
    }
}

// Start of a launched group of rotations: its first rotation and input set
// (and, at the start of a chunk, no failed rotation yet).
__global__ void k_bk_begin(DevState *S, long long rot0, int cur0, int reset_fail) {
    S->bk_rot0 = rot0;
    S->bk_cur0 = cur0;
    if (reset_fail) S->bk_fail = 0x7fffffffffffffffll;
}

// Scatter into a bucket layout of capacity cap (counts zeroed beforehand).
// Source: a dense array of n terms (scnt == nullptr) or a bucket layout of
// 2^sbits buckets.  The largest destination count is recorded in *maxcnt; a
// full bucket sets ERR_OVERFLOW in *err (the caller retries with more buckets).
template <int NW>
__global__ void k_bk_scatter(const u64 *SZ, const u64 *SX, const double *SC, long long n, const int *scnt, int sbits,
                             u64 *DZ, u64 *DX, double *DC, int *dcnt, int dbits, int cap, const u64 *rows,
                             int *maxcnt, int *err) {
    const long long slots = scnt ? ((long long)cap << sbits) : n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < slots;
         i += (long long)gridDim.x * blockDim.x) {
        if (scnt && (int)(i % cap) >= scnt[i / cap]) continue;
        const Key<NW> kk = load_key<NW>(SZ, SX, i);
        const unsigned b = bk_hash<NW>(kk.z, kk.x, rows, dbits);
        const int pos = atomicAdd(&dcnt[b], 1);
        if (pos >= cap) {
            atomicOr(err, ERR_OVERFLOW);
            continue;
        }
        const long long o = (long long)b * cap + pos;
        store_key<NW>(DZ, DX, o, kk);
        DC[o] = SC[i];
        atomicMax(maxcnt, pos + 1);
    }
}

// Exclusive scan of the bucket counts into dense offsets (one CTA), total in
// off[nb]; counts above cap are clipped (a flagged overflow leaves them so).
constexpr int BKS_THREADS = 1024;
__global__ void __launch_bounds__(BKS_THREADS) k_bk_offsets(const int *cnt, int nb, int cap, long long *off) {
    __shared__ long long sm[BKS_THREADS / 32 + 1];
    const int per = (nb + BKS_THREADS - 1) / BKS_THREADS;
    const int t0 = min((int)threadIdx.x * per, nb), t1 = min(t0 + per, nb);
    long long loc = 0;
    for (int b = t0; b < t1; ++b) loc += min(cnt[b], cap);
    long long total;
    long long run = block_excl_scan<BKS_THREADS>(loc, 0ll, OpSum(), sm, &total);
    for (int b = t0; b < t1; ++b) { off[b] = run; run += min(cnt[b], cap); }
    if (threadIdx.x == 0) off[nb] = total;
}

// Gather of a bucket layout into a dense array (one warp per bucket).
template <int NW>
__global__ void k_bk_gather(const u64 *SZ, const u64 *SX, const double *SC, const int *cnt, int nb, int cap,
                            const long long *off, u64 *DZ, u64 *DX, double *DC) {
    const int lane = threadIdx.x & 31;
    const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long b = w0; b < nb; b += nw) {
        const int m = min(cnt[b], cap);
        const long long o = off[b];
        for (int j = lane; j < m; j += 32) {
            const long long s = b * cap + j;
            store_key<NW>(DZ, DX, o + j, load_key<NW>(SZ, SX, s));
            DC[o + j] = SC[s];
        }
    }
}

}  // namespace pp
