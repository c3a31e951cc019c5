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
// b xor delta as well.  A CTA therefore works on whole bucket pairs
// {b, b xor delta} (two neighbouring buckets when delta = 0): it stages a group
// of pairs in shared memory, indexes their keys in a shared-memory hash table,
// finds each anticommuting term's partner there, and appends each output term
// to its bucket of the other bucket set (positions from shared-memory counters,
// so the order inside a bucket is arbitrary; nothing depends on it).  The grid
// is persistent and the next group's terms are copied in (cp.async) while a
// group is processed.  No cross-CTA scan, sort or wait is involved.
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
// one per device.  A CTA of BK_THREADS threads has two staging areas of
// BK_THREADS * ITEMS terms: one holds the group of bucket pairs being processed,
// the other receives the next group's terms in the meantime.
constexpr int BK_ROWS = 26;                    // hash rows: at most 2^26 buckets
constexpr int BK_THREADS = 256;
constexpr int BK_DEFAULT_CAP = 512;
constexpr int BK_DEFAULT_ITEMS = 4;
// Resident CTAs per SM the register budget aims at: four for one-word keys
// (64 registers), three for two-word keys (at 64 they spill and run 10 % slower);
// one for the 8-item variants, whose shared memory allows two at most.
__host__ __device__ constexpr int bk_min_blocks(int nw, int items) { return items >= 8 ? 1 : nw == 1 ? 4 : 3; }

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
    int bits_cap;                   // the bucket sets and counts are allocated for 2^bits_cap buckets
    long long rec_len;              // entries of rec
    const u64 *rows;                // [BK_ROWS][4]: z words 0..1, x words 0..1 of each hash row
    BkRec *rec;
    DevState *S;
    const DevParams *P;
    const GenRec *gens;
    // batched instances (the instance index is z word 1 of every key): angle
    // tables [instance][column] and the rotation each instance ends at
    const double *bcos, *bsin;
    const long long *bend;
    long long ninst;
    int ncol;
    // key-sharded runs: per bucket, foreign terms (received from the partner rank)
    // follow the local ones; remote: the sin branches of local terms belong to the
    // partner rank; pref_forced: the early-merge decision from the global counts
    // (-1: from the rotation record, as on one rank)
    int *fcnt[2];
    int remote;
    int pref_forced;
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

// Slot hash of the shared-memory key index: a 32-bit multiply-xor mix of all
// key words (the terms of a group share their bucket-hash parities, not these).
template <int NW, int TAB>
__device__ __forceinline__ unsigned bk_slot(const Key<NW> &k) {
    unsigned h = (unsigned)k.z[0] ^ ((unsigned)(k.z[0] >> 32) * 0x9E3779B1u);
    h = h * 0x85EBCA77u ^ (unsigned)k.x[0];
    h = h * 0xC2B2AE3Du ^ (unsigned)(k.x[0] >> 32);
    if constexpr (NW == 2) {
        h = h * 0x27D4EB2Fu ^ (unsigned)k.z[1];
        h = h * 0x165667B1u ^ (unsigned)(k.z[1] >> 32);
        h = h * 0x9E3779B1u ^ (unsigned)k.x[1];
        h = h * 0x85EBCA77u ^ (unsigned)(k.x[1] >> 32);
    }
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    return h & (TAB - 1);
}

// Shared memory of k_bk_rotate: two staging areas (keys, coefficients, local
// bucket of each term) and the key index (16-bit slots, twice the area's terms).
template <int NW, int CAP, int ITEMS>
__host__ __device__ constexpr size_t bk_smem_bytes() {
    return (size_t)(BK_THREADS * ITEMS) * (2 * (2 * NW * 8 + 8 + 1) + 2 * 2);
}
// Most bucket pairs a group may hold (at most 16, so that one warp handles a
// group's 32 buckets); the kernel picks the group size of each launch from the
// mean bucket load.
template <int CAP, int ITEMS>
__host__ __device__ constexpr int bk_group_max() {
    return 4 * BK_THREADS * ITEMS / CAP < 16 ? 4 * BK_THREADS * ITEMS / CAP : 16;
}

// 16-byte asynchronous copy global -> shared (both addresses 16-byte aligned).
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Lanes of the warp whose local bucket equals this lane's: the staged terms of a
// group lie in bucket order, so equal buckets form one run of consecutive lanes.
__device__ __forceinline__ unsigned bk_segment(int lb, int lane) {
    const int up = __shfl_up_sync(0xffffffffu, lb, 1);
    const unsigned head = __ballot_sync(0xffffffffu, lane == 0 || up != lb);
    const unsigned upto = 0xffffffffu >> (31 - lane);              // lanes 0 .. lane
    const unsigned above = head & ~upto;
    const int s0 = 31 - __clz(head & upto);
    return (above ? (1u << (__ffs(above) - 1)) - 1u : 0xffffffffu) & ~((1u << s0) - 1u);
}

// Position in output bucket ob for every lane that passes `want` (ob is the same
// across a segment): the segment's first wanting lane takes consecutive slots
// for all of them from one shared-memory atomic.  (Packing a pair's two counters
// into one 64-bit atomic for both claims of a round measured 5 % slower.)
__device__ __forceinline__ int bk_claim(int *s_out, int ob, bool want, unsigned seg, int lane) {
    const unsigned peers = __ballot_sync(0xffffffffu, want) & seg;
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (want && lane == leader) base = atomicAdd(&s_out[ob], __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader < 0 ? lane : leader);
    return want ? base + __popc(peers & ((1u << lane) - 1u)) : -1;
}

// The common criteria of a compiled filter in registers (coefficient
// threshold, weight and X-weight caps); a filter that also uses the Majorana
// weight, a damped threshold or the batched word mask is evaluated in full.
struct FQuick {
    double thresh;
    int wmax, xwmax, full;
};

__device__ __forceinline__ FQuick fquick(const DevFilter &f) {
    FQuick q;
    q.thresh = f.thresh;
    q.wmax = (int)min(f.wmax, 1ll << 30);
    q.xwmax = (int)min(f.xwmax, 1ll << 30);
    q.full = (f.use_mw || f.use_dw || f.use_dxw || f.wlow) ? 1 : 0;
    return q;
}

// should_drop (spv_kernels.jl:64-79) through FQuick.
template <int NW>
__device__ __forceinline__ bool drop_q(const FQuick &q, const DevFilter &f, const Key<NW> &k, double absc) {
    if (q.full) return should_drop<NW>(f, k, absc);
    if (absc <= q.thresh) return true;
    int wt = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) wt += __popcll(k.z[w] | k.x[w]);
    if (wt > q.wmax) return true;
    if (q.xwmax >= 64 * NW) return false;        // the X-weight cap cannot drop
    int xw = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) xw += __popcll(k.x[w]);
    return xw > q.xwmax;
}

// The generator's key words and popcount(gz & gx), copied to registers by a
// kernel whose loops also issue shared-memory atomics (after which a GenRec in
// shared memory would be read again).  anticommutes and rotate_anti take either.
template <int NW>
struct GenKey {
    u64 gz[NW], gx[NW];
    int ng;
};

// P anticommutes with G (the parity test of rotate_term).
template <int NW, class Gen>
__device__ __forceinline__ bool anticommutes(const Key<NW> &p, const Gen &g) {
    int m = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) m += __popcll(g.gx[w] & p.z[w]) + __popcll(g.gz[w] & p.x[w]);
    return (m & 1) != 0;
}

// rotate_term for a P already known to anticommute with G: the sin branch's key
// P xor M and its phase sign k - 2 (_rotate_range!, spv_kernels.jl:155-163),
// without the parity test.
template <int NW, class Gen>
__device__ __forceinline__ void rotate_anti(const Key<NW> &p, const Gen &g, Key<NW> *q, double *sgn) {
    int m1 = 0, nzp = 0, nzx = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        q->z[w] = g.gz[w] ^ p.z[w];
        q->x[w] = g.gx[w] ^ p.x[w];
        m1 += __popcll(g.gx[w] & p.z[w]);
        nzp += __popcll(q->z[w] & q->x[w]);
        nzx += __popcll(p.z[w] & p.x[w]);
    }
    *sgn = (double)(((nzp - g.ng - nzx + 2 * m1) & 3) - 2);
}

// Buckets of pair p: (b0, b0 xor delta), or (2p, 2p + 1) when delta = 0.
__device__ __forceinline__ void bk_pair(unsigned delta, long long p, int *b0, int *b1) {
    if (delta == 0) {
        *b0 = (int)(2 * p);
        *b1 = *b0 + 1;
    } else {
        const int low = __ffs(delta) - 1;
        *b0 = (int)(((p >> low) << (low + 1)) | (p & ((1ll << low) - 1)));
        *b1 = *b0 ^ (int)delta;
    }
}

// One window-1 rotation.  The grid is persistent: CTA c processes the groups
// c, c + gridDim.x, ... of G consecutive bucket pairs, and while it processes one
// group its copies of the next group's terms are in flight (cp.async into the
// other staging area).  G is the largest power of two up to GMAX whose expected
// terms stay within 3/4 of a staging area at the entering set's mean bucket load
// and that leaves every CTA a group.  A group whose terms exceed the staging
// area is processed in sub-groups of consecutive pairs, loaded in turn (a single
// pair always fits: 2 * CAP <= BK_THREADS * ITEMS).  Three block barriers per
// group: staged terms visible, key index built, outputs claimed.  k is the
// rotation's index within the launched graph (rotation S->bk_rot0 + k, input set
// (S->bk_cur0 + k) & 1).
//
// BATCH (two-word keys only): the live set holds many instances, instance i's
// terms carrying i in z word 1, which no generator changes, so a term's partner
// is in its own instance.  Each term rotates by its instance's angle column; a
// term whose instance has ended is kept as it is (no rotation, no filter, no
// channel) until it is harvested.
template <int NW, int CAP, int ITEMS, bool BATCH = false>
__global__ void __launch_bounds__(BK_THREADS, bk_min_blocks(NW, ITEMS)) k_bk_rotate(BkArgs A, int k) {
    constexpr int T = BK_THREADS;
    constexpr int SMI = T * ITEMS;                 // staged terms per area
    constexpr int TAB = 2 * SMI;                   // key index slots
    constexpr int GMAX = bk_group_max<CAP, ITEMS>();
    constexpr int NBK = 2 * GMAX;                  // buckets of a group
    static_assert(2 * CAP <= SMI, "a pair of full buckets fits");
    static_assert(NBK <= 32, "one warp handles a group's buckets");
    static_assert(SMI < 0x10000, "16-bit key index entries");
    static_assert(!BATCH || NW == 2, "batched instances use two-word keys");
    DevState *S = A.S;
    // Launched as a programmatic dependent of the previous rotation: the next
    // rotation's CTAs may start as this one's finish.  Everything before
    // griddepcontrol.wait reads only what no rotation writes (the cursor set
    // before the graph launch, the generator, the hash rows).
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    __shared__ int s_err;
    const long long r = S->bk_rot0 + k;
    if (r >= S->rot_end) return;
    const int cur = (S->bk_cur0 + k) & 1;
    __shared__ GenRec g;
    __shared__ unsigned s_delta;
    __shared__ int s_b[2][NBK], s_n[2][NBK], s_nl[2][NBK], s_off[2][NBK + 1], s_j1[2];
    __shared__ int s_out[NBK], s_mx, s_bad;
    __shared__ int s_red[3][T / 32];
    extern __shared__ __align__(128) u64 bsm[];
    // staging area a: keys (NW words each, z then x), coefficients; then the key
    // index and, per area, a byte per staged slot: its local bucket in bits 0-4,
    // bit 5 once the index pass has found that the term anticommutes with G, bit
    // 6 for a foreign term (key-sharded runs), bit 7 when the slot holds no term
    // (a run's padding slot) or one the early merge drops
    constexpr int AREA = (2 * NW + 1) * SMI;       // u64 words of one staging area
    auto skz = [&](int a) { return bsm + a * AREA; };
    auto skx = [&](int a) { return bsm + a * AREA + NW * SMI; };
    auto sc = [&](int a) { return reinterpret_cast<double *>(bsm + a * AREA + 2 * NW * SMI); };
    unsigned short *tab = reinterpret_cast<unsigned short *>(bsm + 2 * AREA);   // [TAB]
    unsigned char *sbk0 = reinterpret_cast<unsigned char *>(tab + TAB);        // [2][SMI]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        g = A.gens[r];
        s_delta = bk_hash<NW>(g.gz, g.gx, A.rows, A.bits);
        s_bad = 0;
        s_mx = 0;
    }
    if (r + 1 >= A.rec_len) {
        if (tid == 0) flag_bounds(S, 2, r);
        return;
    }
    {
        uint4 *t4 = reinterpret_cast<uint4 *>(tab);
        for (int i = tid; i < TAB / 8; i += T) t4[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    if (tid < NBK) s_out[tid] = 0;
    // the previous rotation's outputs (and error word) are visible from here on;
    // one read of the error word for the whole CTA (another CTA may set it meanwhile)
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (tid == 0) s_err = S->err;
    __syncthreads();
    if (s_err) return;
    // the state entering this rotation, from the previous rotation's record (the
    // early-merge rule of spv_evolve.jl:356-362)
    const BkRec &prev = A.rec[r];
    const long long n_r = (long long)prev.n_out;
    long long acap = prev.acap;
    if (prev.pref && (long long)prev.np > acap) acap = max(2 * acap, (long long)prev.np);
    const bool pref = A.pref_forced >= 0 ? A.pref_forced != 0 : n_r > acap;
    if (blockIdx.x == 0 && tid == 0) {
        BkRec &me = A.rec[r + 1];
        me.n_in = n_r;
        me.acap = acap;
        me.pref = pref ? 1 : 0;
    }
    const unsigned delta = s_delta;
    const long long nb = 1ll << A.bits;
    const long long pairs = nb / 2;
    int G = GMAX;
    while (G > 1 && (8ll * G * n_r > 3ll * SMI * nb || pairs / G < (long long)gridDim.x)) G >>= 1;
    const long long ngroups = pairs / G;
    if (A.bits > A.bits_cap || A.bits < 1 || pairs % G != 0) {
        if (tid == 0) flag_bounds(S, 1, ((long long)A.bits << 16) | G);
        return;
    }
    // (selected, not indexed: a runtime index into the parameter struct would copy it to the stack)
    const int *CNT = cur ? A.cnt[1] : A.cnt[0];
    int *OCNT = cur ? A.cnt[0] : A.cnt[1];
    const int *FCNT = A.fcnt[0] ? (cur ? A.fcnt[1] : A.fcnt[0]) : nullptr;
    int *OFCNT = A.fcnt[0] ? (cur ? A.fcnt[0] : A.fcnt[1]) : nullptr;
    const bool remote = A.remote != 0;
    const u64 *Z = cur ? A.z[1] : A.z[0], *X = cur ? A.x[1] : A.x[0];
    const double *C = cur ? A.c[1] : A.c[0];
    u64 *OZ = cur ? A.z[0] : A.z[1], *OX = cur ? A.x[0] : A.x[1];
    double *OC = cur ? A.c[0] : A.c[1];
    const DevParams &P = *A.P;
    const bool do_chan = (g.flags & GEN_CHANNEL) != 0 && P.chan_kind >= 0;
    const bool local_on = P.local_active != 0;
    const FQuick fs = fquick(P.strict);
    const double cv = g.cosv, sv = g.sinv;
    GenKey<NW> gk;                   // the generator in registers
#pragma unroll
    for (int w = 0; w < NW; ++w) { gk.gz[w] = g.gz[w]; gk.gx[w] = g.gx[w]; }
    gk.ng = g.ng;
    const int flip = delta != 0 ? 1 : 0;

    // pair buckets and counts of group gi into area a (threads < G); -1 group: none
    auto load_info = [&](int a, long long gi) {
        if (tid < G) {
            int b0 = 0, b1 = 0, n0 = 0, n1 = 0, f0 = 0, f1 = 0;
            if (gi >= 0) {
                bk_pair(delta, gi * G + tid, &b0, &b1);
                if (b0 < 0 || b1 < 0 || b0 >= nb || b1 >= nb) { flag_bounds(S, 3, b0); s_bad = 1; b0 = b1 = 0; }
                else {
                    n0 = CNT[b0];
                    n1 = CNT[b1];
                    if (FCNT) { f0 = FCNT[b0]; f1 = FCNT[b1]; }
                    if (n0 < 0 || n1 < 0 || f0 < 0 || f1 < 0 || n0 + f0 > CAP || n1 + f1 > CAP) {
                        flag_bounds(S, 4, ((long long)n0 << 20) | (n1 & 0xfffff));
                        s_bad = 1;
                        n0 = n1 = f0 = f1 = 0;
                    }
                }
            }
            s_b[a][2 * tid] = b0; s_b[a][2 * tid + 1] = b1;
            s_n[a][2 * tid] = n0 + f0; s_n[a][2 * tid + 1] = n1 + f1;
            s_nl[a][2 * tid] = n0; s_nl[a][2 * tid + 1] = n1;
        }
    };
    // first sub-group [j0, j1) of pairs from j0 that fits the staging area, and its
    // offsets: a prefix sum over the pairs in warp 0 (G <= 16 pairs, one per lane;
    // called by warp 0 only).  Each bucket's run is padded to an even length, so
    // every run starts 16-byte aligned for the bulk copies.  A single pair always
    // fits (counts are at most CAP, which is even).
    auto plan = [&](int a, int j0) {
        const int j = j0 + lane;
        int n0 = j < G ? s_n[a][2 * j] : 0, n1 = j < G ? s_n[a][2 * j + 1] : 0;
        n0 += n0 & 1;
        n1 += n1 & 1;
        int inc = n0 + n1;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= d) inc += y;
        }
        const int exc = inc - n0 - n1;
        const bool fits = j < G && (inc <= SMI || lane == 0);
        const int cnt = __popc(__ballot_sync(0xffffffffu, fits));       // fits is a prefix of the lanes
        if (fits) {
            s_off[a][2 * lane] = exc;
            s_off[a][2 * lane + 1] = exc + n0;
        }
        const int tot = __shfl_sync(0xffffffffu, inc, max(cnt, 1) - 1);
        if (lane == 0) {
            s_off[a][2 * cnt] = tot;
            s_j1[a] = j0 + cnt;
        }
    };
    // copies of the planned sub-group's terms into area a (asynchronous): warp w
    // copies buckets w, w + 8, ... with cp.async, two slots per lane and copy (16
    // bytes of keys or coefficients: every run starts at an even slot of an even
    // bucket offset), and writes each staged slot's local-bucket byte (bit 7 on a
    // run's padding slot, whose copy is the bucket's next, unused slot).  (Bulk
    // copies, one lane per run on an mbarrier, measured 2.5 % slower on config 2.)
    auto issue = [&](int a, int j0) {
        const int nloc = 2 * (s_j1[a] - j0);
        const int ntot = s_off[a][nloc];
        unsigned char *sbk = sbk0 + a * SMI;
        if (ntot > SMI || nloc > NBK) {      // the planner never builds such a sub-group
            if (tid == 0) flag_bounds(S, 5, ((long long)ntot << 16) | nloc);
            return;
        }
        for (int lb = warp; lb < nloc; lb += T / 32) {
            const int bq = s_b[a][2 * j0 + lb];
            const int o0 = s_off[a][lb], len = s_off[a][lb + 1] - o0, cnt = s_n[a][2 * j0 + lb];
            const int loc = s_nl[a][2 * j0 + lb];     // local terms first, then foreign ones
            if (bq < 0 || bq >= nb || len < 0 || len > CAP || (o0 & 1) || (len & 1)) {
                if (lane == 0) flag_bounds(S, 6, ((long long)bq << 20) | (len & 0xfffff));
                for (int t = lane; t < len; t += 32) sbk[o0 + t] = (unsigned char)(0x80 | lb);
                continue;
            }
            const long long p0 = (long long)bq * CAP;
            for (int t = 2 * lane; t < len; t += 64) {
                const int i = o0 + t;
                const long long p = p0 + t;
#pragma unroll
                for (int w = 0; w < NW; ++w) {
                    // slots t, t + 1 of key word plane w (NW = 1) or slot t's, then t + 1's words (NW = 2)
                    cp_async16(skz(a) + NW * i + 2 * w, Z + NW * p + 2 * w);
                    cp_async16(skx(a) + NW * i + 2 * w, X + NW * p + 2 * w);
                }
                cp_async16(sc(a) + i, C + p);
                sbk[i] = (unsigned char)(t < loc ? lb : t < cnt ? (0x40 | lb) : (0x80 | lb));
                sbk[i + 1] = (unsigned char)(t + 1 < loc ? lb : t + 1 < cnt ? (0x40 | lb) : (0x80 | lb));
            }
        }
        cp_async_commit();
    };
    auto staged = [&](int a) { cp_async_wait_all(); };   // this thread's copies of area a
    int cre = 0, alive = 0, kept = 0;
    bool over = false;
    auto skey = [&](int a, int i) {
        Key<NW> kk;
#pragma unroll
        for (int w = 0; w < NW; ++w) { kk.z[w] = skz(a)[NW * i + w]; kk.x[w] = skx(a)[NW * i + w]; }
        return kk;
    };
    // process the staged sub-group [j0, j1) of area a; leaves the index clear and
    // returns j1.  The plan of area a is read here, before the first barrier: once
    // the outputs are claimed (the last barrier) the area may be planned anew.
    auto run = [&](int a, int j0) {
        unsigned char *sbk = sbk0 + a * SMI;
        const int j1 = s_j1[a];
        const int ntot = s_off[a][2 * (j1 - j0)];
        if (ntot > SMI) {                    // uniform: skipped by every thread (flagged in issue)
            __syncthreads();
            return j1;
        }
        // mark the terms the early merge drops, and index the live terms that
        // anticommute with G: only they can be a partner (P xor G anticommutes
        // exactly when P does), and a dropped partner counts as absent
        for (int i = tid; i < ntot; i += T) {
            if (sbk[i] & 0x80) continue;     // a run's padding slot
            const Key<NW> kk = skey(a, i);
            if (pref && !(sbk[i] & 0x40) && drop_q<NW>(fs, P.strict, kk, fabs(sc(a)[i]))) {
                sbk[i] |= 0x80;
                continue;
            }
            if (!anticommutes<NW>(kk, gk)) continue;
            sbk[i] |= 0x20;                  // the rotation pass reads this instead of the parity
            unsigned h = bk_slot<NW, TAB>(kk);
            for (int probe = 0; probe < TAB; ++probe) {
                if (atomicCAS(&tab[h], (unsigned short)0, (unsigned short)(i + 1)) == (unsigned short)0) break;
                h = (h + 1) & (TAB - 1);
            }
        }
        __syncthreads();
        auto find = [&](const Key<NW> &q) {
            unsigned h = bk_slot<NW, TAB>(q);
            for (int probe = 0; probe < TAB; ++probe) {
                const int e = tab[h];
                if (e == 0) return -1;
                if (key_eq<NW>(skey(a, e - 1), q)) return e - 1;
                h = (h + 1) & (TAB - 1);
            }
            return -1;
        };
        const int rounds = (ntot + T - 1) / T;
        for (int rd = 0; rd < rounds; ++rd) {
            const int i = rd * T + tid;
            // local bucket (0x7f past the staged terms keeps buckets nondecreasing
            // across the warp) and early-merge drop flag
            const int tag = i < ntot ? sbk[i] : 0x7f;
            int lb = tag & 0x1f;
            const bool in = i < ntot && tag < 0x80;
            const bool fgn = (tag & 0x40) != 0;      // a foreign term: its sin branch only
            if (i < ntot && lb >= 2 * (j1 - j0)) {
                flag_bounds(S, 7, lb);
                lb = 0;
            }
            bool own = false, nw_ = false;
            double oval = 0.0, nval = 0.0;
            Key<NW> kk;                  // kept in registers for the stores (no reload after the claims)
            if (in) {
                alive += fgn ? 0 : 1;
                kk = skey(a, i);
                const double c = sc(a)[i];
                double v = c;
                Key<NW> qk;
                double sg = 0.0;
                double cvt = cv, svt = sv;
                bool act = true;                                 // the term's instance is running
                if constexpr (BATCH) {
                    const u64 t = kk.z[NW - 1];
                    if (t >= (u64)A.ninst) {
                        flag_bounds(S, 11, (long long)t);
                        act = false;
                    } else if (r >= A.bend[t]) {
                        act = false;
                    } else {
                        const long long ai = (long long)t * A.ncol + g.acol;
                        cvt = A.bcos[ai];
                        svt = A.bsin[ai];
                    }
                }
                if (act && (tag & 0x20)) {
                    rotate_anti<NW>(kk, gk, &qk, &sg);
                    v = __dmul_rn(c, cvt);
                    const double s = __dmul_rn(sg * svt, c);     // (k - 2) * sin(theta) * c, spv_kernels.jl:163
                    const bool s_ok = !(local_on && should_drop<NW>(P.local, qk, fabs(s)));
                    cre += (s_ok && !fgn) ? 1 : 0;
                    const int j = find(qk);
                    if (j >= ntot) flag_bounds(S, 8, j);
                    if (j >= 0 && j < ntot) {
                        // the partner's sin branch lands on this key: live value first, then
                        // the append.  Its phase factor is -sg: for Q = P xor G,
                        // k(P) + k(Q) = 2 (m1(P) + m1(Q) - ng) = 4 (m1(P) - popc(gx & gz & zP))
                        // (mod 4) in _rotate_range!'s k (spv_kernels.jl:162-163), and k is odd
                        const double t = __dmul_rn(-(sg * svt), sc(a)[j]);
                        if (!(local_on && should_drop<NW>(P.local, kk, fabs(t)))) v = __dadd_rn(v, t);
                    } else if (s_ok && (fgn || !remote) && !drop_q<NW>(fs, P.strict, qk, fabs(s))) {
                        // (a local term's sin branch belongs to the partner rank when remote)
                        nval = do_chan ? __dmul_rn(s, channel_factor<NW>(P, qk)) : s;
                        nw_ = true;
                    }
                }
                if (fgn) {
                    // a foreign term's own key belongs to the partner rank
                } else if (!act) {
                    oval = v;                                    // an ended instance is kept as it is
                    own = true;
                } else if (!drop_q<NW>(fs, P.strict, kk, fabs(v))) {
                    oval = do_chan ? __dmul_rn(v, channel_factor<NW>(P, kk)) : v;
                    own = true;
                }
            }
            kept += (own ? 1 : 0) + (nw_ ? 1 : 0);
            const unsigned seg = bk_segment(lb, lane);
            const int ob = 2 * j0 + lb;                      // group bucket of the own output
            const int po = bk_claim(s_out, ob, own, seg, lane);
            if (own) {
                if (po < CAP) {
                    const long long o = (long long)s_b[a][ob] * CAP + po;
                    store_key<NW>(OZ, OX, o, kk);
                    OC[o] = oval;
                } else {
                    over = true;
                }
            }
            const int tb = ob ^ flip;                        // the partner bucket of the pair
            const int pn = __any_sync(0xffffffffu, nw_) ? bk_claim(s_out, tb, nw_, seg, lane) : -1;   // new terms are rare
            if (nw_) {
                if (pn < CAP) {
                    const long long o = (long long)s_b[a][tb] * CAP + pn;
                    Key<NW> nk = kk;
#pragma unroll
                    for (int w = 0; w < NW; ++w) { nk.z[w] ^= gk.gz[w]; nk.x[w] ^= gk.gx[w]; }
                    store_key<NW>(OZ, OX, o, nk);
                    OC[o] = nval;
                } else {
                    over = true;
                }
            }
        }
        __syncthreads();
        uint4 *t4 = reinterpret_cast<uint4 *>(tab);                      // for the next sub-group
        for (int q = tid; q < TAB / 8; q += T) t4[q] = make_uint4(0u, 0u, 0u, 0u);
        return j1;
    };

    // ---- prologue: group c staged into area 0 (copies in flight), group c + grid planned in area 1
    long long gi = blockIdx.x;
    load_info(0, gi < ngroups ? gi : -1);
    load_info(1, gi + gridDim.x < ngroups ? gi + gridDim.x : -1);
    __syncthreads();
    if (warp == 0) {
        plan(0, 0);
        plan(1, 0);
    }
    __syncthreads();
    if (gi < ngroups) issue(0, 0);
    for (int it = 0; gi < ngroups; ++it, gi += gridDim.x) {
        const int a = it & 1;
        const long long gnext = gi + gridDim.x, gafter = gi + 2 * (long long)gridDim.x;
        // the group after next: its pair counts load while this group is processed
        int pb0 = 0, pb1 = 0, pn0 = 0, pn1 = 0, pf0 = 0, pf1 = 0;
        if (tid < G && gafter < ngroups) {
            bk_pair(delta, gafter * G + tid, &pb0, &pb1);
            if (pb0 < nb && pb1 < nb) {
                pn0 = CNT[pb0];
                pn1 = CNT[pb1];
                if (FCNT) { pf0 = FCNT[pb0]; pf1 = FCNT[pb1]; }
            }
        }
        staged(a);
        __syncthreads();
        // the next group's copies (planned last iteration) go in flight now
        if (gnext < ngroups) issue(a ^ 1, 0);
        // this group: its first sub-group is staged in area a, later ones are loaded in turn
        int j0 = 0;
        for (;;) {
            j0 = run(a, j0);
            if (j0 >= G) break;
            if (warp == 0) plan(a, j0);
            __syncthreads();
            issue(a, j0);
            staged(a);
            __syncthreads();
        }
        // output counts of the group's buckets, then area a takes the group after
        // next and is planned (warp 0 alone: 2 * G <= 32); the next iteration's
        // first barrier publishes both
        if (warp == 0) {
            if (lane < 2 * G) {
                const int m = s_out[lane];
                OCNT[s_b[a][lane]] = min(m, CAP);
                if (OFCNT) OFCNT[s_b[a][lane]] = 0;
                atomicMax(&s_mx, m);
                s_out[lane] = 0;
            }
            __syncwarp();
            if (lane < G) {
                if (gafter < ngroups) {
                    if (pb0 >= nb || pb1 >= nb || pn0 < 0 || pn1 < 0 || pf0 < 0 || pf1 < 0 || pn0 + pf0 > CAP ||
                        pn1 + pf1 > CAP) {
                        flag_bounds(S, 10, ((long long)pn0 << 20) | (pn1 & 0xfffff));
                        s_bad = 1;
                        pb0 = pb1 = pn0 = pn1 = pf0 = pf1 = 0;
                    }
                }
                s_b[a][2 * lane] = pb0; s_b[a][2 * lane + 1] = pb1;
                s_n[a][2 * lane] = pn0 + pf0; s_n[a][2 * lane + 1] = pn1 + pf1;
                s_nl[a][2 * lane] = pn0; s_nl[a][2 * lane + 1] = pn1;
            }
            __syncwarp();
            plan(a, 0);
        }
    }
    // ---- per-rotation totals
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        kept += __shfl_xor_sync(0xffffffffu, kept, d);
        cre += __shfl_xor_sync(0xffffffffu, cre, d);
        alive += __shfl_xor_sync(0xffffffffu, alive, d);
    }
    if (lane == 0) { s_red[0][warp] = kept; s_red[1][warp] = cre; s_red[2][warp] = alive; }
    if (over) atomicOr(&S->err, ERR_OVERFLOW);
    __syncthreads();
    if (tid == 0) {
        BkRec &me = A.rec[r + 1];
        int kt = 0, ct = 0, at = 0;
        for (int w = 0; w < T / 32; ++w) { kt += s_red[0][w]; ct += s_red[1][w]; at += s_red[2][w]; }
        atomicAdd(&me.n_out, (unsigned long long)kt);
        atomicAdd(&me.created, (unsigned long long)ct);
        if (pref) atomicAdd(&me.np, (unsigned long long)at);
        atomicMax(&me.maxcnt, s_mx);
        if (s_mx > CAP) {
            atomicOr(&S->err, ERR_OVERFLOW);
            atomicMin(&S->bk_fail, r);
        }
        if (s_bad) atomicOr(&S->err, ERR_BOUNDS);
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
        if (b >= (1u << dbits)) {
            atomicOr(err, ERR_BOUNDS);
            continue;
        }
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
                            const long long *off, u64 *DZ, u64 *DX, double *DC, long long dcap, DevState *S) {
    const int lane = threadIdx.x & 31;
    const long long w0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long b = w0; b < nb; b += nw) {
        const int m = min(cnt[b], cap);
        const long long o = off[b];
        if (o < 0 || o + m > dcap) {
            if (lane == 0) flag_bounds(S, 9, o);
            continue;
        }
        for (int j = lane; j < m; j += 32) {
            const long long s = b * cap + j;
            store_key<NW>(DZ, DX, o + j, load_key<NW>(SZ, SX, s));
            DC[o + j] = SC[s];
        }
    }
}

// Owner rank of a key in a key-sharded run over 2^rank_bits ranks: bit k is the
// parity of P & R_(BK_ROWS - 1 - k), rows the bucket hash of a layout with at most
// BK_ROWS - rank_bits row bits never uses.  Linear like the bucket hash, so the
// sin branch P xor M of a term owned by r is owned by r xor owner(M).
template <int NW>
__host__ __device__ __forceinline__ unsigned bk_owner(const u64 *kz, const u64 *kx, const u64 *rows, int rank_bits) {
    unsigned o = 0;
    for (int k = 0; k < rank_bits; ++k) {
        const u64 *R = rows + 4 * (BK_ROWS - 1 - k);
        int p = 0;
        for (int w = 0; w < NW; ++w) p += popc64(kz[w] & R[w]) + popc64(kx[w] & R[2 + w]);   // NW: 1 or 2
        o |= (unsigned)(p & 1) << k;
    }
    return o;
}

// Key-sharded runs: the local terms of bucket set (Z, X, C, CNT) that anticommute
// with the generator and survive the early-merge pre-filter (when pref) -- the
// terms whose sin branches belong to the partner rank -- packed into (OZ, OX, OC)
// in any order; their number in *nout.  More than cap of them: ERR_OVERFLOW.
template <int NW>
__global__ void k_bk_send(const u64 *Z, const u64 *X, const double *C, const int *CNT, int bits, int cap,
                          const GenRec *gen, int pref, const DevParams *P, u64 *OZ, u64 *OX, double *OC, long long ocap,
                          unsigned long long *nout, DevState *S) {
    const long long slots = (long long)cap << bits;
    const FQuick fs = fquick(P->strict);
    const int lane = threadIdx.x & 31;
    for (long long base = (long long)blockIdx.x * blockDim.x; base < slots; base += (long long)gridDim.x * blockDim.x) {
        const long long i = base + threadIdx.x;
        bool send = false;
        Key<NW> kk;
        if (i < slots && (int)(i % cap) < CNT[i / cap]) {
            kk = load_key<NW>(Z, X, i);
            send = anticommutes<NW>(kk, *gen) && !(pref && drop_q<NW>(fs, P->strict, kk, fabs(C[i])));
        }
        const unsigned m = __ballot_sync(0xffffffffu, send);
        if (!m) continue;
        const int leader = __ffs(m) - 1;
        unsigned long long b0 = 0;
        if (lane == leader) b0 = atomicAdd(nout, (unsigned long long)__popc(m));
        b0 = __shfl_sync(0xffffffffu, b0, leader);
        if (send) {
            const long long o = (long long)b0 + __popc(m & ((1u << lane) - 1u));
            if (o < ocap) {
                store_key<NW>(OZ, OX, o, kk);
                OC[o] = C[i];
            } else {
                atomicOr(&S->err, ERR_OVERFLOW);
            }
        }
    }
}

// Key-sharded runs: n received terms appended to their buckets of the set
// (Z, X, C) as foreign terms, after the CNT[b] local ones (FCNT[b] counts them).
// A bucket that would exceed cap: ERR_OVERFLOW, the term is not written.
template <int NW>
__global__ void k_bk_absorb(const u64 *RZ, const u64 *RX, const double *RC, long long n, u64 *Z, u64 *X, double *C,
                            const int *CNT, int *FCNT, int bits, int cap, const u64 *rows, DevState *S) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const Key<NW> kk = load_key<NW>(RZ, RX, i);
        const unsigned b = bk_hash<NW>(kk.z, kk.x, rows, bits);
        const int pos = CNT[b] + atomicAdd(&FCNT[b], 1);
        if (pos >= cap) {
            atomicOr(&S->err, ERR_OVERFLOW);
            continue;
        }
        const long long o = (long long)b * cap + pos;
        store_key<NW>(Z, X, o, kk);
        C[o] = RC[i];
    }
}

}  // namespace pp
