// Shared device-side definitions for the SparsePauliVector propagation engine.
//
// Term storage is structure-of-arrays in HBM, byte-identical to the reference's
// Vector{UInt64} / Vector{UInt128} fields (src/type_SparsePauliVector.jl:69-84):
// z[i], x[i] are NW little-endian 64-bit words (NW = 1 for N <= 64, 2 for
// N <= 128, _word_type at type_SparsePauliVector.jl:23-26), c[i] is Float64.
// The sort key is (z, x) z-major, unsigned (_key_lt, spv_kernels.jl:14-16); as
// a single 2*64*NW-bit integer its bit "level" L is
//   L = 64*NW + 64*w + t   for bit t of z word w,
//   L =         64*w + t   for bit t of x word w.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace pp {

typedef unsigned long long u64;

constexpr int KMAX = 16;          // mask levels handled by the structured (permutation) path
constexpr int TAU_MAX = 2 * KMAX; // scan thresholds per rotation (h >= b and h >= b+1 per level)
constexpr int H_INF = 1000;       // "group boundary above every level" (first element)

// Error bits in DevState::err.
constexpr int ERR_OVERFLOW = 1;      // output would exceed the physical capacity: resume after growth
constexpr int ERR_TIMEOUT = 2;       // a bounded look-back wait gave up
constexpr int ERR_TILE = 4;          // a merge tile exceeded its shared-memory staging size
constexpr int ERR_CHECK = 8;         // check kernel found unsorted / duplicate keys
constexpr int ERR_BOUNDS = 16;       // a computed index fell outside its buffer (access skipped)

// Compiled truncation predicate (the reference's MergeFilter, spv_kernels.jl:33-42)
// with the damped-filter exponentials precomputed on the host by libm exp, so that
// should_drop agrees bit for bit with absc * exp(-alpha * w) <= dthresh.
struct DevFilter {
    long long wmax, xwmax, mwmax;
    double thresh, dthresh_w, dthresh_xw;
    int use_mw, use_dw, use_dxw;
    int coeff_based;              // 1 if any criterion reads |c|
    int wlow;                     // 1: weights count z/x word 0 only (batched instances keep a tag in z word 1)
    double expw[130];             // exp(-alpha_w * w),  w = popcount(z|x) in 0..128
    double expxw[130];            // exp(-alpha_xw * w), w = popcount(x)   in 0..128
};

// Per-call parameters living in device memory.
struct DevParams {
    DevFilter strict, local, clip;
    int local_active;             // local filter can drop appends
    int corr_kind;                // 0 none, 1 EnergyCorrection
    u64 ket[2];                   // EnergyCorrection / measurement ket
    int chan_kind;                // -1 none, 0 depolarizing, 1 dephasing, 2 bit_flip, 3 bit_phase_flip, 4 pauli
    u64 chan_mask[2];
    double chanX[130], chanY[130], chanZ[130];  // lambda^k tables (host-computed)
};

// One rotation exp(iθ/2 G): packed generator and host-computed cos/sin
// (spv_evolve.jl:333-343), plus the structured-sort metadata.
struct GenRec {
    u64 gz[2], gx[2];
    double cosv, sinv;
    int ng;                       // popcount(gz & gx)
    int k;                        // number of mask levels
    int flags;                    // GEN_MEASURE | GEN_CHANNEL
    int acol;                     // batched instances: column of this rotation's angle in the instance table
    short level[KMAX];            // mask levels, strictly descending
};
constexpr int GEN_MEASURE = 1;    // reduce <ket|O|ket> partials after this rotation
constexpr int GEN_CHANNEL = 2;    // apply the channel in this rotation's merge epilogue
constexpr int GEN_HARVEST = 4;    // compaction (MODE 2) also drops batched instances that have finished

struct DevState {
    long long n;                  // live terms
    long long a;                  // appends of the current rotation (structured path)
    long long an;                 // pending appends (general path)
    long long acap_logical;       // the reference's append capacity (early-merge rule)
    long long need;               // requested capacity on ERR_OVERFLOW
    long long rot, rot_end;       // rotation cursor within the current call
    long long created, merge_in, merge_out, early;  // WindowCounters totals
    long long npref;              // survivors of the window-1 early-merge pre-filter
    long long live_in;            // sum of live counts entering rotations
    long long peak;               // largest live count after a merge
    long long nseg;               // segments of the live set's segment table
    double expect_val;            // last reduced <ket|O|ket> (after the merge)
    double corr_energy;           // EnergyCorrection.accumulated_energy (delta this call)
    int cur;                      // live buffer set (0/1)
    int err;
    unsigned epoch;               // look-back epoch (30 bits used)
    int b_tile_ctr, b_done;       // merge kernel tile dispenser / completion
    int g_tile_ctr, g_done;       // general rotate kernel
    int measure_valid;
    int seg_dense;                // 0: live set cur is the last window-1 merge's per-tile slots (segment table)
    int pad;
    long long bk_rot0;            // bucketed rotations: first rotation of the launched group
    long long bk_fail;            // bucketed rotations: first rotation whose output overflowed a bucket
    int bk_cur0;                  // bucketed rotations: input bucket set of the group's first rotation
    int bk_pad;
    unsigned long long dbg;       // first failed device check: site << 40 | value (0: none)
};

// Records a failed device-side check (the access it guards is skipped): the
// error bit ERR_BOUNDS and, for the first failure only, which check and value.
__device__ __forceinline__ void flag_bounds(DevState *S, int site, long long value) {
    atomicOr(&S->err, ERR_BOUNDS);
    atomicCAS(&S->dbg, 0ull, ((unsigned long long)site << 40) | ((unsigned long long)value & 0xffffffffffull));
}

// Static per-kernel configuration.
constexpr int A_THREADS = 512;
constexpr int A_ITEMS = 5;
constexpr int A_TILE = A_THREADS * A_ITEMS;   // 2560 terms per classify/permute tile
constexpr int B_THREADS = 512;
constexpr int B_D = 2048;                     // merge-path diagonal step (outputs per tile)
constexpr int B_IPTMAX = 5;                   // per-thread outputs at most
constexpr int B_CAP = B_THREADS * B_IPTMAX;   // 2560: a tile plus an equal-key run past its diagonal
constexpr int SEG = B_CAP;                    // slot of one window-1 merge tile's output; dense segment size
static_assert(A_TILE >= SEG, "a classify tile holds one live segment");
constexpr int G_THREADS = 256;
constexpr int G_ITEMS = 8;
constexpr int G_TILE = G_THREADS * G_ITEMS;   // general rotate tile
constexpr int SPIN_LIMIT = 1 << 22;           // bounded look-back waits

// Population count usable in host and device code.
__host__ __device__ __forceinline__ int popc64(u64 v) {
#ifdef __CUDA_ARCH__
    return __popcll(v);
#else
    return __builtin_popcountll(v);
#endif
}

// mbarrier in shared memory (addresses are shared-window addresses).
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(mbar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase of the given parity; false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (int i = 0; i < SPIN_LIMIT; ++i)
        if (mbar_try(mbar, parity)) return true;
    return false;
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.expect_tx.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// One bulk copy global -> this CTA's shared memory, completing bytes on mbar
// (addresses 16-byte aligned, bytes a multiple of 16; this GPU's own memory).
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}


// Tile aggregate of the classify pass.
struct TileAggA {
    int count;
    int pad;
    u64 first[4], last[4];        // z words then x words of the first/last emitted key
    short firstpos[TAU_MAX];      // first local j >= 1 with h(j) >= tau (0x7fff: none)
    short lastpos[TAU_MAX];       // last local j >= 1 with h(j) >= tau (-1: none)
};

template <int NW>
struct Key {
    u64 z[NW], x[NW];
};

template <int NW>
__device__ __forceinline__ Key<NW> load_key(const u64 *__restrict__ Z, const u64 *__restrict__ X, long long i) {
    Key<NW> k;
    if constexpr (NW == 1) {
        k.z[0] = __ldg(Z + i);
        k.x[0] = __ldg(X + i);
    } else {
        ulonglong2 a = __ldg(reinterpret_cast<const ulonglong2 *>(Z) + i);
        ulonglong2 b = __ldg(reinterpret_cast<const ulonglong2 *>(X) + i);
        k.z[0] = a.x; k.z[1] = a.y; k.x[0] = b.x; k.x[1] = b.y;
    }
    return k;
}

template <int NW>
__device__ __forceinline__ void store_key(u64 *Z, u64 *X, long long i, const Key<NW> &k) {
    if constexpr (NW == 1) {
        Z[i] = k.z[0];
        X[i] = k.x[0];
    } else {
        reinterpret_cast<ulonglong2 *>(Z)[i] = make_ulonglong2(k.z[0], k.z[1]);
        reinterpret_cast<ulonglong2 *>(X)[i] = make_ulonglong2(k.x[0], k.x[1]);
    }
}

template <int NW>
__device__ __forceinline__ bool key_lt(const Key<NW> &a, const Key<NW> &b) {
#pragma unroll
    for (int w = NW - 1; w >= 0; --w)
        if (a.z[w] != b.z[w]) return a.z[w] < b.z[w];
#pragma unroll
    for (int w = NW - 1; w >= 0; --w)
        if (a.x[w] != b.x[w]) return a.x[w] < b.x[w];
    return false;
}

template <int NW>
__device__ __forceinline__ bool key_eq(const Key<NW> &a, const Key<NW> &b) {
    bool e = true;
#pragma unroll
    for (int w = 0; w < NW; ++w) e = e && (a.z[w] == b.z[w]) && (a.x[w] == b.x[w]);
    return e;
}

// Highest differing bit level between two keys (-1 if equal).
template <int NW>
__device__ __forceinline__ int hdiff(const Key<NW> &a, const Key<NW> &b) {
#pragma unroll
    for (int w = NW - 1; w >= 0; --w) {
        u64 d = a.z[w] ^ b.z[w];
        if (d) return 64 * NW + 64 * w + 63 - __clzll(d);
    }
#pragma unroll
    for (int w = NW - 1; w >= 0; --w) {
        u64 d = a.x[w] ^ b.x[w];
        if (d) return 64 * w + 63 - __clzll(d);
    }
    return -1;
}

template <int NW>
__device__ __forceinline__ int key_bit(const Key<NW> &a, int level) {
    if (level >= 64 * NW) {
        int l = level - 64 * NW;
        return (int)((a.z[l >> 6] >> (l & 63)) & 1ull);
    }
    return (int)((a.x[level >> 6] >> (level & 63)) & 1ull);
}

__device__ __forceinline__ int popc1(u64 v) { return __popcll(v); }

template <int NW>
__device__ __forceinline__ int popc_w(const u64 *v) {
    int s = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) s += __popcll(v[w]);
    return s;
}

// _majorana_weight_bits (spv_kernels.jl:51-62) over the full word width.
template <int NW>
__device__ __forceinline__ long long majorana(const Key<NW> &k) {
    if constexpr (NW == 1) {
        u64 z = k.z[0], x = k.x[0];
        u64 zonly = z & ~x, S = x;
#pragma unroll
        for (int s = 1; s < 64; s <<= 1) S ^= S >> s;
        u64 ctrl = ~(S ^ x);
        return (long long)__popcll(x) + 2ll * __popcll(zonly & ctrl) + 2ll * __popcll(~(z | x) & ~ctrl);
    } else {
        unsigned __int128 z = ((unsigned __int128)k.z[1] << 64) | k.z[0];
        unsigned __int128 x = ((unsigned __int128)k.x[1] << 64) | k.x[0];
        unsigned __int128 zonly = z & ~x, S = x;
#pragma unroll
        for (int s = 1; s < 128; s <<= 1) S ^= S >> s;
        unsigned __int128 ctrl = ~(S ^ x);
        auto pc = [](unsigned __int128 v) { return __popcll((u64)v) + __popcll((u64)(v >> 64)); };
        return (long long)pc(x) + 2ll * pc(zonly & ctrl) + 2ll * pc(~(z | x) & ~ctrl);
    }
}

// Majorana weight of the term; with wlow (batched instances) over word 0 alone,
// which is the 64-bit word an instance of N <= 64 qubits has on its own.
template <int NW>
__device__ __forceinline__ long long majorana_f(const Key<NW> &k, int wlow) {
    if constexpr (NW == 2) {
        if (wlow) {
            Key<1> k1;
            k1.z[0] = k.z[0];
            k1.x[0] = k.x[0];
            return majorana<1>(k1);
        }
    }
    return majorana<NW>(k);
}

// should_drop (spv_kernels.jl:64-79).
template <int NW>
__device__ __forceinline__ bool should_drop(const DevFilter &f, const Key<NW> &k, double absc) {
    if (absc <= f.thresh) return true;
    u64 o[NW], xx[NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) { o[w] = k.z[w] | k.x[w]; xx[w] = k.x[w]; }
    if constexpr (NW == 2) {
        if (f.wlow) { o[1] = 0; xx[1] = 0; }
    }
    int wt = popc_w<NW>(o);
    if (wt > f.wmax) return true;
    int xw = popc_w<NW>(xx);
    if (xw > f.xwmax) return true;
    if (f.use_mw && majorana_f<NW>(k, f.wlow) > f.mwmax) return true;
    if (f.use_dw && __dmul_rn(absc, f.expw[wt]) <= f.dthresh_w) return true;
    if (f.use_dxw && __dmul_rn(absc, f.expxw[xw]) <= f.dthresh_xw) return true;
    return false;
}

// Rotation of one term (the per-term body of _rotate_range!, spv_kernels.jl:155-164).
// Returns true if P anticommutes with G; then *q = P xor G and *sgn = +-1 is the
// factor (k - 2) of the sin branch.
template <int NW>
__device__ __forceinline__ bool rotate_term(const Key<NW> &p, const GenRec &g, Key<NW> *q, double *sgn) {
    int m1 = 0, m2 = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        m1 += __popcll(g.gx[w] & p.z[w]);
        m2 += __popcll(g.gz[w] & p.x[w]);
    }
    if (((m1 - m2) & 1) == 0) return false;
    int nzp = 0, nzx = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        q->z[w] = g.gz[w] ^ p.z[w];
        q->x[w] = g.gx[w] ^ p.x[w];
        nzp += __popcll(q->z[w] & q->x[w]);
        nzx += __popcll(p.z[w] & p.x[w]);
    }
    int k = (nzp - g.ng - nzx + 2 * m1) & 3;
    *sgn = (double)(k - 2);
    return true;
}

// Channel factor lambda^k for one term (channels.jl:203-265); tables from the host.
template <int NW>
__device__ __forceinline__ double channel_factor(const DevParams &P, const Key<NW> &k) {
    int kind = P.chan_kind;
    if (kind == 4) {
        int nX = 0, nY = 0, nZ = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            u64 xM = k.x[w] & P.chan_mask[w], zM = k.z[w] & P.chan_mask[w];
            nX += __popcll(xM & ~k.z[w]);
            nY += __popcll(xM & k.z[w]);
            nZ += __popcll(zM & ~k.x[w]);
        }
        return __dmul_rn(__dmul_rn(P.chanX[nX], P.chanY[nY]), P.chanZ[nZ]);
    }
    int cnt = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) {
        u64 s = kind == 0 ? (k.z[w] | k.x[w]) : kind == 1 ? k.x[w] : kind == 2 ? k.z[w] : (k.x[w] ^ k.z[w]);
        cnt += __popcll(s & P.chan_mask[w]);
    }
    return P.chanX[cnt];
}

// (-1)^popcount(z & ket) for a diagonal term (expectation_value, expectation_value.jl:8-11).
template <int NW>
__device__ __forceinline__ double ket_sign(const Key<NW> &k, const u64 *ket) {
    int s = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) s += __popcll(k.z[w] & ket[w]);
    return (s & 1) ? -1.0 : 1.0;
}

template <int NW>
__device__ __forceinline__ bool is_diag(const Key<NW> &k) {
    u64 o = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) o |= k.x[w];
    return o == 0;
}

// Neumaier compensated accumulation.
struct Neu {
    double s, c;
    __device__ __forceinline__ void add(double t) {
        double u = __dadd_rn(s, t);
        if (fabs(s) >= fabs(t)) c = __dadd_rn(c, __dadd_rn(__dsub_rn(s, u), t));
        else c = __dadd_rn(c, __dadd_rn(__dsub_rn(t, u), s));
        s = u;
    }
};

}  // namespace pp
