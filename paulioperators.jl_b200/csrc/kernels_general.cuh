// General-path kernels: windowed rotation with pending appends (window > 1,
// or generators with more than KMAX mask levels), the stable LSD radix sort of
// appended terms, and the stand-alone channel / expectation / invariant kernels.
#pragma once
#include "kernels_struct.cuh"

namespace pp {

// ------------------------------------------------------------ general rotate
// _rotate_spv! (spv_evolve.jl:207-218) over live [0, n) then pending appends
// [0, an): cos branch scaled in place, sin branches appended at an + rank in
// sweep order (order-preserving compaction with decoupled look-back, so the
// append order is the reference's).  Capacity 2*an + n is guaranteed by the host.
template <int NW>
__global__ void __launch_bounds__(G_THREADS) k_rotate_general(Bufs B, GenRec g) {
    DevState *S = B.S;
    if (S->err) return;
    __shared__ int s_tile;
    __shared__ int wtot[G_ITEMS * (G_THREADS / 32)];
    __shared__ int s_total;
    __shared__ unsigned s_base;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const DevParams &P = *B.P;
    const long long n = S->n, an = S->an, tot = n + an;
    const int cur = S->cur;
    u64 *Z = B.z[cur], *X = B.x[cur];
    double *C = B.c[cur];
    const int ntiles = (int)max(1ll, (tot + G_TILE - 1) / G_TILE);
    const unsigned epoch = S->epoch;
    const bool local_on = P.local_active != 0;
    while (true) {
        if (tid == 0) s_tile = atomicAdd(&S->g_tile_ctr, 1);
        __syncthreads();
        const int t = s_tile;
        if (t >= ntiles) break;
        const long long base = (long long)t * G_TILE;
        bool emit[G_ITEMS];
        Key<NW> q[G_ITEMS];
        double cn[G_ITEMS];
#pragma unroll
        for (int it = 0; it < G_ITEMS; ++it) {
            const long long e = base + it * G_THREADS + tid;
            emit[it] = false;
            if (e < tot) {
                const bool live = e < n;
                const long long i = live ? e : e - n;
                u64 *ZZ = live ? Z : B.az;
                u64 *XX = live ? X : B.ax;
                double *CC = live ? C : B.ac;
                const Key<NW> k = load_key<NW>(ZZ, XX, i);
                double sg;
                if (rotate_term<NW>(k, g, &q[it], &sg)) {
                    const double c = CC[i];
                    cn[it] = __dmul_rn(sg * g.sinv, c);
                    CC[i] = __dmul_rn(c, g.cosv);
                    emit[it] = !(local_on && should_drop<NW>(P.local, q[it], fabs(cn[it])));
                }
            }
        }
        int lpre[G_ITEMS];
#pragma unroll
        for (int it = 0; it < G_ITEMS; ++it) {
            unsigned m = __ballot_sync(0xffffffffu, emit[it]);
            lpre[it] = __popc(m & lanemask_lt());
            if (lane == 0) wtot[it * (G_THREADS / 32) + warp] = __popc(m);
        }
        __syncthreads();
        if (warp == 0) {
            constexpr int NE = G_ITEMS * (G_THREADS / 32);  // 64 entries, 2 per lane
            int v[NE / 32];
            int s = 0;
#pragma unroll
            for (int k = 0; k < NE / 32; ++k) { v[k] = wtot[lane * (NE / 32) + k]; s += v[k]; }
            int incl = warp_incl_scan(s, OpSum());
            int ex = incl - s;
#pragma unroll
            for (int k = 0; k < NE / 32; ++k) { wtot[lane * (NE / 32) + k] = ex; ex += v[k]; }
            if (lane == 31) s_total = incl;
        }
        __syncthreads();
        if (warp == 0) {
            const unsigned ex = lookback_warp(B.gstat, t, epoch, (unsigned)s_total, &S->err);
            if (lane == 0) s_base = ex;
        }
        __syncthreads();
        const long long obase = an + (long long)s_base;
#pragma unroll
        for (int it = 0; it < G_ITEMS; ++it) {
            if (emit[it]) {
                const long long o = obase + wtot[it * (G_THREADS / 32) + warp] + lpre[it];
                if (o < B.acap) {
                    store_key<NW>(B.az, B.ax, o, q[it]);
                    B.ac[o] = cn[it];
                } else {
                    atomicOr(&S->err, ERR_BOUNDS);
                }
            }
        }
        __syncthreads();
    }
}

// Commit of k_rotate_general: an += created (one thread, after the launch).
__global__ void k_rotate_commit(Bufs B) {
    DevState *S = B.S;
    if (S->err & ~ERR_TIMEOUT) return;
    const long long n = S->n, an = S->an, tot = n + an;
    const int ntiles = (int)max(1ll, (tot + G_TILE - 1) / G_TILE);
    const u64 st = st_load(B.gstat + (ntiles - 1));
    const long long created = (long long)(unsigned)(st & 0xffffffffu);
    S->an = an + created;
    S->created += created;
    S->live_in += n + an;
    S->g_tile_ctr = 0;
    S->epoch += 1;
}

// ------------------------------------------------------------ radix sort
// Stable LSD radix sort of (z, x, c) records by the (z, x) key, 8-bit digits,
// digits on which all keys agree are skipped (host decides from k_keybits).
constexpr int R_THREADS = 256;
constexpr int R_WARPS = R_THREADS / 32;
constexpr int R_PER_WARP = 512;
constexpr int R_TILE = R_WARPS * R_PER_WARP;  // 4096

__device__ __forceinline__ unsigned digit_of(const u64 *Z, const u64 *X, int NW, long long i, int d) {
    const int lvl = 8 * d;
    if (lvl >= 64 * NW) {
        const int l = lvl - 64 * NW;
        return (unsigned)((Z[i * NW + (l >> 6)] >> (l & 63)) & 0xffu);
    }
    return (unsigned)((X[i * NW + (lvl >> 6)] >> (lvl & 63)) & 0xffu);
}

template <int NW>
__global__ void k_keybits(const u64 *Z, const u64 *X, long long n, u64 *orand /* [4 or] [4 and] */) {
    u64 o[2 * NW], a[2 * NW];
#pragma unroll
    for (int w = 0; w < 2 * NW; ++w) { o[w] = 0; a[w] = ~0ull; }
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            const u64 z = Z[i * NW + w], x = X[i * NW + w];
            o[w] |= z; a[w] &= z; o[NW + w] |= x; a[NW + w] &= x;
        }
    }
#pragma unroll
    for (int w = 0; w < 2 * NW; ++w) {
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            o[w] |= __shfl_xor_sync(0xffffffffu, o[w], d);
            a[w] &= __shfl_xor_sync(0xffffffffu, a[w], d);
        }
        if ((threadIdx.x & 31) == 0) { atomicOr(orand + w, o[w]); atomicAnd(orand + 4 + w, a[w]); }
    }
}

template <int NW>
__global__ void __launch_bounds__(R_THREADS) k_radix_hist(const u64 *Z, const u64 *X, long long n, int d, int *hist, int ntiles) {
    __shared__ int h[256];
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        h[threadIdx.x] = 0;
        __syncthreads();
        const long long base = (long long)t * R_TILE;
        for (int e = threadIdx.x; e < R_TILE; e += R_THREADS) {
            const long long i = base + e;
            if (i < n) atomicAdd(&h[digit_of(Z, X, NW, i, d)], 1);
        }
        __syncthreads();
        hist[(long long)threadIdx.x * ntiles + t] = h[threadIdx.x];
        __syncthreads();
    }
}

// Device-wide exclusive scan of int (three launches).
constexpr int SC_THREADS = 512;
constexpr int SC_ITEMS = 8;
constexpr int SC_TILE = SC_THREADS * SC_ITEMS;

__global__ void __launch_bounds__(SC_THREADS) k_scan_tiles(int *v, long long m, int *sums) {
    __shared__ int sm[SC_THREADS / 32 + 1];
    const long long base = (long long)blockIdx.x * SC_TILE + threadIdx.x * SC_ITEMS;
    int loc[SC_ITEMS];
    int s = 0;
#pragma unroll
    for (int q = 0; q < SC_ITEMS; ++q) { loc[q] = base + q < m ? v[base + q] : 0; s += loc[q]; }
    int tot;
    int ex = block_excl_scan<SC_THREADS>(s, 0, OpSum(), sm, &tot);
#pragma unroll
    for (int q = 0; q < SC_ITEMS; ++q) { if (base + q < m) v[base + q] = ex; ex += loc[q]; }
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(1024) k_scan_sums(int *sums, int nb) {
    __shared__ int sm[1024 / 32 + 1];
    const int per = (nb + 1023) / 1024;
    const int b0 = min((int)threadIdx.x * per, nb), b1 = min(b0 + per, nb);
    int s = 0;
    for (int b = b0; b < b1; ++b) s += sums[b];
    int tot;
    int ex = block_excl_scan<1024>(s, 0, OpSum(), sm, &tot);
    for (int b = b0; b < b1; ++b) { const int v = sums[b]; sums[b] = ex; ex += v; }
}

__global__ void k_scan_add(int *v, long long m, const int *sums) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < m) v[i] += sums[i / SC_TILE];
}

template <int NW>
__global__ void __launch_bounds__(R_THREADS) k_radix_scatter(const u64 *Z, const u64 *X, const double *C, long long n, int d,
                                                           const int *hist, int ntiles, u64 *OZ, u64 *OX, double *OC) {
    __shared__ int wcnt[R_WARPS][256];
    __shared__ int wbase[R_WARPS][256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        for (int i = tid; i < R_WARPS * 256; i += R_THREADS) (&wcnt[0][0])[i] = 0;
        __syncthreads();
        const long long wb = (long long)t * R_TILE + (long long)warp * R_PER_WARP;
        for (int ch = 0; ch < R_PER_WARP / 32; ++ch) {
            const long long i = wb + ch * 32 + lane;
            if (i < n) atomicAdd(&wcnt[warp][digit_of(Z, X, NW, i, d)], 1);
        }
        __syncthreads();
        {
            const int dg = tid;  // R_THREADS == 256 digits
            int run = hist[(long long)dg * ntiles + t];
            for (int w = 0; w < R_WARPS; ++w) { wbase[w][dg] = run; run += wcnt[w][dg]; wcnt[w][dg] = 0; }
        }
        __syncthreads();
        for (int ch = 0; ch < R_PER_WARP / 32; ++ch) {
            const long long i = wb + ch * 32 + lane;
            bool valid = i < n;
            const unsigned dg = valid ? digit_of(Z, X, NW, i, d) : 256u + lane;
            const unsigned peers = __match_any_sync(0xffffffffu, dg);
            const int rank = __popc(peers & lanemask_lt());
            int before = 0;
            if (valid) before = wcnt[warp][dg];
            __syncwarp();
            if (valid && ((long long)wbase[warp][dg] + before + rank >= n || (long long)wbase[warp][dg] + before + rank < 0)) {
                valid = false;  // impossible for a correct histogram; never write out of bounds
            }
            if (valid) {
                const long long o = (long long)wbase[warp][dg] + before + rank;
                const Key<NW> k = load_key<NW>(Z, X, i);
                store_key<NW>(OZ, OX, o, k);
                OC[o] = C[i];
                if (rank == 0) wcnt[warp][dg] = before + __popc(peers);
            }
            __syncwarp();
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ channel (stand-alone)
// SPV channel fast paths (channels.jl:203-265): c *= lambda^k, in place.
template <int NW>
__global__ void k_channel(Bufs B) {
    DevState *S = B.S;
    if (S->err) return;
    const DevParams &P = *B.P;
    const long long n = S->n;
    const int cur = S->cur;
    const u64 *Z = B.z[cur], *X = B.x[cur];
    double *C = B.c[cur];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const Key<NW> k = load_key<NW>(Z, X, i);
        C[i] = __dmul_rn(C[i], channel_factor<NW>(P, k));
    }
}

// ------------------------------------------------------------ expectation
// _expectation_spv (spv_kernels.jl:441-452) over live and pending appends,
// compensated; per-block partials reduced in block order by k_expect_final.
template <int NW>
__global__ void __launch_bounds__(256) k_expect(Bufs B, u64 k0, u64 k1, double *partials) {
    DevState *S = B.S;
    __shared__ double sm[256 / 32][2];
    const long long n = S->n, an = S->an, tot = n + an;
    const int cur = S->cur;
    const u64 *Z = B.z[cur], *X = B.x[cur];
    const double *C = B.c[cur];
    const u64 ket[2] = {k0, k1};
    Neu acc{0.0, 0.0};
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        const bool live = e < n;
        const long long i = live ? e : e - n;
        const u64 *XX = live ? X : B.ax;
        bool diag = true;
#pragma unroll
        for (int w = 0; w < NW; ++w) diag = diag && XX[i * NW + w] == 0;
        if (!diag) continue;
        const Key<NW> k = load_key<NW>(live ? Z : B.az, XX, i);
        acc.add(ket_sign<NW>(k, ket) * (live ? C[i] : B.ac[i]));
    }
    double s = acc.s, c = acc.c;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) { s += __shfl_xor_sync(0xffffffffu, s, d); c += __shfl_xor_sync(0xffffffffu, c, d); }
    if ((threadIdx.x & 31) == 0) { sm[threadIdx.x >> 5][0] = s; sm[threadIdx.x >> 5][1] = c; }
    __syncthreads();
    if (threadIdx.x == 0) {
        Neu r{0.0, 0.0};
        for (int w = 0; w < 256 / 32; ++w) { r.add(sm[w][0]); r.add(sm[w][1]); }
        partials[blockIdx.x] = r.s + r.c;
    }
}

// ------------------------------------------------------------------ variance
// variance(O, psi) (statistics.jl:6-22): sigma[x xor psi] += i^(thetas + 2 popc(z & (x xor psi))) c
// over the live terms in storage order, thetas = (4 - popc(z & x) % 4) % 4
// (symplectic_phase, type_PauliBasis.jl:36; PauliBasis * Ket, multiplication.jl:48-52);
// Var = sum |sigma|^2 - sigma[psi]^2.  k_var_records writes one record per term:
// key (x, flag) with flag 1 for an imaginary contribution, value +-c; a stable
// sort by key then puts each sigma entry's real and imaginary contributions in
// storage order, as the reference accumulates them.
template <int NW>
__global__ void k_var_records(Bufs B, u64 k0, u64 k1, u64 *RZ, u64 *RX, double *RC) {
    DevState *S = B.S;
    const long long n = S->n;
    const int cur = S->cur;
    const u64 *Z = B.z[cur], *X = B.x[cur];
    const double *C = B.c[cur];
    const u64 ket[2] = {k0, k1};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const Key<NW> k = load_key<NW>(Z, X, i);
        int yc = 0, sg = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            yc += __popcll(k.z[w] & k.x[w]);
            sg += __popcll(k.z[w] & (k.x[w] ^ ket[w]));
        }
        const int ph = ((4 - (yc & 3)) % 4 + 2 * (sg & 1)) & 3;   // power of i
        Key<NW> r;
#pragma unroll
        for (int w = 0; w < NW; ++w) { r.z[w] = k.x[w]; r.x[w] = 0; }
        r.x[0] = (u64)(ph & 1);
        store_key<NW>(RZ, RX, i, r);
        RC[i] = ph >= 2 ? -C[i] : C[i];
    }
}

// One thread per sigma entry (run of equal x in the sorted records): its real and
// imaginary parts summed in record order; gval[i] = |sigma|^2 at the run's first
// record (0 elsewhere), e1 = sigma[psi] (the x = 0 run, always real).
template <int NW>
__global__ void k_var_groups(const u64 *RZ, const u64 *RX, const double *RC, long long n, double *gval, double *e1) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const Key<NW> k = load_key<NW>(RZ, RX, i);
        bool head = i == 0;
        if (!head) {
            const Key<NW> p = load_key<NW>(RZ, RX, i - 1);
            bool same = true;
#pragma unroll
            for (int w = 0; w < NW; ++w) same = same && p.z[w] == k.z[w];
            head = !same;
        }
        if (!head) { gval[i] = 0.0; continue; }
        double re = 0.0, im = 0.0;
        for (long long j = i; j < n; ++j) {
            const Key<NW> q = load_key<NW>(RZ, RX, j);
            bool same = true;
#pragma unroll
            for (int w = 0; w < NW; ++w) same = same && q.z[w] == k.z[w];
            if (!same) break;
            if (q.x[0] & 1ull) im = __dadd_rn(im, RC[j]);
            else re = __dadd_rn(re, RC[j]);
        }
        gval[i] = __dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im));
        bool zero = true;
#pragma unroll
        for (int w = 0; w < NW; ++w) zero = zero && k.z[w] == 0;
        if (zero) *e1 = re;
    }
}

// Compensated per-block partial sums of v[0, n) in block order (for k_expect_final).
__global__ void __launch_bounds__(256) k_sum_partials(const double *v, long long n, double *partials) {
    __shared__ double sm[256 / 32][2];
    const long long per = (n + gridDim.x - 1) / gridDim.x;
    const long long b0 = blockIdx.x * per, b1 = min(n, b0 + per);
    Neu acc{0.0, 0.0};
    for (long long i = b0 + threadIdx.x; i < b1; i += blockDim.x) acc.add(v[i]);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double s = acc.s, c = acc.c;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, d);
        c += __shfl_xor_sync(0xffffffffu, c, d);
    }
    if (lane == 0) { sm[warp][0] = s; sm[warp][1] = c; }
    __syncthreads();
    if (threadIdx.x == 0) {
        Neu t{0.0, 0.0};
        for (int w = 0; w < 256 / 32; ++w) { t.add(sm[w][0]); t.add(sm[w][1]); }
        partials[blockIdx.x] = t.s + t.c;
    }
}

__global__ void k_expect_final(const double *partials, int nb, double *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        Neu r{0.0, 0.0};
        for (int b = 0; b < nb; ++b) r.add(partials[b]);
        *out = r.s + r.c;
    }
}

// ------------------------------------------------------------ check_spv
// Strictly increasing live keys (type_SparsePauliVector.jl:273-276).
template <int NW>
__global__ void k_check(Bufs B) {
    DevState *S = B.S;
    const long long n = S->n;
    const int cur = S->cur;
    const u64 *Z = B.z[cur], *X = B.x[cur];
    for (long long i = 1 + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (!key_lt<NW>(load_key<NW>(Z, X, i - 1), load_key<NW>(Z, X, i))) { atomicOr(&S->err, ERR_CHECK); return; }
    }
}

}  // namespace pp
