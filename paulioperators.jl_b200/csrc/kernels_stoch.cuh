// Stochastic truncation strategies (spv_evolve.jl:35-52, 69-99), drawing their
// random numbers from a counter-based generator: u(seed, i) = splitmix64 of the
// seed and the term's index, as a double in [0, 1).  Results are reproducible for
// a seed and statistically equivalent to the reference's (its Julia RNG stream
// cannot be reproduced), which is how they are tested.
//
//   stochastic_clip!  a term with |c| < eps survives with probability |c|/eps and
//                     is promoted to eps * sign(c); order-preserving compaction.
//   StochasticSamplingTruncation(n_keep)  weighted sampling without replacement
//                     (keys u^(1/|c|^2), the n_keep largest kept -- the method of
//                     the reference), then every kept coefficient scaled by
//                     sqrt(sum |c|^2 / sum_kept |c|^2).
#pragma once
#include "kernels_learned.cuh"

namespace pp {

__device__ __forceinline__ double counter_uniform(unsigned long long seed, long long i) {
    unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * 0x1.0p-53;
}

constexpr int FC_THREADS = 256, FC_ITEMS = 8, FC_TILE = FC_THREADS * FC_ITEMS;

// Marks: keep[i] and the coefficient a kept term gets.
__global__ void k_stoch_clip_mark(const double *C, long long n, double eps, unsigned long long seed,
                                  unsigned char *keep, double *nc) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double c = C[i];
        const double ac = fabs(c);
        unsigned char k = 1;
        double o = c;
        if (ac < eps) {
            k = counter_uniform(seed, i) < ac / eps ? 1 : 0;
            o = eps * (c / ac);
        }
        keep[i] = k;
        nc[i] = o;
    }
}

// Sampling keys: the reference's u^(1/w) with w = c^2, as the order-equivalent
// log(u) / w; a 64-bit key that grows with it (non-negative doubles order as
// their bits, so the key is ~bits(-log(u) / w)).
__global__ void k_stoch_sample_keys(const double *C, long long n, unsigned long long seed, unsigned long long *key) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double w = C[i] * C[i];
        const double u = counter_uniform(seed, i);
        double t = -log(u) / w;                    // in [0, inf]; smaller is better
        if (!(t >= 0.0)) t = INFINITY;             // w = 0 (or NaN): never preferred
        key[i] = ~(unsigned long long)__double_as_longlong(t);
    }
}

__global__ void k_key64_hist(const unsigned long long *key, long long n, Select64 *sel, int shift) {
    __shared__ unsigned h[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const unsigned long long pre = sel->prefix, msk = sel->mask;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = key[i];
        if ((k & msk) == pre) atomicAdd(&h[(k >> shift) & 255ull], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (h[i]) atomicAdd(&sel->hist[i], h[i]);
}

// keep[i] for the n_keep largest keys (ties at the cut: the smaller index); the
// per-tile tie counts come from k_flag_count on keyeq.
__global__ void k_stoch_sample_mark(const unsigned long long *key, long long n, const Select64 *sel,
                                    unsigned char *keep, unsigned char *keyeq) {
    const unsigned long long cut = sel->prefix;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        keep[i] = key[i] > cut ? 1 : 0;
        keyeq[i] = key[i] == cut ? 1 : 0;
    }
}

// Per tile of FC_TILE items: number of set flags.
__global__ void k_flag_count(const unsigned char *f, long long n, int *cnt) {
    __shared__ int sc[FC_THREADS / 32 + 1];
    const long long ntiles = (n + FC_TILE - 1) / FC_TILE;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        int c = 0;
        for (int q = 0; q < FC_ITEMS; ++q) {
            const long long i = t * FC_TILE + q * FC_THREADS + threadIdx.x;
            if (i < n) c += f[i];
        }
        int tot;
        block_excl_scan<FC_THREADS>(c, 0, OpSum(), sc, &tot);
        if (threadIdx.x == 0) cnt[t] = tot;
    }
}

// One CTA: exclusive scan of per-tile counts; *total = their sum.
__global__ void k_flag_scan(long long ntiles, const int *cnt, int *off, long long *total) {
    __shared__ long long sl[1024 / 32 + 1];
    const int per = (int)((ntiles + 1023) / 1024);
    const long long t0 = min((long long)threadIdx.x * per, ntiles), t1 = min(t0 + per, ntiles);
    long long loc = 0;
    for (long long t = t0; t < t1; ++t) loc += cnt[t];
    long long all;
    long long run = block_excl_scan<1024>(loc, 0ll, OpSum(), sl, &all);
    for (long long t = t0; t < t1; ++t) { off[t] = (int)run; run += cnt[t]; }
    if (threadIdx.x == 0) *total = all;
}

// Sampling: turns the ties at the cut into kept terms, the first `remaining` of
// them in index order (tie_off from k_flag_scan over keyeq).
__global__ void k_stoch_sample_ties(long long n, const Select64 *sel, const unsigned char *keyeq, const int *tie_off,
                                    unsigned char *keep) {
    __shared__ int sc[FC_THREADS / 32 + 1];
    const long long need = sel->remaining;
    const long long ntiles = (n + FC_TILE - 1) / FC_TILE;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long long base = t * FC_TILE + (long long)threadIdx.x * FC_ITEMS;
        int e = 0;
        for (int q = 0; q < FC_ITEMS; ++q) e += (base + q < n) ? keyeq[base + q] : 0;
        int tot;
        long long r = block_excl_scan<FC_THREADS>(e, 0, OpSum(), sc, &tot) + tie_off[t];
        for (int q = 0; q < FC_ITEMS; ++q) {
            if (base + q < n && keyeq[base + q]) {
                if (r < need) keep[base + q] = 1;
                ++r;
            }
        }
        __syncthreads();
    }
}

// Order-preserving copy of the flagged terms; coefficients from NC (or C when NC
// is null), scaled by *scale when scale is not null.
__global__ void k_flag_write(const unsigned char *f, long long n, const int *off, const u64 *Zs, const u64 *Xs,
                             const double *C, const double *NC, int NW, const double *scale, u64 *Zd, u64 *Xd,
                             double *Cd) {
    __shared__ int sc[FC_THREADS / 32 + 1];
    const double sf = scale ? *scale : 1.0;
    const long long ntiles = (n + FC_TILE - 1) / FC_TILE;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long long base = t * FC_TILE + (long long)threadIdx.x * FC_ITEMS;
        int k = 0;
        for (int q = 0; q < FC_ITEMS; ++q) k += (base + q < n) ? f[base + q] : 0;
        int tot;
        long long o = block_excl_scan<FC_THREADS>(k, 0, OpSum(), sc, &tot) + off[t];
        for (int q = 0; q < FC_ITEMS; ++q) {
            const long long i = base + q;
            if (i < n && f[i]) {
                for (int w = 0; w < NW; ++w) { Zd[o * NW + w] = Zs[i * NW + w]; Xd[o * NW + w] = Xs[i * NW + w]; }
                const double c = NC ? NC[i] : C[i];
                Cd[o] = scale ? c * sf : c;
                ++o;
            }
        }
        __syncthreads();
    }
}

// sum_i c_i^2 over all terms (w[0]) and over the flagged ones (w[1]), compensated,
// per block in block order (k_expect_final then combines the partials).
__global__ void __launch_bounds__(256) k_norm_partials(const double *C, const unsigned char *f, long long n,
                                                       double *pall, double *pkept) {
    __shared__ double sm[2][256 / 32];
    const long long per = (n + gridDim.x - 1) / gridDim.x;
    const long long b0 = blockIdx.x * per, b1 = min(n, b0 + per);
    Neu a{0.0, 0.0}, k{0.0, 0.0};
    for (long long i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        const double w = C[i] * C[i];
        a.add(w);
        if (f[i]) k.add(w);
    }
    double va = a.s + a.c, vk = k.s + k.c;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        va += __shfl_xor_sync(0xffffffffu, va, d);
        vk += __shfl_xor_sync(0xffffffffu, vk, d);
    }
    if ((threadIdx.x & 31) == 0) { sm[0][threadIdx.x >> 5] = va; sm[1][threadIdx.x >> 5] = vk; }
    __syncthreads();
    if (threadIdx.x == 0) {
        Neu ta{0.0, 0.0}, tk{0.0, 0.0};
        for (int w = 0; w < 256 / 32; ++w) { ta.add(sm[0][w]); tk.add(sm[1][w]); }
        pall[blockIdx.x] = ta.s + ta.c;
        pkept[blockIdx.x] = tk.s + tk.c;
    }
}

// scale = sqrt(all / kept) (1 when nothing is kept or kept == 0).
__global__ void k_norm_scale(const double *all, const double *kept, double *scale) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *scale = (*kept > 0.0) ? sqrt(*all / *kept) : 1.0;
}

}  // namespace pp
