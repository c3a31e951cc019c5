// Block-wide scans and the decoupled look-back used by the order-preserving
// compactions (merge output, general-path appends).
#pragma once
#include "common.cuh"

namespace pp {

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <typename T, typename Op>
__device__ __forceinline__ T warp_incl_scan(T v, Op op) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v = op(v, o);
    }
    return v;
}

// Inclusive suffix scan within a warp (lane l gets op over lanes l..31).
template <typename T, typename Op>
__device__ __forceinline__ T warp_incl_suffix(T v, Op op) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T o = __shfl_down_sync(0xffffffffu, v, d);
        if (lane + d < 32) v = op(v, o);
    }
    return v;
}

// Exclusive prefix over threads in index order; returns the combination of all
// lower threads (identity for thread 0) and writes the block total.  sm needs
// THREADS/32 + 1 elements.  Contains __syncthreads(): call uniformly.
template <int THREADS, typename T, typename Op>
__device__ __forceinline__ T block_excl_scan(T v, T identity, Op op, T *sm, T *total) {
    constexpr int NWARP = THREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T incl = warp_incl_scan(v, op);
    if (lane == 31) sm[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        T w = lane < NWARP ? sm[lane] : identity;
        T wi = warp_incl_scan(w, op);
        if (lane < NWARP) sm[lane] = wi;
    }
    __syncthreads();
    T excl_in_warp = __shfl_up_sync(0xffffffffu, incl, 1);
    if (lane == 0) excl_in_warp = identity;
    T warp_off = warp == 0 ? identity : sm[warp - 1];
    T res = op(warp_off, excl_in_warp);
    if (total) *total = sm[NWARP - 1];
    __syncthreads();
    return res;
}

// Exclusive suffix over threads: combination of all higher threads.
template <int THREADS, typename T, typename Op>
__device__ __forceinline__ T block_excl_suffix(T v, T identity, Op op, T *sm) {
    constexpr int NWARP = THREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T incl = warp_incl_suffix(v, op);
    if (lane == 0) sm[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        T w = lane < NWARP ? sm[lane] : identity;
        T wi = warp_incl_suffix(w, op);
        if (lane < NWARP) sm[lane] = wi;
    }
    __syncthreads();
    T excl_in_warp = __shfl_down_sync(0xffffffffu, incl, 1);
    if (lane == 31) excl_in_warp = identity;
    T warp_off = warp == NWARP - 1 ? identity : sm[warp + 1];
    T res = op(warp_off, excl_in_warp);
    __syncthreads();
    return res;
}

// Vector variants: NV independent scans sharing one set of barriers.  sm must
// hold NV * (THREADS/32) ints.  Only the first `nact` components are scanned.
template <int THREADS, int NV, typename Op>
__device__ __forceinline__ void block_excl_scan_vec(int (&v)[NV], int identity, Op op, int *sm, int nact) {
    constexpr int NWARP = THREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl[NV];
#pragma unroll
    for (int c = 0; c < NV; ++c) {
        if (c < nact) {
            incl[c] = warp_incl_scan(v[c], op);
            if (lane == 31) sm[c * NWARP + warp] = incl[c];
        }
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int c = 0; c < NV; ++c) {
            if (c < nact) {
                int w = lane < NWARP ? sm[c * NWARP + lane] : identity;
                int wi = warp_incl_scan(w, op);
                if (lane < NWARP) sm[c * NWARP + lane] = wi;
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < NV; ++c) {
        if (c < nact) {
            int ex = __shfl_up_sync(0xffffffffu, incl[c], 1);
            if (lane == 0) ex = identity;
            v[c] = op(warp == 0 ? identity : sm[c * NWARP + warp - 1], ex);
        }
    }
    __syncthreads();
}

template <int THREADS, int NV, typename Op>
__device__ __forceinline__ void block_excl_suffix_vec(int (&v)[NV], int identity, Op op, int *sm, int nact) {
    constexpr int NWARP = THREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl[NV];
#pragma unroll
    for (int c = 0; c < NV; ++c) {
        if (c < nact) {
            incl[c] = warp_incl_suffix(v[c], op);
            if (lane == 0) sm[c * NWARP + warp] = incl[c];
        }
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int c = 0; c < NV; ++c) {
            if (c < nact) {
                int w = lane < NWARP ? sm[c * NWARP + lane] : identity;
                int wi = warp_incl_suffix(w, op);
                if (lane < NWARP) sm[c * NWARP + lane] = wi;
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < NV; ++c) {
        if (c < nact) {
            int ex = __shfl_down_sync(0xffffffffu, incl[c], 1);
            if (lane == 31) ex = identity;
            v[c] = op(warp == NWARP - 1 ? identity : sm[c * NWARP + warp + 1], ex);
        }
    }
    __syncthreads();
}

struct OpSum { template <typename T> __device__ __forceinline__ T operator()(T a, T b) const { return a + b; } };
struct OpMax { template <typename T> __device__ __forceinline__ T operator()(T a, T b) const { return a > b ? a : b; } };
struct OpMin { template <typename T> __device__ __forceinline__ T operator()(T a, T b) const { return a < b ? a : b; } };

// ---- Decoupled look-back (single-pass prefix over tiles) ----------------------
// Status word: [63:62] flag (1 aggregate, 2 inclusive prefix), [61:32] epoch,
// [31:0] value.  Statuses of an older epoch read as "not ready", so the arrays
// never need clearing between launches.
constexpr u64 ST_AGG = 1ull << 62;
constexpr u64 ST_PRE = 2ull << 62;

__device__ __forceinline__ u64 st_make(u64 flag, unsigned epoch, unsigned value) {
    return flag | ((u64)(epoch & 0x3fffffffu) << 32) | (u64)value;
}

__device__ __forceinline__ void st_publish(u64 *p, u64 v) {
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ u64 st_load(const u64 *p) {
    u64 v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Called by warp 0 of the tile's CTA.  Publishes `agg`, walks predecessors 32 at
// a time and returns the exclusive prefix (all lanes).  A wait that exceeds
// SPIN_LIMIT polls sets ERR_TIMEOUT and proceeds with what it has, so a lost
// predecessor can never hang the GPU.
__device__ __forceinline__ unsigned lookback_warp(u64 *status, int tile, unsigned epoch, unsigned agg, int *err,
                                                  long long limit = SPIN_LIMIT) {
    const int lane = threadIdx.x & 31;
    if (tile == 0) {
        if (lane == 0) st_publish(status, st_make(ST_PRE, epoch, agg));
        return 0;
    }
    if (lane == 0) st_publish(status + tile, st_make(ST_AGG, epoch, agg));
    unsigned excl = 0;
    int look = tile - 1;
    long long spins = 0;
    const unsigned ep = epoch & 0x3fffffffu;
    while (true) {
        int idx = look - lane;
        u64 st = idx >= 0 ? st_load(status + idx) : st_make(ST_PRE, epoch, 0);
        unsigned flag = (unsigned)(st >> 62);
        unsigned sep = (unsigned)((st >> 32) & 0x3fffffffu);
        if (sep != ep) flag = 0;
        unsigned pre = __ballot_sync(0xffffffffu, flag == 2);
        unsigned rdy = __ballot_sync(0xffffffffu, flag != 0);
        int fp = pre ? (__ffs(pre) - 1) : 31;
        unsigned need = fp == 31 ? 0xffffffffu : ((2u << fp) - 1u);
        if ((rdy & need) != need) {
            if (++spins > limit) {
                if (lane == 0) atomicOr(err, ERR_TIMEOUT);
                break;
            }
            continue;
        }
        unsigned v = (lane <= fp) ? (unsigned)(st & 0xffffffffu) : 0u;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
        excl += v;
        if (pre) break;
        look -= 32;
    }
    if (lane == 0) st_publish(status + tile, st_make(ST_PRE, epoch, excl + agg));
    return excl;
}

}  // namespace pp
