// Batched instances: many independent SparsePauliVectors of N <= 64 qubits held in
// one live set.  A term of instance i stores the instance's own 64-bit words in
// z/x word 0 and i in z word 1 (x word 1 = 0).  z word 1 is the most significant
// key word, so every instance is one contiguous, sorted run of the live set and
// the window-1 rotation kernels process all instances in each launch: the sin
// branch P xor M never leaves its instance (M has no word-1 bits), the rank
// identity sees an instance boundary as a group boundary above every mask level,
// and merges never combine terms of different instances.  Per-instance angles
// and depths are read in k_classify / k_merge (term_angle); weights ignore word 1
// (DevFilter::wlow).
//
// Harvest: when instances reach their last rotation, <ket|O_i|ket> and the term
// count of each finished instance are reduced over its run (located by binary
// search on z word 1), in a fixed order; a compaction (k_merge MODE 2 with
// GEN_HARVEST) then removes their terms.
#pragma once
#include "kernels_struct.cuh"

namespace pp {

constexpr int HV_THREADS = 256;
constexpr int HV_CHUNKS = 32;     // CTAs per finished instance

// First dense index whose instance tag (z word 1) is >= tag.
__device__ __forceinline__ long long tag_lower_bound(const u64 *Z, long long n, u64 tag) {
    long long lo = 0, hi = n;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (Z[2 * mid + 1] < tag) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Partial <ket|O|ket> of chunk blockIdx.x of finished instance fin[blockIdx.y].
__global__ void __launch_bounds__(HV_THREADS) k_harvest_part(Bufs B, const int *fin, double *part, long long *range) {
    DevState *S = B.S;
    const int f = blockIdx.y;
    const u64 tag = (u64)fin[f];
    const long long n = S->n;
    const int cur = S->cur;
    const u64 *Z = B.z[cur], *X = B.x[cur];
    const double *C = B.c[cur];
    __shared__ long long s_b[2];
    __shared__ double s_red[HV_THREADS / 32];
    if (threadIdx.x < 2) s_b[threadIdx.x] = tag_lower_bound(Z, n, tag + threadIdx.x);
    __syncthreads();
    const long long lo = s_b[0], hi = s_b[1];
    if (blockIdx.x == 0 && threadIdx.x == 0) { range[2 * f] = lo; range[2 * f + 1] = hi; }
    const long long len = hi - lo;
    const long long c0 = lo + len * blockIdx.x / HV_CHUNKS, c1 = lo + len * (blockIdx.x + 1) / HV_CHUNKS;
    const u64 ket[2] = {B.P->ket[0], B.P->ket[1]};
    Neu acc{0.0, 0.0};
    for (long long i = c0 + threadIdx.x; i < c1; i += HV_THREADS) {
        const Key<2> k = load_key<2>(Z, X, i);
        if (is_diag<2>(k)) acc.add(ket_sign<2>(k, ket) * C[i]);
    }
    double v = acc.s + acc.c;
    // fixed-order reduction: warp tree, then warps in order
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        Neu t{0.0, 0.0};
        for (int w = 0; w < HV_THREADS / 32; ++w) t.add(s_red[w]);
        part[(long long)f * HV_CHUNKS + blockIdx.x] = t.s + t.c;
    }
}

// Combines the chunk partials of each finished instance in chunk order.
__global__ void k_harvest_fin(const int *fin, int nfin, const double *part, const long long *range, double *eout,
                              long long *nout) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfin) return;
    Neu t{0.0, 0.0};
    for (int c = 0; c < HV_CHUNKS; ++c) t.add(part[(long long)f * HV_CHUNKS + c]);
    eout[fin[f]] = t.s + t.c;
    nout[fin[f]] = range[2 * f + 1] - range[2 * f];
}

}  // namespace pp
