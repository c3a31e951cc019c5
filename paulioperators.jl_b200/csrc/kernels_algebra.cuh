// SparsePauliVector algebra for real (Float64) coefficients (spv_ops.jl): scalar
// multiply, norms, trace, sum! / + / -, inner_product, products and
// anticommutators.  Sums and products reuse the engine's machinery: the right
// operand (or the all-pairs triples, compacted in generation order and stably
// radix-sorted) becomes the sorted append run of an unfiltered merge, which sums
// equal keys live-first and keeps zeros -- _merge_spv!(v, m, NOFILTER) and
// _triples_to_live! (spv_kernels.jl:326-386, spv_ops.jl:234-255).
#pragma once
#include "kernels_stoch.cuh"

namespace pp {

// mul!(v, a) (spv_ops.jl:12-17)
__global__ void k_scale(double *C, long long n, double a) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        C[i] = __dmul_rn(C[i], a);
}

// (z, x, sign * c) of one term set into another (sign = +-1 exactly).
__global__ void k_copy_terms(const u64 *Zs, const u64 *Xs, const double *Cs, long long n, int NW, double sign, u64 *Zd,
                             u64 *Xd, double *Cd) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        for (int w = 0; w < NW; ++w) { Zd[i * NW + w] = Zs[i * NW + w]; Xd[i * NW + w] = Xs[i * NW + w]; }
        Cd[i] = sign < 0.0 ? -Cs[i] : Cs[i];
    }
}

// All pairs (i, j) of A x B at slot i * nB + j: key (zA ^ zB, xA ^ xB), the
// phase exponent k of _mul_spv (spv_ops.jl:264-276), and
//   kind 0 (product):        c = (i^k * cA) * cB; an odd k has an imaginary
//                            coefficient a real vector cannot hold -> *err
//   kind 1 (anticommutator): pairs with odd k vanish; c = (2(1 - k) * cA) * cB
//                            (_commutator_triples!, spv_ops.jl:400-444)
template <int NW>
__global__ void k_pairs(const u64 *ZA, const u64 *XA, const double *CA, long long nA, const u64 *ZB, const u64 *XB,
                        const double *CB, long long nB, int kind, u64 *PZ, u64 *PX, double *PC, unsigned char *keep,
                        int *err) {
    const long long tot = nA * nB;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        const long long i = e / nB, j = e - i * nB;
        const Key<NW> a = load_key<NW>(ZA, XA, i), b = load_key<NW>(ZB, XB, j);
        Key<NW> p;
        int na = 0, nb = 0, m1 = 0, nzp = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            p.z[w] = a.z[w] ^ b.z[w];
            p.x[w] = a.x[w] ^ b.x[w];
            na += __popcll(a.z[w] & a.x[w]);
            nb += __popcll(b.z[w] & b.x[w]);
            m1 += __popcll(a.x[w] & b.z[w]);
            nzp += __popcll(p.z[w] & p.x[w]);
        }
        const int k = (nzp - na - nb + 2 * m1) & 3;
        double c = 0.0;
        unsigned char kp = 1;
        if (kind == 0) {
            if (k & 1) { atomicOr(err, 1); kp = 0; }
            else c = __dmul_rn(k == 0 ? CA[i] : -CA[i], CB[j]);
        } else {
            if (k & 1) kp = 0;
            else c = __dmul_rn(__dmul_rn((double)(2 * (1 - k)), CA[i]), CB[j]);
        }
        store_key<NW>(PZ, PX, e, p);
        PC[e] = c;
        keep[e] = kp;
    }
}

// inner_product (spv_ops.jl:378-399) term values: for each term of v1 the product
// with v2's term of the same key (0 when absent), found by binary search.
template <int NW>
__global__ void k_inner_terms(const u64 *Z1, const u64 *X1, const double *C1, long long n1, const u64 *Z2,
                              const u64 *X2, const double *C2, long long n2, double *val) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n1; i += (long long)gridDim.x * blockDim.x) {
        const Key<NW> k = load_key<NW>(Z1, X1, i);
        long long lo = 0, hi = n2;
        while (lo < hi) {
            const long long mid = (lo + hi) >> 1;
            if (key_lt<NW>(load_key<NW>(Z2, X2, mid), k)) lo = mid + 1; else hi = mid;
        }
        val[i] = (lo < n2 && key_eq<NW>(load_key<NW>(Z2, X2, lo), k)) ? __dmul_rn(C1[i], C2[lo]) : 0.0;
    }
}

// norm(v, p) (spv_ops.jl:57-86) term values: c^2 (p = 2), |c| (p = 1), |c|^p.
__global__ void k_norm_terms(const double *C, long long n, double p, double *val) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double a = fabs(C[i]);
        val[i] = p == 2.0 ? __dmul_rn(C[i], C[i]) : p == 1.0 ? a : pow(a, p);
    }
}

// max |c| (exact; order-free), per block, then combined.
__global__ void k_absmax(const double *C, long long n, double *part) {
    __shared__ double sm[256 / 32];
    double m = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmax(m, fabs(C[i]));
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, d));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 256 / 32; ++w) t = fmax(t, sm[w]);
        part[blockIdx.x] = t;
    }
}

__global__ void k_max_final(const double *part, int nb, double *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double t = 0.0;
        for (int b = 0; b < nb; ++b) t = fmax(t, part[b]);
        *out = t;
    }
}

}  // namespace pp
