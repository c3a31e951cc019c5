// Learned truncation: term features, the 16 -> 64 -> 64 -> 1 GELU network on the
// 5th-generation tensor cores (tcgen05.mma, BF16 operands in shared memory, FP32
// accumulators in tensor memory), its training step, and the exact top-budget
// selection that keeps the `budget` terms of largest predicted contribution.
//
// Tensor-core use.  A CTA of 128 threads owns a tile of 128 rows (terms or
// training samples); thread r owns row r, which is TMEM lane r of every M = 128
// accumulator.  Operands live in shared memory in the canonical no-swizzle
// layouts: 8 x 8 bf16 "core matrices" of 128 contiguous bytes (8 rows of 16 B).
// A buffer holding matrix T[r][c] places core matrix (r/8, c/8) at
// (r/8) * SR + (c/8) * SC; it is read K-major (K along c) with LBO = SC,
// SBO = SR, or MN-major (MN along c, K along r) with LBO = SR, SBO = SC, so the
// same bytes serve a GEMM and its transpose:
//   forward   D1 = X  W1^T        (M 128, N 64, K 16)   A = X  K-major
//             D2 = H1 W2^T        (M 128, N 64, K 64)   A = H1 K-major
//   backward  dH1 = dZ2 W2        (M 128, N 64, K 64)   B = W2 MN-major
//             DW  = [dZ2^T; dZ1^T] [H1^T; X^T]^T
//                                 (M 128, N 80, K = 128 rows), both MN-major:
//             rows 0..63 x cols 0..63 of DW are dW2, rows 64..127 x cols 64..79 dW1.
// One thread issues the MMAs and commits them to an mbarrier; every wait is
// bounded (SPIN_LIMIT) and reports ERR_TIMEOUT.
//
// The reference has no learned truncation; the network's arithmetic is checked
// against a CPU restatement with the same bf16 rounding points, and its gradient
// against that restatement's analytic (finite-difference-checked) gradient.
#pragma once
#include <cuda_bf16.h>

#include "blockscan.cuh"

namespace pp {

constexpr int MLP_F = 16, MLP_H = 64;
constexpr int MLP_NPARAM = MLP_H * MLP_F + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H + 1;   // 5313
constexpr int MLP_ROWS = 128;                     // rows per tile = threads per CTA
// offsets in the FP32 parameter vector: W1[64][16], b1, W2[64][64], b2, w3, b3
constexpr int PO_W1 = 0, PO_B1 = 1024, PO_W2 = 1088, PO_B2 = 5184, PO_W3 = 5248, PO_B3 = 5312;

// Device copy of the network: bf16 matrices (row-major [out][in]) and FP32
// biases; w3 holds the bf16-rounded value of the last layer's weights.
struct MlpDev {
    unsigned short W1[MLP_H * MLP_F];
    unsigned short W2[MLP_H * MLP_H];
    float b1[MLP_H], b2[MLP_H], w3[MLP_H];
    float b3;
    int pad[3];
};

// Feature context: the lattice geometry and the position in the circuit.
struct FeatCtx {
    int nq, pad;
    u64 nbr[64];
    u64 light_cone, boundary;
    unsigned char row[64], col[64];
    float layer_frac, remaining_frac, theta_j, theta_h;
};

// ------------------------------------------------------------------ primitives
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (no swizzle, sm100 version field = 1).
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: BF16 x BF16 -> FP32, M x N, operand majors (0 K, 1 MN).
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N, int amaj, int bmaj) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)amaj << 15) | ((uint32_t)bmaj << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
        "[%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_alloc(uint32_t slot_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_smem), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ unsigned short bf16_bits(float f) { return __bfloat16_as_ushort(__float2bfloat16_rn(f)); }
__device__ __forceinline__ float bf16_val(float f) { return __bfloat162float(__float2bfloat16_rn(f)); }

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * expf(-0.5f * x * x) * 0.39894228040143268f;
}

// Byte offset of element (r, c) of a core-matrix buffer with block strides SR, SC.
__device__ __forceinline__ uint32_t cm_off(int r, int c, uint32_t SR, uint32_t SC) {
    return (uint32_t)(r >> 3) * SR + (uint32_t)(c >> 3) * SC + (uint32_t)(r & 7) * 16u + (uint32_t)(c & 7) * 2u;
}

// Stores 8 consecutive bf16 values of row r starting at column c (c % 8 == 0).
__device__ __forceinline__ void cm_store8(unsigned char *buf, int r, int c, uint32_t SR, uint32_t SC, const float *v) {
    uint4 q;
    q.x = (uint32_t)bf16_bits(v[0]) | ((uint32_t)bf16_bits(v[1]) << 16);
    q.y = (uint32_t)bf16_bits(v[2]) | ((uint32_t)bf16_bits(v[3]) << 16);
    q.z = (uint32_t)bf16_bits(v[4]) | ((uint32_t)bf16_bits(v[5]) << 16);
    q.w = (uint32_t)bf16_bits(v[6]) | ((uint32_t)bf16_bits(v[7]) << 16);
    *reinterpret_cast<uint4 *>(buf + cm_off(r, c, SR, SC)) = q;
}

// Shared-memory buffers of one tile (byte strides of the core-matrix blocks).
constexpr uint32_t HX_SR = 1280, HX_SC = 128;     // Hx[128][80]: H1 (cols 0..63), X (cols 64..79)
constexpr uint32_t G_SR = 2048, G_SC = 128;       // G[128][128]: dZ2 (cols 0..63), dZ1 (cols 64..127)
constexpr uint32_t W1_SR = 256, W1_SC = 128;      // W1[64][16]
constexpr uint32_t W2_SR = 1024, W2_SC = 128;     // W2[64][64]
constexpr uint32_t HX_BYTES = 16 * HX_SR, G_BYTES = 16 * G_SR, W1_BYTES = 8 * W1_SR, W2_BYTES = 8 * W2_SR;

// Loads the bf16 weight matrices into their core-matrix buffers.
__device__ __forceinline__ void load_weights(const MlpDev *W, unsigned char *w1s, unsigned char *w2s) {
    for (int e = threadIdx.x; e < MLP_H * MLP_F; e += blockDim.x) {
        const int j = e / MLP_F, f = e % MLP_F;
        *reinterpret_cast<unsigned short *>(w1s + cm_off(j, f, W1_SR, W1_SC)) = W->W1[e];
    }
    for (int e = threadIdx.x; e < MLP_H * MLP_H; e += blockDim.x) {
        const int j = e / MLP_H, k = e % MLP_H;
        *reinterpret_cast<unsigned short *>(w2s + cm_off(j, k, W2_SR, W2_SC)) = W->W2[e];
    }
}

// ------------------------------------------------------------------ features
// The 16 features of a term of an N <= 64 qubit lattice vector (word 0):
//  0 (log10|c| + 3) / 3          1-3 nX, nY, nZ / 12       4 weight / 12
//  5 |support & light cone| / 12  6 layer / L               7 remaining layers / L
//  8 adjacent support pairs / 12  9 connected components of the support / 12
// 10 row span / 8                11 column span / 8        12 support on the boundary / 12
// 13 adjacent X/Y pairs / 12     14 theta_J / 0.5          15 theta_h / 0.5
__device__ __forceinline__ void term_features(const FeatCtx &F, u64 z, u64 x, double c, float *f) {
    const u64 s = z | x;
    const double ac = fabs(c);
    const double lg = ac > 0.0 ? log10(ac) : -300.0;
    f[0] = (float)fmax((lg + 3.0) / 3.0, -4.0);
    f[1] = (float)__popcll(x & ~z) * (1.0f / 12.0f);
    f[2] = (float)__popcll(x & z) * (1.0f / 12.0f);
    f[3] = (float)__popcll(z & ~x) * (1.0f / 12.0f);
    f[4] = (float)__popcll(s) * (1.0f / 12.0f);
    f[5] = (float)__popcll(s & F.light_cone) * (1.0f / 12.0f);
    f[6] = F.layer_frac;
    f[7] = F.remaining_frac;
    int pairs = 0, xpairs = 0, rmin = 255, rmax = -1, cmin = 255, cmax = -1;
    for (u64 m = s; m; m &= m - 1) {
        const int q = __ffsll((long long)m) - 1;
        pairs += __popcll(F.nbr[q] & s);
        if ((x >> q) & 1ull) xpairs += __popcll(F.nbr[q] & x);
        const int rr = F.row[q], cc = F.col[q];
        rmin = min(rmin, rr); rmax = max(rmax, rr);
        cmin = min(cmin, cc); cmax = max(cmax, cc);
    }
    int comps = 0;
    for (u64 rem = s; rem;) {
        u64 comp = rem & (~rem + 1ull), prev = 0;
        while (comp != prev) {
            prev = comp;
            for (u64 m = comp; m; m &= m - 1) comp |= F.nbr[__ffsll((long long)m) - 1] & s;
        }
        rem &= ~comp;
        ++comps;
    }
    f[8] = (float)(pairs / 2) * (1.0f / 12.0f);
    f[9] = (float)comps * (1.0f / 12.0f);
    f[10] = s ? (float)(rmax - rmin + 1) * 0.125f : 0.0f;
    f[11] = s ? (float)(cmax - cmin + 1) * 0.125f : 0.0f;
    f[12] = (float)__popcll(s & F.boundary) * (1.0f / 12.0f);
    f[13] = (float)(xpairs / 2) * (1.0f / 12.0f);
    f[14] = F.theta_j * 2.0f;
    f[15] = F.theta_h * 2.0f;
}

__global__ void k_features(const u64 *Z, const u64 *X, const double *C, long long n, const FeatCtx *F, float *out) {
    __shared__ FeatCtx fs;
    for (int i = threadIdx.x; i < (int)(sizeof(FeatCtx) / 4); i += blockDim.x)
        reinterpret_cast<int *>(&fs)[i] = reinterpret_cast<const int *>(F)[i];
    __syncthreads();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float f[MLP_F];
        term_features(fs, Z[i], X[i], C[i], f);
#pragma unroll
        for (int k = 0; k < MLP_F; ++k) out[i * MLP_F + k] = f[k];
    }
}

// ------------------------------------------------------------------ forward
// Ordered 32-bit key of a float (larger float -> larger key).
__device__ __forceinline__ uint32_t fkey(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

struct SelectState {
    unsigned prefix, mask;        // key bits fixed so far
    long long remaining;          // how many of the keys matching the prefix are still to keep
    unsigned hist[256];
};

// Network output for rows [0, n): SRC 0 reads FP32 features feat[n][16]; SRC 1
// computes them from the live terms (Z, X, C) and also adds every score's top key
// byte to the selection histogram.  One 128-row tile per loop iteration.
template <int SRC>
__global__ void __launch_bounds__(MLP_ROWS) k_mlp_fwd(const float *feat, const u64 *Z, const u64 *Xw, const double *C,
                                                      long long n, const FeatCtx *F, const MlpDev *W, float *out,
                                                      SelectState *sel, int *err) {
    extern __shared__ __align__(128) unsigned char smraw[];
    unsigned char *hx = smraw;                      // HX_BYTES
    unsigned char *w1s = hx + HX_BYTES;             // W1_BYTES
    unsigned char *w2s = w1s + W1_BYTES;            // W2_BYTES
    __shared__ float sb1[MLP_H], sb2[MLP_H], sw3[MLP_H];
    __shared__ __align__(8) unsigned long long mbar;
    __shared__ uint32_t tslot;
    __shared__ unsigned shist[256];
    __shared__ FeatCtx fs;
    __shared__ int s_bad;
    const int r = threadIdx.x, warp = r >> 5;
    load_weights(W, w1s, w2s);
    if (r < MLP_H) { sb1[r] = W->b1[r]; sb2[r] = W->b2[r]; sw3[r] = W->w3[r]; }
    if (SRC == 1) {
        for (int i = r; i < (int)(sizeof(FeatCtx) / 4); i += MLP_ROWS)
            reinterpret_cast<int *>(&fs)[i] = reinterpret_cast<const int *>(F)[i];
        for (int i = r; i < 256; i += MLP_ROWS) shist[i] = 0;
    }
    const float b3 = W->b3;
    const uint32_t mb = smem_u32(&mbar);
    if (r == 0) { mbar_init(mb, 1); s_bad = 0; }
    if (warp == 0) tmem_alloc(smem_u32(&tslot), 128);
    fence_async_smem();
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = tslot;
    const uint32_t tlane = tbase + ((uint32_t)(warp * 32) << 16);
    const uint32_t hx_a = smem_u32(hx), w1_a = smem_u32(w1s), w2_a = smem_u32(w2s);
    const uint32_t id64 = umma_idesc(128, 64, 0, 0);
    uint32_t phase = 0;
    const long long ntiles = (n + MLP_ROWS - 1) / MLP_ROWS;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long long i = t * MLP_ROWS + r;
        const bool valid = i < n;
        float f[MLP_F];
#pragma unroll
        for (int k = 0; k < MLP_F; ++k) f[k] = 0.0f;
        if (valid) {
            if (SRC == 0) {
#pragma unroll
                for (int k = 0; k < MLP_F; ++k) f[k] = feat[i * MLP_F + k];
            } else {
                term_features(fs, Z[i], Xw[i], C[i], f);
            }
        }
        cm_store8(hx, r, 64, HX_SR, HX_SC, f);
        cm_store8(hx, r, 72, HX_SR, HX_SC, f + 8);
        fence_async_smem();
        __syncthreads();
        if (r == 0) {
            tc_fence_after();
            umma_bf16(tbase, umma_desc(hx_a + 8 * HX_SC, HX_SC, HX_SR), umma_desc(w1_a, W1_SC, W1_SR), id64, 0);
            umma_commit(mb);
        }
        if (!mbar_wait(mb, phase)) s_bad = 1;
        phase ^= 1;
        tc_fence_after();
        float h[16];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            tmem_ld16(tlane + 16 * q, h);
#pragma unroll
            for (int k = 0; k < 16; ++k) h[k] = gelu(h[k] + sb1[16 * q + k]);
            cm_store8(hx, r, 16 * q, HX_SR, HX_SC, h);
            cm_store8(hx, r, 16 * q + 8, HX_SR, HX_SC, h + 8);
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (r == 0) {
            tc_fence_after();
#pragma unroll
            for (int s = 0; s < 4; ++s)
                umma_bf16(tbase + 64, umma_desc(hx_a + 2 * s * HX_SC, HX_SC, HX_SR),
                          umma_desc(w2_a + 2 * s * W2_SC, W2_SC, W2_SR), id64, s > 0);
            umma_commit(mb);
        }
        if (!mbar_wait(mb, phase)) s_bad = 1;
        phase ^= 1;
        tc_fence_after();
        float y = b3;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            tmem_ld16(tlane + 64 + 16 * q, h);
#pragma unroll
            for (int k = 0; k < 16; ++k) y += gelu(h[k] + sb2[16 * q + k]) * sw3[16 * q + k];
        }
        if (valid) {
            out[i] = y;
            if (SRC == 1) atomicAdd(&shist[fkey(y) >> 24], 1u);
        }
        tc_fence_before();
        __syncthreads();
    }
    if (SRC == 1) {
        __syncthreads();
        for (int k = r; k < 256; k += MLP_ROWS)
            if (shist[k]) atomicAdd(&sel->hist[k], shist[k]);
    }
    tc_fence_before();
    __syncthreads();
    if (s_bad && r == 0) atomicOr(err, ERR_TIMEOUT);
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tbase, 128);
}

// Dynamic shared memory of the forward kernel: its buffers, padded so that at
// most 4 CTAs share an SM (4 x 128 TMEM columns = all 512: no allocation waits).
constexpr size_t MLP_FWD_SMEM = 48 * 1024;
static_assert(HX_BYTES + W1_BYTES + W2_BYTES <= MLP_FWD_SMEM, "forward buffers");

// ------------------------------------------------------------------ training
// Per-CTA gradient partial: dW1, db1, dW2, db2, dw3, db3 (parameter layout) and
// the loss sum, over the tiles [blockIdx.x, ntiles) step gridDim.x of the
// minibatch idx[0, B).  Deterministic: every sum has a fixed order.
__global__ void __launch_bounds__(MLP_ROWS, 1) k_mlp_grad(const float *feat, const float *target, const int *idx,
                                                          long long B, const MlpDev *W, float *gpart, int *err) {
    extern __shared__ __align__(128) unsigned char smraw[];
    unsigned char *hx = smraw;                       // HX_BYTES
    unsigned char *gb = hx + HX_BYTES;               // G_BYTES
    unsigned char *w1s = gb + G_BYTES;               // W1_BYTES
    unsigned char *w2s = w1s + W1_BYTES;             // W2_BYTES
    float *red = reinterpret_cast<float *>(w2s + W2_BYTES);   // [128][65]: per-row values for column sums
    __shared__ float sb1[MLP_H], sb2[MLP_H], sw3[MLP_H];
    __shared__ float acc_b1[MLP_H], acc_b2[MLP_H], acc_w3[MLP_H];
    __shared__ float srow[MLP_ROWS][2];
    __shared__ __align__(8) unsigned long long mbar;
    __shared__ uint32_t tslot;
    __shared__ int s_bad;
    const int r = threadIdx.x, warp = r >> 5;
    load_weights(W, w1s, w2s);
    if (r < MLP_H) {
        sb1[r] = W->b1[r]; sb2[r] = W->b2[r]; sw3[r] = W->w3[r];
        acc_b1[r] = 0.0f; acc_b2[r] = 0.0f; acc_w3[r] = 0.0f;
    }
    const float b3 = W->b3;
    float acc_b3 = 0.0f, acc_loss = 0.0f;
    const uint32_t mb = smem_u32(&mbar);
    if (r == 0) { mbar_init(mb, 1); s_bad = 0; }
    if (warp == 0) tmem_alloc(smem_u32(&tslot), 512);
    fence_async_smem();
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = tslot;
    const uint32_t tlane = tbase + ((uint32_t)(warp * 32) << 16);
    // TMEM columns: D1 0..63, D2 64..127, dH1 128..191, DW 256..335
    const uint32_t hx_a = smem_u32(hx), g_a = smem_u32(gb), w1_a = smem_u32(w1s), w2_a = smem_u32(w2s);
    const uint32_t id64 = umma_idesc(128, 64, 0, 0);
    const uint32_t id64_bmn = umma_idesc(128, 64, 0, 1);
    const uint32_t id80_mn = umma_idesc(128, 80, 1, 1);
    const float inv_b = 2.0f / (float)B;
    uint32_t phase = 0;
    int first = 1;
    const long long ntiles = (B + MLP_ROWS - 1) / MLP_ROWS;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long long row = t * MLP_ROWS + r;
        const bool valid = row < B;
        float f[MLP_F];
        float tgt = 0.0f;
#pragma unroll
        for (int k = 0; k < MLP_F; ++k) f[k] = 0.0f;
        if (valid) {
            const long long s = idx[row];
#pragma unroll
            for (int k = 0; k < MLP_F; ++k) f[k] = feat[s * MLP_F + k];
            tgt = target[s];
        }
        cm_store8(hx, r, 64, HX_SR, HX_SC, f);
        cm_store8(hx, r, 72, HX_SR, HX_SC, f + 8);
        fence_async_smem();
        __syncthreads();
        if (r == 0) {
            tc_fence_after();
            umma_bf16(tbase, umma_desc(hx_a + 8 * HX_SC, HX_SC, HX_SR), umma_desc(w1_a, W1_SC, W1_SR), id64, 0);
            umma_commit(mb);
        }
        if (!mbar_wait(mb, phase)) s_bad = 1;
        phase ^= 1;
        tc_fence_after();
        float h[16];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            tmem_ld16(tlane + 16 * q, h);
#pragma unroll
            for (int k = 0; k < 16; ++k) h[k] = gelu(h[k] + sb1[16 * q + k]);
            cm_store8(hx, r, 16 * q, HX_SR, HX_SC, h);
            cm_store8(hx, r, 16 * q + 8, HX_SR, HX_SC, h + 8);
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (r == 0) {
            tc_fence_after();
#pragma unroll
            for (int s = 0; s < 4; ++s)
                umma_bf16(tbase + 64, umma_desc(hx_a + 2 * s * HX_SC, HX_SC, HX_SR),
                          umma_desc(w2_a + 2 * s * W2_SC, W2_SC, W2_SR), id64, s > 0);
            umma_commit(mb);
        }
        if (!mbar_wait(mb, phase)) s_bad = 1;
        phase ^= 1;
        tc_fence_after();
        // output, loss and dy
        float y = b3;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            tmem_ld16(tlane + 64 + 16 * q, h);
#pragma unroll
            for (int k = 0; k < 16; ++k) y += gelu(h[k] + sb2[16 * q + k]) * sw3[16 * q + k];
        }
        const float dy = valid ? (y - tgt) * inv_b : 0.0f;
        srow[r][0] = dy;
        srow[r][1] = valid ? (y - tgt) * (y - tgt) : 0.0f;
        // dZ2 = dy w3 GELU'(Z2) -> G cols 0..63; H2 dy and dZ2 per row for the column sums
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            tmem_ld16(tlane + 64 + 16 * q, h);
            float d[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                const float z2 = h[k] + sb2[16 * q + k];
                d[k] = dy * sw3[16 * q + k] * gelu_grad(z2);
                red[r * 65 + 16 * q + k] = d[k];
            }
            cm_store8(gb, r, 16 * q, G_SR, G_SC, d);
            cm_store8(gb, r, 16 * q + 8, G_SR, G_SC, d + 8);
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (r == 0) {
            tc_fence_after();
            // dH1 = dZ2 W2: A = G (K-major, K = hidden j), B = W2 read MN-major (N = k, K = j)
#pragma unroll
            for (int s = 0; s < 4; ++s)
                umma_bf16(tbase + 128, umma_desc(g_a + 2 * s * G_SC, G_SC, G_SR),
                          umma_desc(w2_a + 2 * s * W2_SR, W2_SR, W2_SC), id64_bmn, s > 0);
            umma_commit(mb);
        }
        // column sums of this tile: db2 (+= dZ2), then dw3 (+= dy H2), db3, loss
        if (r < MLP_H) {
            float sacc = 0.0f;
            for (int q = 0; q < MLP_ROWS; ++q) sacc += red[q * 65 + r];
            acc_b2[r] += sacc;
        }
        if (!mbar_wait(mb, phase)) s_bad = 1;
        phase ^= 1;
        tc_fence_after();
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            tmem_ld16(tlane + 64 + 16 * q, h);
#pragma unroll
            for (int k = 0; k < 16; ++k) red[r * 65 + 16 * q + k] = dy * gelu(h[k] + sb2[16 * q + k]);
        }
        __syncthreads();
        if (r < MLP_H) {
            float sacc = 0.0f;
            for (int q = 0; q < MLP_ROWS; ++q) sacc += red[q * 65 + r];
            acc_w3[r] += sacc;
        }
        if (r == 0) {
            for (int q = 0; q < MLP_ROWS; ++q) { acc_b3 += srow[q][0]; acc_loss += srow[q][1]; }
        }
        __syncthreads();
        // dZ1 = dH1 GELU'(Z1) -> G cols 64..127
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float z1[16];
            tmem_ld16(tlane + 128 + 16 * q, h);
            tmem_ld16(tlane + 16 * q, z1);
            float d[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) {
                d[k] = h[k] * gelu_grad(z1[k] + sb1[16 * q + k]);
                red[r * 65 + 16 * q + k] = d[k];
            }
            cm_store8(gb, r, 64 + 16 * q, G_SR, G_SC, d);
            cm_store8(gb, r, 64 + 16 * q + 8, G_SR, G_SC, d + 8);
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        if (r == 0) {
            tc_fence_after();
            // DW += [dZ2^T; dZ1^T] [H1^T; X^T]^T over the tile's 128 rows (K), both operands MN-major
#pragma unroll
            for (int s = 0; s < 8; ++s)
                umma_bf16(tbase + 256, umma_desc(g_a + 2 * s * G_SR, G_SR, G_SC),
                          umma_desc(hx_a + 2 * s * HX_SR, HX_SR, HX_SC), id80_mn, (first && s == 0) ? 0u : 1u);
            umma_commit(mb);
        }
        if (r < MLP_H) {
            float sacc = 0.0f;
            for (int q = 0; q < MLP_ROWS; ++q) sacc += red[q * 65 + r];
            acc_b1[r] += sacc;
        }
        if (!mbar_wait(mb, phase)) s_bad = 1;
        phase ^= 1;
        tc_fence_after();
        first = 0;
        __syncthreads();
    }
    // write the partial: rows 0..63 of DW are dW2[j][*] (cols 0..63), rows 64..127 dW1[k][*] (cols 64..79)
    float *gp = gpart + (long long)blockIdx.x * (MLP_NPARAM + 1);
    float v[16];
    if (first) {
        // no tile: zero partial
        for (int e = r; e < MLP_NPARAM + 1; e += MLP_ROWS) gp[e] = 0.0f;
    } else {
        // warps 0-1 hold TMEM lanes 0..63, warps 2-3 lanes 64..127: each branch is warp-uniform
        if (r < MLP_H) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                tmem_ld16(tlane + 256 + 16 * q, v);
#pragma unroll
                for (int k = 0; k < 16; ++k) gp[PO_W2 + r * MLP_H + 16 * q + k] = v[k];
            }
        } else {
            tmem_ld16(tlane + 256 + 64, v);
#pragma unroll
            for (int k = 0; k < 16; ++k) gp[PO_W1 + (r - MLP_H) * MLP_F + k] = v[k];
        }
        if (r < MLP_H) { gp[PO_B1 + r] = acc_b1[r]; gp[PO_B2 + r] = acc_b2[r]; gp[PO_W3 + r] = acc_w3[r]; }
        if (r == 0) { gp[PO_B3] = acc_b3; gp[MLP_NPARAM] = acc_loss; }
    }
    tc_fence_before();
    __syncthreads();
    if (s_bad && r == 0) atomicOr(err, ERR_TIMEOUT);
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tbase, 512);
}

// The training kernel allocates all 512 TMEM columns; its shared memory keeps it
// alone on its SM.
constexpr size_t MLP_GRAD_SMEM = 120 * 1024;
static_assert(HX_BYTES + G_BYTES + W1_BYTES + W2_BYTES + MLP_ROWS * 65 * 4 <= MLP_GRAD_SMEM, "training buffers");

// Sums the per-CTA partials in CTA order: grad[0, NPARAM) and the loss sum.
__global__ void k_mlp_reduce(const float *gpart, int nparts, float *grad) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e > MLP_NPARAM) return;
    float s = 0.0f;
    for (int p = 0; p < nparts; ++p) s += gpart[(long long)p * (MLP_NPARAM + 1) + e];
    grad[e] = s;
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters; refreshes the bf16 copy.
__global__ void k_mlp_adam(float *p, float *m, float *v, const float *g, int step, float lr, MlpDev *W, float *loss_slot,
                           long long B) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e == 0 && loss_slot) *loss_slot = g[MLP_NPARAM] / (float)B;
    if (e >= MLP_NPARAM) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float ge = g[e];
    const float me = b1 * m[e] + (1.0f - b1) * ge;
    const float ve = b2 * v[e] + (1.0f - b2) * ge * ge;
    m[e] = me;
    v[e] = ve;
    const float mh = me / (1.0f - powf(b1, (float)step));
    const float vh = ve / (1.0f - powf(b2, (float)step));
    const float pe = p[e] - lr * mh / (sqrtf(vh) + eps);
    p[e] = pe;
    if (e < PO_B1) W->W1[e] = bf16_bits(pe);
    else if (e < PO_W2) W->b1[e - PO_B1] = pe;
    else if (e < PO_B2) W->W2[e - PO_W2] = bf16_bits(pe);
    else if (e < PO_W3) W->b2[e - PO_B2] = pe;
    else if (e < PO_B3) W->w3[e - PO_W3] = bf16_val(pe);
    else W->b3 = pe;
}

// FP32 parameter vector -> device network.
__global__ void k_mlp_set(const float *p, MlpDev *W) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= MLP_NPARAM) return;
    const float pe = p[e];
    if (e < PO_B1) W->W1[e] = bf16_bits(pe);
    else if (e < PO_W2) W->b1[e - PO_B1] = pe;
    else if (e < PO_B2) W->W2[e - PO_W2] = bf16_bits(pe);
    else if (e < PO_W3) W->b2[e - PO_B2] = pe;
    else if (e < PO_B3) W->w3[e - PO_W3] = bf16_val(pe);
    else W->b3 = pe;
}

// ------------------------------------------------------------------ top-budget selection
// Radix select of the budget-th largest score key, 8 bits per pass from the top:
// k_sel_hist counts the next byte of the keys that match the prefix so far
// (pass 0's histogram comes from k_mlp_fwd<1>), k_sel_pick fixes that byte.
__global__ void k_sel_hist(const float *score, long long n, SelectState *sel, int shift) {
    __shared__ unsigned h[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const unsigned pre = sel->prefix, msk = sel->mask;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const uint32_t k = fkey(score[i]);
        if ((k & msk) == pre) atomicAdd(&h[(k >> shift) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (h[i]) atomicAdd(&sel->hist[i], h[i]);
}

__global__ void k_sel_pick(SelectState *sel, int shift) {
    if (threadIdx.x != 0) return;
    long long rem = sel->remaining;
    int b = 255;
    for (; b > 0; --b) {
        if ((long long)sel->hist[b] >= rem) break;
        rem -= sel->hist[b];
    }
    sel->prefix |= (unsigned)b << shift;
    sel->mask |= 255u << shift;
    sel->remaining = rem;
    for (int i = 0; i < 256; ++i) sel->hist[i] = 0;
}

constexpr int SL_THREADS = 256, SL_ITEMS = 8, SL_TILE = SL_THREADS * SL_ITEMS;

// Per tile: keys above the cut, keys equal to it.
__global__ void k_sel_count(const float *score, long long n, const SelectState *sel, int *cgt, int *ceq) {
    __shared__ int sc[SL_THREADS / 32 + 1];
    const unsigned cut = sel->prefix;
    const long long ntiles = (n + SL_TILE - 1) / SL_TILE;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        int gt = 0, eq = 0;
        for (int q = 0; q < SL_ITEMS; ++q) {
            const long long i = t * SL_TILE + q * SL_THREADS + threadIdx.x;
            if (i < n) {
                const uint32_t k = fkey(score[i]);
                gt += k > cut;
                eq += k == cut;
            }
        }
        int tg, te;
        block_excl_scan<SL_THREADS>(gt, 0, OpSum(), sc, &tg);
        block_excl_scan<SL_THREADS>(eq, 0, OpSum(), sc, &te);
        if (threadIdx.x == 0) { cgt[t] = tg; ceq[t] = te; }
        __syncthreads();
    }
}

// One CTA: per tile, the ties it may keep (ties kept in index order = key order)
// and its output offset; total kept.
__global__ void k_sel_scan(long long ntiles, const SelectState *sel, const int *cgt, const int *ceq, int *tie_off,
                           int *out_off, long long *total) {
    __shared__ long long sl[1024 / 32 + 1];
    const long long need = sel->remaining;
    const int per = (int)((ntiles + 1023) / 1024);
    const long long t0 = min((long long)threadIdx.x * per, ntiles), t1 = min(t0 + per, ntiles);
    long long le = 0;
    for (long long t = t0; t < t1; ++t) le += ceq[t];
    long long all;
    long long te = block_excl_scan<1024>(le, 0ll, OpSum(), sl, &all);
    long long lk = 0;
    for (long long t = t0; t < t1; ++t) {
        const long long keep_eq = max(0ll, min((long long)ceq[t], need - te));
        tie_off[t] = (int)te;
        lk += cgt[t] + keep_eq;
        te += ceq[t];
    }
    long long kall;
    long long ko = block_excl_scan<1024>(lk, 0ll, OpSum(), sl, &kall);
    for (long long t = t0; t < t1; ++t) {
        out_off[t] = (int)ko;
        const long long te2 = tie_off[t];
        ko += cgt[t] + max(0ll, min((long long)ceq[t], need - te2));
    }
    if (threadIdx.x == 0) *total = kall;
}

// Order-preserving copy of the kept terms (score above the cut, or equal to it
// among the first `remaining` ties) from set (Zs, Xs, Cs) to (Zd, Xd, Cd).
__global__ void k_sel_write(const float *score, long long n, const SelectState *sel, const int *tie_off,
                            const int *out_off, const u64 *Zs, const u64 *Xs, const double *Cs, u64 *Zd, u64 *Xd,
                            double *Cd) {
    __shared__ int sc[SL_THREADS / 32 + 1];
    const unsigned cut = sel->prefix;
    const long long need = sel->remaining;
    const long long ntiles = (n + SL_TILE - 1) / SL_TILE;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        // blocked ownership: thread handles items base + tid*SL_ITEMS + q, in index order
        const long long base = t * SL_TILE + (long long)threadIdx.x * SL_ITEMS;
        int eq = 0;
        uint32_t k[SL_ITEMS];
        for (int q = 0; q < SL_ITEMS; ++q) {
            k[q] = base + q < n ? fkey(score[base + q]) : 0u;
            eq += (base + q < n) && k[q] == cut;
        }
        int te_all;
        int te = block_excl_scan<SL_THREADS>(eq, 0, OpSum(), sc, &te_all) + tie_off[t];
        int kp = 0;
        bool keep[SL_ITEMS];
        for (int q = 0; q < SL_ITEMS; ++q) {
            keep[q] = false;
            if (base + q < n) {
                if (k[q] > cut) keep[q] = true;
                else if (k[q] == cut) { keep[q] = te < need; ++te; }
            }
            kp += keep[q];
        }
        int kall;
        int o = block_excl_scan<SL_THREADS>(kp, 0, OpSum(), sc, &kall) + out_off[t];
        for (int q = 0; q < SL_ITEMS; ++q) {
            if (keep[q]) {
                Zd[o] = Zs[base + q];
                Xd[o] = Xs[base + q];
                Cd[o] = Cs[base + q];
                ++o;
            }
        }
        __syncthreads();
    }
}

// Uniform sample of the terms a cut drops (score key below the cut): term i is
// taken when a hash of (seed, i) falls below thr, i.e. with probability thr / 2^64;
// at most cap of them are written (their order is that of arrival).
__global__ void k_sel_sample(const float *score, long long n, const SelectState *sel, unsigned long long seed,
                             unsigned long long thr, const u64 *Z, const u64 *X, const double *C, u64 *sz, u64 *sx,
                             double *sc, long long cap, unsigned long long *cnt) {
    const unsigned cut = sel->prefix;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (fkey(score[i]) >= cut) continue;
        unsigned long long h = seed ^ ((unsigned long long)i * 0x9E3779B97F4A7C15ull);
        h = (h ^ (h >> 30)) * 0xBF58476D1CE4E5B9ull;
        h = (h ^ (h >> 27)) * 0x94D049BB133111EBull;
        h ^= h >> 31;
        if (h >= thr) continue;
        const unsigned long long pos = atomicAdd(cnt, 1ull);
        if (pos < (unsigned long long)cap) {
            sz[pos] = Z[i];
            sx[pos] = X[i];
            sc[pos] = C[i];
        }
    }
}

// Stratified sampling of live terms by log10 |c|: nb bins of equal width over
// [lo, hi) (values outside fall into the end bins).
__device__ __forceinline__ int lgc_bin(double c, double lo, double hi, int nb) {
    const double a = fabs(c);
    const double l = a > 0.0 ? log10(a) : -300.0;
    int b = (int)floor((l - lo) / (hi - lo) * nb);
    return min(max(b, 0), nb - 1);
}

__global__ void k_lgc_hist(const double *C, long long n, double lo, double hi, int nb, unsigned long long *hist) {
    __shared__ unsigned long long h[64];
    for (int i = threadIdx.x; i < nb; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        atomicAdd(&h[lgc_bin(C[i], lo, hi, nb)], 1ull);
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], h[i]);
}

// Term i of bin b is taken when a hash of (seed, i) falls below thr[b].
__global__ void k_lgc_sample(const u64 *Z, const u64 *X, const double *C, long long n, double lo, double hi, int nb,
                             const unsigned long long *thr, unsigned long long seed, u64 *sz, u64 *sx, double *sc,
                             long long cap, unsigned long long *cnt) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        unsigned long long h = seed ^ ((unsigned long long)i * 0x9E3779B97F4A7C15ull);
        h = (h ^ (h >> 30)) * 0xBF58476D1CE4E5B9ull;
        h = (h ^ (h >> 27)) * 0x94D049BB133111EBull;
        h ^= h >> 31;
        if (h >= thr[lgc_bin(C[i], lo, hi, nb)]) continue;
        const unsigned long long pos = atomicAdd(cnt, 1ull);
        if (pos < (unsigned long long)cap) {
            sz[pos] = Z[i];
            sx[pos] = X[i];
            sc[pos] = C[i];
        }
    }
}

// ------------------------------------------------------------------ |c| top-k select
// Radix select over the 64-bit patterns of |c| (non-negative doubles order as
// their bit patterns), 8 bits per pass from the top: the key of the
// `remaining`-th largest |c|.  Used by AdaptiveTruncation.
struct Select64 {
    unsigned long long prefix, mask;
    long long remaining;
    unsigned hist[256];
};

__global__ void k_abs_hist(const double *C, long long n, Select64 *sel, int shift) {
    __shared__ unsigned h[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const unsigned long long pre = sel->prefix, msk = sel->mask;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = (unsigned long long)__double_as_longlong(fabs(C[i]));
        if ((k & msk) == pre) atomicAdd(&h[(k >> shift) & 255ull], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (h[i]) atomicAdd(&sel->hist[i], h[i]);
}

__global__ void k_sel64_pick(Select64 *sel, int shift) {
    if (threadIdx.x != 0) return;
    long long rem = sel->remaining;
    int b = 255;
    for (; b > 0; --b) {
        if ((long long)sel->hist[b] >= rem) break;
        rem -= sel->hist[b];
    }
    sel->prefix |= (unsigned long long)b << shift;
    sel->mask |= 255ull << shift;
    sel->remaining = rem;
    for (int i = 0; i < 256; ++i) sel->hist[i] = 0;
}

}  // namespace pp
