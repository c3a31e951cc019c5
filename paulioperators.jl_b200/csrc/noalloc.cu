// pp_compact_static: the clip / compaction kernel for callers that must not
// allocate device memory.
//
// Who needs it: code that runs while another component owns the device memory
// (a caller whose pool allocator has reserved the whole GPU, a host runtime that
// forbids allocation inside its latency-critical phase, or an embedding where the
// only device buffers are the ones the caller already holds).  Such a caller
// cannot create a pp_spv handle, because a handle allocates its own term sets and
// workspaces.  This entry point works on term arrays the caller passes in and
// out, and keeps its only scratch (the per-tile look-back statuses of the
// order-preserving compaction and a tile dispenser) in the file-scope array
// below, so it performs no cudaMalloc, cudaFree or other allocation.
//
// The scratch array lives in every GPU that loads the library, from load until
// process exit.  All calls share it: each call clears the part it uses before
// its kernel runs, and two calls whose work overlaps on the GPU (for example on
// two streams) race on it and produce wrong results.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/pauliprop.h"
#include "blockscan.cuh"

namespace pp {

constexpr int NA_THREADS = 256;
constexpr int NA_ITEMS = 4;
constexpr int NA_TILE = NA_THREADS * NA_ITEMS;                 // 1024 terms per tile
constexpr long long NA_MAX_TILES = PP_COMPACT_STATIC_MAX_TERMS / NA_TILE;
static_assert(PP_COMPACT_STATIC_MAX_TERMS % NA_TILE == 0, "whole tiles");
constexpr int NA_HDR = 8;                                      // [0] tile dispenser, [1] survivors

// Scratch of the no-allocation compaction: header words, then one look-back
// status per tile (flag in bits 62-63, value in bits 0-31).
static __device__ __align__(256) unsigned long long g_compact_scratch[NA_HDR + NA_MAX_TILES];

struct NaFilter {
    long long wmax, xwmax, mwmax;
    double thresh, dthresh_w, dthresh_xw;
    int use_mw, use_dw, use_dxw;
    double expw[130], expxw[130];
};

template <int NW>
__device__ __forceinline__ bool na_drop(const NaFilter &f, const Key<NW> &k, double absc) {
    if (absc <= f.thresh) return true;
    u64 o[NW];
#pragma unroll
    for (int w = 0; w < NW; ++w) o[w] = k.z[w] | k.x[w];
    const int wt = popc_w<NW>(o);
    if (wt > f.wmax) return true;
    const int xw = popc_w<NW>(k.x);
    if (xw > f.xwmax) return true;
    if (f.use_mw && majorana<NW>(k) > f.mwmax) return true;
    if (f.use_dw && __dmul_rn(absc, f.expw[wt]) <= f.dthresh_w) return true;
    if (f.use_dxw && __dmul_rn(absc, f.expxw[xw]) <= f.dthresh_xw) return true;
    return false;
}

__device__ __forceinline__ unsigned na_wait_prefix(u64 *st, int t, unsigned agg, int *bad) {
    // serial look-back by one thread, bounded: statuses start cleared (flag 0)
    if (t == 0) { st_publish(st, ST_PRE | agg); return 0; }
    st_publish(st + t, ST_AGG | agg);
    unsigned excl = 0;
    int look = t - 1;
    long long spins = 0;
    while (look >= 0) {
        const u64 v = st_load(st + look);
        const unsigned flag = (unsigned)(v >> 62);
        if (flag == 0) {
            if (++spins > SPIN_LIMIT) { *bad = 1; break; }
            continue;
        }
        excl += (unsigned)(v & 0xffffffffu);
        if (flag == 2) break;
        --look;
    }
    st_publish(st + t, ST_PRE | (u64)(excl + agg));
    return excl;
}

// Order-preserving compaction of (z, x, c)[0, n) under the filter, as
// _compact_spv! (spv_kernels.jl:395-408) but out of place; scratch = sc.
template <int NW>
__global__ void __launch_bounds__(NA_THREADS) k_compact_static(const u64 *Z, const u64 *X, const double *C, long long n,
                                                               NaFilter f, u64 *OZ, u64 *OX, double *OC,
                                                               unsigned long long *sc, int *err) {
    __shared__ int s_tile, s_bad;
    __shared__ unsigned s_base;
    __shared__ int s_scan[NA_THREADS / 32 + 1];
    __shared__ u64 s_z[NW][NA_TILE], s_x[NW][NA_TILE];
    __shared__ double s_c[NA_TILE];
    const int ntiles = (int)((n + NA_TILE - 1) / NA_TILE);
    u64 *st = sc + NA_HDR;
    const int tid = threadIdx.x;
    while (true) {
        if (tid == 0) { s_tile = (int)atomicAdd(&sc[0], 1ull); s_bad = 0; }
        __syncthreads();
        const int t = s_tile;
        if (t >= ntiles) break;
        const long long base = (long long)t * NA_TILE;
        // blocked ownership: thread tid handles terms base + tid*NA_ITEMS + q
        bool keep[NA_ITEMS];
        Key<NW> kk[NA_ITEMS];
        double cc[NA_ITEMS];
        int cnt = 0;
#pragma unroll
        for (int q = 0; q < NA_ITEMS; ++q) {
            const long long i = base + tid * NA_ITEMS + q;
            keep[q] = false;
            if (i < n) {
                kk[q] = load_key<NW>(Z, X, i);
                cc[q] = C[i];
                keep[q] = !na_drop<NW>(f, kk[q], fabs(cc[q]));
                cnt += keep[q];
            }
        }
        int tot;
        int off = block_excl_scan<NA_THREADS>(cnt, 0, OpSum(), s_scan, &tot);
        if (tid == 0) {
            int bad = 0;
            s_base = na_wait_prefix(st, t, (unsigned)tot, &bad);
            if (bad) s_bad = 1;
        }
#pragma unroll
        for (int q = 0; q < NA_ITEMS; ++q) {
            if (keep[q]) {
#pragma unroll
                for (int w = 0; w < NW; ++w) { s_z[w][off] = kk[q].z[w]; s_x[w][off] = kk[q].x[w]; }
                s_c[off] = cc[q];
                ++off;
            }
        }
        __syncthreads();
        if (s_bad && tid == 0) atomicOr(err, ERR_TIMEOUT);
        const long long ob = s_base;
        for (int e = tid; e < tot; e += NA_THREADS) {
            Key<NW> k;
#pragma unroll
            for (int w = 0; w < NW; ++w) { k.z[w] = s_z[w][e]; k.x[w] = s_x[w][e]; }
            store_key<NW>(OZ, OX, ob + e, k);
            OC[ob + e] = s_c[e];
        }
        if (t == ntiles - 1 && tid == 0) sc[1] = ob + (unsigned)tot;
        __syncthreads();
    }
}

}  // namespace pp

using namespace pp;

int pp_fail_msg(int code, const char *msg);   // sets pp_last_error() (api.cu)

// Device address of the scratch array in the calling thread's current CUDA
// context.  Host code only holds a stand-in for a __device__ symbol; the address
// must be looked up with the device current before a kernel can be given it.
// The lookup is made once per context and cached under the context's unique id
// (cuCtxGetId), so a context created after cudaDeviceReset, or another context on
// the same device, gets its own lookup instead of a stale address.
typedef CUresult (*CtxGetCurrentFn)(CUcontext *);
typedef CUresult (*CtxGetIdFn)(CUcontext, unsigned long long *);
struct NaCache {
    unsigned long long ctx_id;
    unsigned long long *ptr;
};
static std::mutex g_na_mu;
static NaCache g_na_cache[64];            // per device: the context id of the last lookup and its address
static CtxGetCurrentFn g_ctx_current = nullptr;
static CtxGetIdFn g_ctx_id = nullptr;

static int na_context_id(unsigned long long *id) {
    CUcontext ctx = nullptr;
    if (g_ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return 1;
    return g_ctx_id(ctx, id) == CUDA_SUCCESS ? 0 : 1;
}

static int na_scratch(unsigned long long **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return pp_fail_msg(PP_DEVICE_ERROR, "no usable CUDA device");
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (!g_ctx_current || !g_ctx_id) {
        void *f1 = nullptr, *f2 = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
            q2 != cudaDriverEntryPointSuccess)
            return pp_fail_msg(PP_DEVICE_ERROR, "pp_compact_static: driver context queries unavailable");
        g_ctx_current = (CtxGetCurrentFn)f1;
        g_ctx_id = (CtxGetIdFn)f2;
    }
    unsigned long long id = 0;
    const bool have_ctx = na_context_id(&id) == 0;
    NaCache &c = g_na_cache[dev];
    if (have_ctx && c.ptr && c.ctx_id == id) {
        *out = c.ptr;
        return PP_OK;
    }
    // first call in this context (the lookup also makes the runtime's context current)
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_compact_scratch);
    if (e != cudaSuccess)
        return pp_fail_msg(PP_DEVICE_ERROR, (std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e)).c_str());
    if (na_context_id(&id) != 0) return pp_fail_msg(PP_DEVICE_ERROR, "pp_compact_static: no current CUDA context");
    c.ctx_id = id;
    c.ptr = (unsigned long long *)p;
    *out = c.ptr;
    return PP_OK;
}

extern "C" int pp_compact_static(int32_t N, const void *z, const void *x, const double *c, int64_t n,
                                 const pp_filter *f, void *z_out, void *x_out, double *c_out, int64_t *n_out,
                                 void *stream) {
    if (N < 0 || N > 128) return pp_fail_msg(PP_ARGUMENT_ERROR, "pp_compact_static: N must be in 0..128");
    if (n < 0 || !n_out || (n > 0 && (!z || !x || !c || !z_out || !x_out || !c_out)))
        return pp_fail_msg(PP_ARGUMENT_ERROR, "pp_compact_static: null array or negative n");
    if (n > PP_COMPACT_STATIC_MAX_TERMS)
        return pp_fail_msg(PP_ARGUMENT_ERROR,
                           "pp_compact_static: n exceeds PP_COMPACT_STATIC_MAX_TERMS (the size of its static scratch)");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned long long *sc = nullptr;
    int r = na_scratch(&sc);
    if (r) return r;
    if (n == 0) { *n_out = 0; return PP_OK; }
    const pp_filter F = f ? *f : pp_filter{INT64_MAX, INT64_MAX, INT64_MAX, -1.0, 0.0, -1.0, 0.0, -1.0};
    NaFilter nf;
    nf.wmax = F.wmax; nf.xwmax = F.xwmax; nf.mwmax = F.mwmax;
    nf.thresh = F.thresh; nf.dthresh_w = F.dthresh_w; nf.dthresh_xw = F.dthresh_xw;
    nf.use_mw = F.mwmax != INT64_MAX; nf.use_dw = F.dthresh_w >= 0.0; nf.use_dxw = F.dthresh_xw >= 0.0;
    for (int w = 0; w < 130; ++w) {
        nf.expw[w] = std::exp(-F.alpha_w * (double)w);
        nf.expxw[w] = std::exp(-F.alpha_xw * (double)w);
    }
    const int ntiles = (int)((n + NA_TILE - 1) / NA_TILE);
    // the header (dispenser, survivors, error word) and the statuses this call uses start at zero
    if (cudaMemsetAsync(sc, 0, (size_t)(NA_HDR + ntiles) * sizeof(unsigned long long), s) != cudaSuccess)
        return pp_fail_msg(PP_DEVICE_ERROR, "pp_compact_static: clearing the scratch failed");
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int grid = std::min(ntiles, nsm * 4);
    int *err = (int *)(sc + 2);
    if (N <= 64)
        k_compact_static<1><<<grid, NA_THREADS, 0, s>>>((const u64 *)z, (const u64 *)x, c, n, nf, (u64 *)z_out,
                                                       (u64 *)x_out, c_out, sc, err);
    else
        k_compact_static<2><<<grid, NA_THREADS, 0, s>>>((const u64 *)z, (const u64 *)x, c, n, nf, (u64 *)z_out,
                                                       (u64 *)x_out, c_out, sc, err);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return pp_fail_msg(PP_DEVICE_ERROR, cudaGetErrorString(e));
    unsigned long long hdr[3] = {0, 0, 0};
    e = cudaMemcpyAsync(hdr, sc, sizeof hdr, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return pp_fail_msg(PP_DEVICE_ERROR, cudaGetErrorString(e));
    if ((int)hdr[2] & ERR_TIMEOUT) return pp_fail_msg(PP_TIMEOUT, "pp_compact_static: a look-back wait timed out");
    *n_out = (int64_t)hdr[1];
    return PP_OK;
}
