// libpauliprop: C ABI (include/pauliprop.h) over the sm_100a kernels.
//
// A handle owns every device buffer of one SparsePauliVector (live + scratch
// term sets, permutation / merge workspaces, the append and sort buffers of the
// general path) and one CUDA stream.  The live term count, the live/scratch
// parity and the rotation cursor live in device memory (DevState), so a whole
// sequence of window-1 rotations is launched without host round trips; the host
// reads the state back only at chunk boundaries to grow buffers when a kernel
// flagged that the next merge would not fit (it then resumes at the rotation
// that stopped, which is result-invariant like the reference's _grow_live!
// retry, spv_kernels.jl:377-386).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/pauliprop.h"
#include "kernels_general.cuh"
#include "kernels_batch.cuh"
#include "kernels_learned.cuh"
#include "kernels_stoch.cuh"
#include "kernels_algebra.cuh"
#include "kernels_small.cuh"
#include "kernels_bucket.cuh"

using namespace pp;

static thread_local std::string g_err;
static int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

// PAULIPROP_TRACE=1: one line on stderr per engine transition (bucketed spans,
// splits, hand-overs to the sorted-merge kernels, growth of the live sets).
static bool trace_on() {
    static const bool on = [] {
        const char *e = getenv("PAULIPROP_TRACE");
        return e && *e && strcmp(e, "0") != 0;
    }();
    return on;
}
#define PP_TRACE(...)                                   \
    do {                                                \
        if (trace_on()) {                               \
            fprintf(stderr, "[pauliprop] " __VA_ARGS__); \
            fputc('\n', stderr);                        \
        }                                               \
    } while (0)
extern "C" const char *pp_last_error(void) { return g_err.c_str(); }
int pp_fail_msg(int code, const char *msg) { return fail(code, msg); }

#define CU(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            return fail(e_ == cudaErrorMemoryAllocation ? PP_OUT_OF_MEMORY : PP_DEVICE_ERROR, \
                        std::string(#call) + ": " + cudaGetErrorString(e_));             \
        }                                                                                \
    } while (0)
#define TRY(call)                     \
    do {                              \
        int r_ = (call);              \
        if (r_ != PP_OK) return r_;   \
    } while (0)

static const pp_filter NOFILTER_H = {INT64_MAX, INT64_MAX, INT64_MAX, -1.0, 0.0, -1.0, 0.0, -1.0};
static constexpr int CHUNK_ROT = 64;   // rotations launched between state read-backs

struct pp_spv {
    int N = 0, NW = 1, dev = 0, nsm = 148;
    cudaStream_t stream = nullptr;
    long long cap = 0;          // physical capacity of each live set
    long long acap_phys = 0;    // physical append capacity (general path)
    long long tcap = 0;         // sort temp capacity
    u64 *z[2] = {nullptr, nullptr}, *x[2] = {nullptr, nullptr};
    double *c[2] = {nullptr, nullptr};
    int *srcidx = nullptr, *src = nullptr;
    unsigned *meta = nullptr;
    TileAggA *aggA = nullptr;
    int *offA = nullptr, *hfirstA = nullptr, *fwdA = nullptr, *bwdA = nullptr;
    int *split_i = nullptr, *split_j = nullptr, *split_k = nullptr;
    u64 *tstat = nullptr, *gstat = nullptr;
    double *part = nullptr;
    long long nsplit_cap = 0, gtiles_cap = 0;
    u64 *az = nullptr, *ax = nullptr, *tz = nullptr, *tx = nullptr;
    double *ac = nullptr, *tc = nullptr;
    int *rhist = nullptr, *rsums = nullptr;
    long long rhist_cap = 0, rsums_cap = 0;
    u64 *orand = nullptr;
    double *epart = nullptr, *eout = nullptr;
    DevState *S = nullptr;
    DevParams *P = nullptr;
    DevParams *Ph = nullptr;    // pinned host staging
    GenRec *gens = nullptr;
    long long gens_cap = 0;
    GenRec *gens_h = nullptr;   // pinned host staging
    long long gens_h_cap = 0;
    int occA1 = 1, occA3 = 1, occB = 1, occG = 1;
    long long bytes = 0;
    std::unordered_map<void *, size_t> sizes;   // bytes of each live device allocation
    long long acap_logical_init = 16;
    long long buf_gen = 0;                 // bumped by every (re)allocation
    int *sphys = nullptr, *soff = nullptr;   // live segment table (physical base, dense start)
    int *kcnt = nullptr;                     // survivors per window-1 merge tile
    long long *rec = nullptr;             // per-rotation counters (window-1 WindowCounters)
    long long rec_cap = 0;
    bool rec_on = false;
    // batched instances (pp_evolve_batch)
    double *bcos = nullptr, *bsin = nullptr;
    long long *bend = nullptr;
    long long btab_cap = 0, binst_cap = 0;
    long long ninst = 0;
    int ncol = 0;
    bool batch_on = false;
    int *hfin = nullptr;
    Select64 *sel64 = nullptr;                // AdaptiveTruncation's |c| select
    double *vtmp = nullptr;                   // variance: sigma[psi]
    double *hpart = nullptr, *heout = nullptr;
    long long *hrange = nullptr, *hnout = nullptr;
    cudaGraphExec_t gexec[3] = {nullptr, nullptr, nullptr};
    long long gexec_gen[3] = {-1, -1, -1};
    // bucketed window-1 rotations (kernels_bucket.cuh): two bucket sets of
    // 2^bk_bits_cap buckets of bk_cap slots, hash rows, per-rotation records,
    // dense offsets, and the captured rotation graphs per bucket count
    u64 *bkz[2] = {nullptr, nullptr}, *bkx[2] = {nullptr, nullptr};
    double *bkc[2] = {nullptr, nullptr};
    int *bkcnt[2] = {nullptr, nullptr};
    int bk_bits_cap = -1;
    int bk_cap = 0;
    u64 *bk_rows = nullptr;
    BkRec *bk_rec = nullptr;
    long long bk_rec_cap = 0;
    long long *bk_off = nullptr;
    int *bk_aux = nullptr;                  // [0] largest scatter count, [1] scatter error bits
    std::unordered_map<int, cudaGraphExec_t> bk_graphs;   // key: bits * 4 + chunk class
    long long bk_graph_gen = -1;
    pp_tuning tune = {BK_DEFAULT_CAP, BK_DEFAULT_ITEMS, 6, 128};  // pp_set_tuning
    struct { int occ1 = 1, occ2 = 1, occb = 1; } bk_occ[8];        // resident CTAs per SM of each variant
    // key-sharded runs (pp_shard_*): foreign-term counts per bucket of each set,
    // this rank, the current layout, and a device counter for packed terms
    int *bkfcnt[2] = {nullptr, nullptr};
    int bkfcnt_bits = -1;
    bool shard_on = false;
    int shard_rank_bits = 0, shard_rank = 0, shard_cur = 0, shard_bits = 0;
    long long shard_L = 0;
    unsigned long long *shard_cnt = nullptr;
};

// ------------------------------------------------------------------ helpers
static void dfree(pp_spv *h, void *p) {
    if (!p) return;
    auto it = h->sizes.find(p);
    if (it != h->sizes.end()) {
        h->bytes -= (long long)it->second;
        h->sizes.erase(it);
    }
    cudaFree(p);
}

// (Re)allocates *p for count elements.  The new buffer is allocated before the
// old one is freed, so a failure leaves *p (and everything sized from it) as it
// was: callers update their capacity fields only after every allocation of a
// growth step succeeded, and the handle stays usable after an out-of-memory.
// Test hook (pp_debug_fail_alloc): the k-th next device allocation fails.
static std::atomic<long long> g_fail_alloc_after{0};
// Test hook (pp_debug_bucket_limit): bucket layouts above this many term slots
// count as not fitting in device memory (0: no limit).
static std::atomic<long long> g_bk_slot_limit{0};

template <typename T>
static int dalloc(pp_spv *h, T **p, long long count) {
    if (count <= 0) count = 1;
    if (g_fail_alloc_after.load() > 0 && g_fail_alloc_after.fetch_sub(1) == 1)
        return fail(PP_OUT_OF_MEMORY, "cudaMalloc: injected allocation failure (pp_debug_fail_alloc)");
    void *q = nullptr;
    const size_t b = (size_t)count * sizeof(T);
    cudaError_t e = cudaMalloc(&q, b);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(PP_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    dfree(h, *p);
    *p = (T *)q;
    h->sizes[q] = b;
    h->bytes += (long long)b;
    h->buf_gen++;
    return PP_OK;
}

static Bufs make_bufs(pp_spv *h) {
    Bufs B;
    memset(&B, 0, sizeof B);
    for (int s = 0; s < 2; ++s) { B.z[s] = h->z[s]; B.x[s] = h->x[s]; B.c[s] = h->c[s]; }
    B.cap = h->cap;
    B.srcidx = h->srcidx; B.meta = h->meta; B.src = h->src;
    B.aggA = h->aggA; B.offA = h->offA; B.hfirstA = h->hfirstA; B.fwdA = h->fwdA; B.bwdA = h->bwdA;
    B.split_i = h->split_i; B.split_j = h->split_j; B.split_k = h->split_k; B.tstat = h->tstat; B.part = h->part;
    B.az = h->az; B.ax = h->ax; B.ac = h->ac;
    B.acap = h->acap_phys;
    B.vz = h->az; B.vx = h->ax; B.vc = h->ac;
    B.gstat = h->gstat;
    B.rec = h->rec_on ? h->rec : nullptr;
    B.sphys = h->sphys; B.soff = h->soff;
    B.kcnt = h->kcnt;
    B.bcos = h->bcos; B.bsin = h->bsin; B.bend = h->bend;
    B.ninst = h->ninst; B.ncol = h->ncol; B.batch = h->batch_on ? 1 : 0;
    B.S = h->S; B.P = h->P; B.gens = h->gens;
    return B;
}

static int read_state(pp_spv *h, DevState *st) {
    CU(cudaMemcpyAsync(st, h->S, sizeof(DevState), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return PP_OK;
}
// (a copy from pageable memory: the host copy may be reused on return, and the
// stream orders the copy before every later launch, so no synchronisation)
static int write_state(pp_spv *h, const DevState *st) {
    CU(cudaMemcpyAsync(h->S, st, sizeof(DevState), cudaMemcpyHostToDevice, h->stream));
    return PP_OK;
}

// Merge/rotate workspaces sized for live capacity cap and append capacity acap.
// Every buffer of a growth is allocated before any is replaced, so a failure
// leaves the workspaces (and the capacities they were sized for) as they were.
static int alloc_merge_ws(pp_spv *h, long long cap, long long acap) {
    const long long need = (cap + std::max(cap, acap)) / B_D + 4;
    if (need > h->nsplit_cap) {
        int *t[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
        u64 *ts = nullptr;
        double *tp = nullptr;
        int r = 0;
        for (int i = 0; i < 6 && !r; ++i) r = dalloc(h, &t[i], need + 1);
        if (!r) r = dalloc(h, &ts, need);
        if (!r) r = dalloc(h, &tp, need * 4);
        if (r) {
            for (int i = 0; i < 6; ++i) dfree(h, t[i]);
            dfree(h, ts);
            dfree(h, tp);
            return r;
        }
        int **dst[6] = {&h->split_i, &h->split_j, &h->split_k, &h->kcnt, &h->sphys, &h->soff};
        for (int i = 0; i < 6; ++i) { dfree(h, *dst[i]); *dst[i] = t[i]; }
        dfree(h, h->tstat); h->tstat = ts;
        dfree(h, h->part); h->part = tp;
        CU(cudaMemsetAsync(h->tstat, 0, need * sizeof(u64), h->stream));
        h->nsplit_cap = need;
    }
    const long long g = (cap + acap) / G_TILE + 4;
    if (acap > 0 && g > h->gtiles_cap) {
        TRY(dalloc(h, &h->gstat, g));
        CU(cudaMemsetAsync(h->gstat, 0, g * sizeof(u64), h->stream));
        h->gtiles_cap = g;
    }
    return PP_OK;
}

static int sync_check(pp_spv *h);

// Makes the live set dense if the last window-1 merge left it as per-tile
// slots (seg_dense == 0): copies it into the other set and flips the parity.
static int ensure_dense(pp_spv *h) {
    if (!h->soff) return PP_OK;
    Bufs B;
    memset(&B, 0, sizeof B);
    for (int s = 0; s < 2; ++s) { B.z[s] = h->z[s]; B.x[s] = h->x[s]; B.c[s] = h->c[s]; }
    B.S = h->S;
    B.sphys = h->sphys;
    B.soff = h->soff;
    if (h->NW == 1) k_densify<1><<<h->nsm * 4, 256, 0, h->stream>>>(B);
    else k_densify<2><<<h->nsm * 4, 256, 0, h->stream>>>(B);
    k_densify_commit<<<1, 32, 0, h->stream>>>(B);
    return sync_check(h);
}

// Allocates live sets and structured-path workspaces for capacity newcap,
// preserving the live terms (copied into set 0).
// With preserve == false the live terms are not copied (the caller refills the
// sets) and the state's live count becomes 0 once the new sets are in place.
// want: a larger capacity to prefer (growth ahead of time); only need is required.
static int grow_live(pp_spv *h, long long need, bool preserve = true, long long want = 0) {
    long long newcap = std::max(std::max(need, want), std::max(2 * h->cap, (long long)4096));
    if (newcap > 0x7fffffffll - 8192) newcap = std::max(need, 0x7fffffffll - 8192);
    if (need > 0x7fffffffll - 8192) return fail(PP_OUT_OF_MEMORY, "term count exceeds 2^31 - 8192");
    DevState st;
    bool have = h->cap > 0;
    if (have) {
        TRY(ensure_dense(h));
        TRY(read_state(h, &st));
    }
    // refuse a growth that would leave less than 4 GiB of device memory free; when
    // the doubled capacity does not fit, step down towards the capacity needed
    {
        size_t freeb = 0, totalb = 0;
        if (cudaMemGetInfo(&freeb, &totalb) == cudaSuccess) {
            const double per = 2.0 * (2 * h->NW * 8 + 8) + 12.0 + 4.0 * TAU_MAX * 2.0 / SEG;
            const double room = (double)freeb - 4.0 * (1ull << 30);
            while ((double)newcap * per > room && newcap > need) newcap = std::max(need, newcap - newcap / 4);
            if ((double)newcap * per > room)
                return fail(PP_OUT_OF_MEMORY, "growing to " + std::to_string(newcap) +
                                                  " terms would leave less than 4 GiB of device memory free");
        }
    }
    PP_TRACE("grow live sets: need %lld, capacity %lld -> %lld", need, h->cap, newcap);
    // every new buffer first; on failure the handle is unchanged
    u64 *nz[2] = {nullptr, nullptr}, *nx[2] = {nullptr, nullptr};
    double *nc[2] = {nullptr, nullptr};
    int *nsrcidx = nullptr, *nsrc = nullptr, *noffA = nullptr, *nhfirst = nullptr, *nfwd = nullptr, *nbwd = nullptr;
    unsigned *nmeta = nullptr;
    TileAggA *nagg = nullptr;
    auto drop = [&]() {
        for (int s = 0; s < 2; ++s) { dfree(h, nz[s]); dfree(h, nx[s]); dfree(h, nc[s]); }
        dfree(h, nsrcidx); dfree(h, nsrc); dfree(h, noffA); dfree(h, nhfirst); dfree(h, nfwd); dfree(h, nbwd);
        dfree(h, nmeta); dfree(h, nagg);
    };
    const long long ta = newcap / SEG + 4;
    int r = 0;
    for (int s = 0; s < 2 && !r; ++s) {
        r = dalloc(h, &nz[s], newcap * h->NW);
        if (!r) r = dalloc(h, &nx[s], newcap * h->NW);
        if (!r) r = dalloc(h, &nc[s], newcap);
    }
    if (!r) r = dalloc(h, &nsrcidx, newcap + SEG);
    if (!r) r = dalloc(h, &nmeta, newcap + SEG);
    if (!r) r = dalloc(h, &nsrc, newcap + SEG);
    if (!r) r = dalloc(h, &nagg, ta);
    if (!r) r = dalloc(h, &noffA, ta);
    if (!r) r = dalloc(h, &nhfirst, ta);
    if (!r) r = dalloc(h, &nfwd, ta * TAU_MAX);
    if (!r) r = dalloc(h, &nbwd, ta * TAU_MAX);
    if (!r) r = alloc_merge_ws(h, newcap, h->acap_phys);   // transactional itself; larger workspaces are harmless
    if (r) { drop(); return r; }
    cudaError_t ce = cudaSuccess;
    if (have && !preserve) st.n = 0;
    if (have && st.n > 0) {
        ce = cudaMemcpyAsync(nz[0], h->z[st.cur], st.n * h->NW * 8, cudaMemcpyDeviceToDevice, h->stream);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(nx[0], h->x[st.cur], st.n * h->NW * 8, cudaMemcpyDeviceToDevice, h->stream);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(nc[0], h->c[st.cur], st.n * 8, cudaMemcpyDeviceToDevice, h->stream);
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->stream);
    if (ce != cudaSuccess) { drop(); return fail(PP_DEVICE_ERROR, cudaGetErrorString(ce)); }
    for (int s = 0; s < 2; ++s) {
        dfree(h, h->z[s]); dfree(h, h->x[s]); dfree(h, h->c[s]);
        h->z[s] = nz[s]; h->x[s] = nx[s]; h->c[s] = nc[s];
    }
    dfree(h, h->srcidx); h->srcidx = nsrcidx;
    dfree(h, h->meta); h->meta = nmeta;
    dfree(h, h->src); h->src = nsrc;
    dfree(h, h->aggA); h->aggA = nagg;
    dfree(h, h->offA); h->offA = noffA;
    dfree(h, h->hfirstA); h->hfirstA = nhfirst;
    dfree(h, h->fwdA); h->fwdA = nfwd;
    dfree(h, h->bwdA); h->bwdA = nbwd;
    h->cap = newcap;
    if (have) {
        // the live terms (if kept) are in set 0 from here on
        st.cur = 0;
        TRY(write_state(h, &st));
    }
    return PP_OK;
}

static int ensure_live(pp_spv *h, long long need, bool preserve = true, long long want = 0) {
    if (need <= h->cap) return PP_OK;
    return grow_live(h, need, preserve, want);
}

// General path: physical append buffers (keeping pending appends) and sort temps.
static int ensure_append(pp_spv *h, long long need, long long pending) {
    if (need > h->acap_phys) {
        long long nc = std::max(need, std::max(2 * h->acap_phys, (long long)4096));
        u64 *nz = nullptr, *nx = nullptr;
        double *ncc = nullptr;
        int r = dalloc(h, &nz, nc * h->NW);
        if (!r) r = dalloc(h, &nx, nc * h->NW);
        if (!r) r = dalloc(h, &ncc, nc);
        if (!r) r = alloc_merge_ws(h, h->cap, nc);
        if (r) { dfree(h, nz); dfree(h, nx); dfree(h, ncc); return r; }
        if (pending > 0) {
            CU(cudaMemcpyAsync(nz, h->az, pending * h->NW * 8, cudaMemcpyDeviceToDevice, h->stream));
            CU(cudaMemcpyAsync(nx, h->ax, pending * h->NW * 8, cudaMemcpyDeviceToDevice, h->stream));
            CU(cudaMemcpyAsync(ncc, h->ac, pending * 8, cudaMemcpyDeviceToDevice, h->stream));
        }
        CU(cudaStreamSynchronize(h->stream));
        dfree(h, h->az); dfree(h, h->ax); dfree(h, h->ac);
        h->az = nz; h->ax = nx; h->ac = ncc;
        h->acap_phys = nc;
    }
    if (std::max(h->acap_phys, h->cap) > h->tcap) {
        long long tc = std::max(h->acap_phys, h->cap);
        TRY(dalloc(h, &h->tz, tc * h->NW));
        TRY(dalloc(h, &h->tx, tc * h->NW));
        TRY(dalloc(h, &h->tc, tc));
        h->tcap = tc;
    }
    return PP_OK;
}

static int check_err(pp_spv *h, const DevState &st) {
    if (st.err & ERR_BOUNDS) {
        char b[160];
        snprintf(b, sizeof b, "internal error: a computed index fell outside its buffer (check %llu, value %llu)",
                 st.dbg >> 40, st.dbg & 0xffffffffffull);
        return fail(PP_DEVICE_ERROR, b);
    }
    if (st.err & ERR_TIMEOUT) return fail(PP_TIMEOUT, "a device-side look-back wait timed out");
    if (st.err & ERR_TILE) return fail(PP_ERROR_EXCEPTION, "an equal-key run exceeded the merge tile staging size");
    return PP_OK;
}

static int sync_check(pp_spv *h) {
    if (!h->stream) return PP_OK;
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return fail(PP_DEVICE_ERROR, std::string("kernel failure: ") + cudaGetErrorString(e));
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(PP_DEVICE_ERROR, std::string("launch failure: ") + cudaGetErrorString(e));
    return PP_OK;
}

// ------------------------------------------------------------------ host tables
// lambda^k by compensated binary powering (square-and-multiply carrying each
// product's rounding error as a double-double; x*x*x for k == 3), the
// algorithm Julia uses for Float64^Integer.
static double jl_pow_int(double x, long long n) {
    if (n == 0) return 1.0;
    double y = 1.0, xnlo = 0.0, ynlo = 0.0;
    if (n == 3) return x * x * x;
    if (n < 0) {
        double rx = 1.0 / x;
        if (n == -2) return rx * rx;
        if (std::isfinite(x)) xnlo = -std::fma(x, rx, -1.0) * rx;
        x = rx;
        n = -n;
    }
    while (n > 1) {
        if (n & 1) {
            double err = std::fma(y, xnlo, x * ynlo);
            double p = x * y;
            ynlo = std::fma(x, y, -p);
            y = p;
            ynlo += err;
        }
        double err = x * 2.0 * xnlo;
        double p = x * x;
        xnlo = std::fma(x, x, -p);
        x = p;
        xnlo += err;
        n >>= 1;
    }
    if (!std::isfinite(x)) return x * y;
    return std::fma(x, y, std::fma(y, xnlo, x * ynlo));
}

extern "C" int pp_power_table(double lambda, int32_t kmax, double *out) {
    if (!out || kmax < 0) return fail(PP_ARGUMENT_ERROR, "pp_power_table: bad arguments");
    for (int k = 0; k <= kmax; ++k) out[k] = jl_pow_int(lambda, k);
    return PP_OK;
}

static void compile_filter(const pp_filter *f, DevFilter *d) {
    const pp_filter &F = f ? *f : NOFILTER_H;
    d->wmax = F.wmax; d->xwmax = F.xwmax; d->mwmax = F.mwmax;
    d->thresh = F.thresh; d->dthresh_w = F.dthresh_w; d->dthresh_xw = F.dthresh_xw;
    d->use_mw = F.mwmax != INT64_MAX;
    d->use_dw = F.dthresh_w >= 0.0;
    d->use_dxw = F.dthresh_xw >= 0.0;
    d->coeff_based = (F.thresh >= 0.0) || d->use_dw || d->use_dxw;
    d->wlow = 0;
    for (int w = 0; w < 130; ++w) {
        d->expw[w] = std::exp(-F.alpha_w * (double)w);     // absc * exp(-alpha*w), spv_kernels.jl:73
        d->expxw[w] = std::exp(-F.alpha_xw * (double)w);   // spv_kernels.jl:76
    }
}

static bool filter_is_nofilter(const pp_filter *f) {
    if (!f) return true;
    return f->wmax == INT64_MAX && f->xwmax == INT64_MAX && f->mwmax == INT64_MAX && f->thresh < 0.0 &&
           f->dthresh_w < 0.0 && f->dthresh_xw < 0.0;
}

static void load_word(const void *p, int NW, u64 *w) {
    w[0] = w[1] = 0;
    if (p) memcpy(w, p, NW * 8);
}

static u64 lvl_mask_all(int N, int word) {
    int lo = 64 * word;
    if (N <= lo) return 0;
    if (N >= lo + 64) return ~0ull;
    return (1ull << (N - lo)) - 1ull;
}

// Channel argument validation (channels.jl:206-207, 225-226, 236, 247, 258) and tables.
static int build_channel(pp_spv *h, int kind, const double *prm, const void *mask, DevParams *P) {
    if (kind < 0 || kind > 4) return fail(PP_ARGUMENT_ERROR, "unknown channel kind");
    if (!prm) return fail(PP_ARGUMENT_ERROR, "channel parameters missing");
    double lX, lY = 1.0, lZ = 1.0;
    if (kind == 4) {
        const double pX = prm[0], pY = prm[1], pZ = prm[2];
        if (!(pX >= 0 && pY >= 0 && pZ >= 0))
            return fail(PP_ARGUMENT_ERROR, "probabilities must be non-negative");
        if (!(pX + pY + pZ <= 1.0 + 4.0 * 2.220446049250313e-16))
            return fail(PP_ARGUMENT_ERROR, "pX+pY+pZ must be <= 1");
        lX = 1.0 - 2.0 * (pY + pZ);
        lY = 1.0 - 2.0 * (pX + pZ);
        lZ = 1.0 - 2.0 * (pX + pY);
    } else {
        const double p = prm[0];
        if (!(p >= 0.0 && p <= 1.0)) return fail(PP_ARGUMENT_ERROR, "channel parameter p must be in [0,1]");
        lX = kind == 0 ? 1.0 - 4.0 * p / 3.0 : 1.0 - 2.0 * p;
    }
    P->chan_kind = kind;
    for (int k = 0; k < 130; ++k) {
        P->chanX[k] = jl_pow_int(lX, k);
        P->chanY[k] = jl_pow_int(lY, k);
        P->chanZ[k] = jl_pow_int(lZ, k);
    }
    if (mask) {
        load_word(mask, h->NW, P->chan_mask);
    } else {
        P->chan_mask[0] = lvl_mask_all(h->N, 0);
        P->chan_mask[1] = h->NW == 2 ? lvl_mask_all(h->N, 1) : 0;
    }
    return PP_OK;
}

static int upload_params(pp_spv *h) {
    CU(cudaMemcpyAsync(h->P, h->Ph, sizeof(DevParams), cudaMemcpyHostToDevice, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return PP_OK;
}

// GenRec for one generator: mask levels (descending) of M = (gz, gx).
static int make_gen(const pp_spv *h, const u64 *gz, const u64 *gx, double cv, double sv, GenRec *g, bool *structured) {
    memset(g, 0, sizeof *g);
    for (int w = 0; w < 2; ++w) { g->gz[w] = w < h->NW ? gz[w] : 0; g->gx[w] = w < h->NW ? gx[w] : 0; }
    g->cosv = cv;
    g->sinv = sv;
    int ng = 0;
    for (int w = 0; w < h->NW; ++w) ng += __builtin_popcountll(g->gz[w] & g->gx[w]);
    g->ng = ng;
    int k = 0;
    bool ok = true;
    for (int lvl = 128 * h->NW - 1; lvl >= 0; --lvl) {
        int bit;
        if (lvl >= 64 * h->NW) { int l = lvl - 64 * h->NW; bit = (int)((g->gz[l >> 6] >> (l & 63)) & 1); }
        else bit = (int)((g->gx[lvl >> 6] >> (lvl & 63)) & 1);
        if (!bit) continue;
        if (k < KMAX) g->level[k] = (short)lvl;
        ++k;
    }
    if (k > KMAX) { ok = false; k = KMAX; }
    g->k = k;
    *structured = ok;
    return PP_OK;
}

// ------------------------------------------------------------------ launches
template <int NW>
static int launch_setup(pp_spv *h) {
    CU(cudaFuncSetAttribute(k_classify<NW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)(2 * NW * A_TILE * 8 + A_TILE)));
    CU(cudaFuncSetAttribute(k_merge<NW, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)merge_smem_bytes<NW>()));
    CU(cudaFuncSetAttribute(k_tilescan<NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tilescan_smem<NW>()));
    CU(cudaFuncSetAttribute(k_merge<NW, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)merge_smem_bytes<NW>()));
    CU(cudaFuncSetAttribute(k_merge<NW, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)merge_smem_bytes<NW>()));
    CU(cudaFuncSetAttribute(k_small_run<NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)small_smem<NW>()));
    if (NW == 2) {
        // two merge CTAs per SM need the largest shared-memory carveout (2 x 113 KB);
        // N <= 64 leaves the split to the driver (more L1 for the merge's gathers)
        const int mx = (int)cudaSharedmemCarveoutMaxShared;
        CU(cudaFuncSetAttribute(k_merge<NW, 0>, cudaFuncAttributePreferredSharedMemoryCarveout, mx));
        CU(cudaFuncSetAttribute(k_merge<NW, 1>, cudaFuncAttributePreferredSharedMemoryCarveout, mx));
        CU(cudaFuncSetAttribute(k_merge<NW, 2>, cudaFuncAttributePreferredSharedMemoryCarveout, mx));
    }
    int occ = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_classify<NW>, A_THREADS, 2 * NW * A_TILE * 8 + A_TILE));
    h->occA1 = std::max(1, occ);
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_permute<NW>, A_THREADS, 0));
    h->occA3 = std::max(1, occ);
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_merge<NW, 0>, B_THREADS, merge_smem_bytes<NW>()));
    h->occB = std::max(1, occ);
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_rotate_general<NW>, G_THREADS, 0));
    h->occG = std::max(1, occ);
    return PP_OK;
}

// One structured window-1 rotation: 6 launches, no host synchronisation.
template <int NW>
static void launch_struct_rotation(pp_spv *h, const Bufs &B) {
    cudaStream_t s = h->stream;
    k_classify<NW><<<h->nsm * h->occA1, A_THREADS, 2 * NW * A_TILE * 8 + A_TILE, s>>>(B);
    k_tilescan<NW><<<1, S_THREADS, tilescan_smem<NW>(), s>>>(B);
    k_permute<NW><<<h->nsm * h->occA3, A_THREADS, 0, s>>>(B);
    k_partition<NW, 0><<<h->nsm * 4, P_THREADS, 0, s>>>(B);
    k_merge<NW, 0><<<h->nsm * h->occB, B_THREADS, merge_smem_bytes<NW>(), s>>>(B, 0);
    k_commit<0><<<1, 256, 0, s>>>(B, 0);
}

template <int NW, int MODE>
static void launch_merge(pp_spv *h, const Bufs &B, int flags) {
    cudaStream_t s = h->stream;
    k_partition<NW, MODE><<<h->nsm * 4, P_THREADS, 0, s>>>(B);
    k_merge<NW, MODE><<<h->nsm * h->occB, B_THREADS, merge_smem_bytes<NW>(), s>>>(B, flags);
    k_commit<MODE><<<1, 256, 0, s>>>(B, flags);
}

// Digit-histogram and scan workspaces of a radix sort of n records.
static int radix_reserve(pp_spv *h, long long n) {
    const long long m = 256ll * ((n + R_TILE - 1) / R_TILE);
    if (m > h->rhist_cap) { TRY(dalloc(h, &h->rhist, m)); h->rhist_cap = m; }
    const long long nb = (m + SC_TILE - 1) / SC_TILE;
    if (nb > h->rsums_cap) { TRY(dalloc(h, &h->rsums, nb)); h->rsums_cap = nb; }
    return PP_OK;
}

// Stable LSD radix sort of n records in set A (za, xa, ca) using set T as the
// ping-pong partner.  *in_t = 1 if the result ended in T.
template <int NW>
static int radix_sort(pp_spv *h, u64 *za, u64 *xa, double *ca, u64 *zt, u64 *xt, double *ct, long long n, int *in_t) {
    *in_t = 0;
    if (n <= 1) return PP_OK;
    cudaStream_t s = h->stream;
    u64 init[8] = {0, 0, 0, 0, ~0ull, ~0ull, ~0ull, ~0ull};
    CU(cudaMemcpyAsync(h->orand, init, sizeof init, cudaMemcpyHostToDevice, s));
    k_keybits<NW><<<h->nsm * 4, 256, 0, s>>>(za, xa, n, h->orand);
    u64 orand[8];
    CU(cudaMemcpyAsync(orand, h->orand, sizeof orand, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    const int ntiles = (int)((n + R_TILE - 1) / R_TILE);
    const long long m = 256ll * ntiles;
    TRY(radix_reserve(h, n));
    const long long nb = (m + SC_TILE - 1) / SC_TILE;
    u64 *cz = za, *cx = xa, *oz = zt, *ox = xt;
    double *cc = ca, *oc = ct;
    int passes = 0;
    for (int d = 0; d < 16 * NW; ++d) {
        const int lvl = 8 * d;
        u64 vary;
        if (lvl >= 64 * NW) { int l = lvl - 64 * NW; vary = (orand[l >> 6] ^ orand[4 + (l >> 6)]) >> (l & 63); }
        else vary = (orand[NW + (lvl >> 6)] ^ orand[4 + NW + (lvl >> 6)]) >> (lvl & 63);
        if ((vary & 0xffull) == 0) continue;
        const int grid = std::min(ntiles, h->nsm * 8);
        k_radix_hist<NW><<<grid, R_THREADS, 0, s>>>(cz, cx, n, d, h->rhist, ntiles);
        k_scan_tiles<<<(int)nb, SC_THREADS, 0, s>>>(h->rhist, m, h->rsums);
        k_scan_sums<<<1, 1024, 0, s>>>(h->rsums, (int)nb);
        k_scan_add<<<(int)((m + 255) / 256), 256, 0, s>>>(h->rhist, m, h->rsums);
        k_radix_scatter<NW><<<grid, R_THREADS, 0, s>>>(cz, cx, cc, n, d, h->rhist, ntiles, oz, ox, oc);
        std::swap(cz, oz); std::swap(cx, ox); std::swap(cc, oc);
        ++passes;
    }
    *in_t = passes & 1;
    return sync_check(h);
}

static int radix_sort_nw(pp_spv *h, u64 *za, u64 *xa, double *ca, u64 *zt, u64 *xt, double *ct, long long n, int *in_t) {
    return h->NW == 1 ? radix_sort<1>(h, za, xa, ca, zt, xt, ct, n, in_t)
                      : radix_sort<2>(h, za, xa, ca, zt, xt, ct, n, in_t);
}

// ------------------------------------------------------------------ C ABI
extern "C" int pp_create(int32_t N, int64_t live_cap, int64_t append_cap, pp_spv **out) {
    if (!out) return fail(PP_ARGUMENT_ERROR, "pp_create: out is NULL");
    *out = nullptr;
    if (N < 0) return fail(PP_ARGUMENT_ERROR, "N must be >= 0");
    if (N > 128) return fail(PP_ERROR_EXCEPTION, "N > 128 requires a multi-word type (add BitIntegers.jl and extend _word_type)");
    pp_spv *h = new pp_spv();
    h->N = N;
    h->NW = N <= 64 ? 1 : 2;
    h->acap_logical_init = std::max<int64_t>(1, append_cap);
    auto bail = [&](int code) { pp_destroy(h); return code; };
    cudaError_t e = cudaGetDevice(&h->dev);
    if (e != cudaSuccess) { g_err = std::string("no CUDA device: ") + cudaGetErrorString(e); delete h; return PP_DEVICE_ERROR; }
    cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, h->dev);
    e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { g_err = cudaGetErrorString(e); delete h; return PP_DEVICE_ERROR; }
    int r = h->NW == 1 ? launch_setup<1>(h) : launch_setup<2>(h);
    if (r) return bail(r);
    if ((r = dalloc(h, &h->S, 1))) return bail(r);
    if ((r = dalloc(h, &h->P, 1))) return bail(r);
    if ((r = dalloc(h, &h->orand, 8))) return bail(r);
    if ((r = dalloc(h, &h->epart, 4096))) return bail(r);
    if ((r = dalloc(h, &h->eout, 1))) return bail(r);
    if (cudaMallocHost((void **)&h->Ph, sizeof(DevParams)) != cudaSuccess) return bail(fail(PP_OUT_OF_MEMORY, "cudaMallocHost"));
    memset(h->Ph, 0, sizeof(DevParams));
    h->Ph->chan_kind = -1;
    compile_filter(nullptr, &h->Ph->strict);
    compile_filter(nullptr, &h->Ph->local);
    compile_filter(nullptr, &h->Ph->clip);
    if ((r = upload_params(h))) return bail(r);
    DevState st;
    memset(&st, 0, sizeof st);
    st.acap_logical = h->acap_logical_init;
    st.seg_dense = 1;
    if ((r = write_state(h, &st))) return bail(r);
    if ((r = grow_live(h, std::max<int64_t>(live_cap, 4096)))) return bail(r);
    *out = h;
    return PP_OK;
}

extern "C" int pp_destroy(pp_spv *h) {
    if (!h) return PP_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    void *ptrs[] = {h->z[0], h->z[1], h->x[0], h->x[1], h->c[0], h->c[1], h->srcidx, h->src, h->meta, h->aggA,
                    h->offA, h->hfirstA, h->fwdA, h->bwdA, h->split_i, h->split_j, h->tstat, h->gstat, h->part,
                    h->az, h->ax, h->ac, h->tz, h->tx, h->tc, h->rhist, h->rsums, h->orand, h->epart, h->eout,
                    h->S, h->P, h->gens, h->rec, h->sphys, h->soff, h->kcnt, h->split_k,
                    h->bcos, h->bsin, h->bend, h->hfin, h->hpart, h->heout, h->hrange, h->hnout, h->sel64, h->vtmp};
    for (void *p : ptrs) if (p) cudaFree(p);
    for (int i = 0; i < 3; ++i) if (h->gexec[i]) cudaGraphExecDestroy(h->gexec[i]);
    for (auto &kv : h->bk_graphs) cudaGraphExecDestroy(kv.second);
    void *bptrs[] = {h->bkz[0], h->bkz[1], h->bkx[0], h->bkx[1], h->bkc[0], h->bkc[1], h->bkcnt[0], h->bkcnt[1],
                     h->bk_rows, h->bk_rec, h->bk_off, h->bk_aux, h->bkfcnt[0], h->bkfcnt[1], h->shard_cnt};
    for (void *p : bptrs) if (p) cudaFree(p);
    if (h->Ph) cudaFreeHost(h->Ph);
    if (h->gens_h) cudaFreeHost(h->gens_h);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return PP_OK;
}

extern "C" int pp_upload(pp_spv *h, const void *z, const void *x, const double *c, int64_t n, int32_t sorted) {
    if (!h) return fail(PP_ARGUMENT_ERROR, "null handle");
    if (n < 0) return fail(PP_ARGUMENT_ERROR, "n must be >= 0");
    if (n > 0 && (!z || !x || !c)) return fail(PP_ARGUMENT_ERROR, "null term arrays");
    DevState st;
    TRY(read_state(h, &st));
    st.n = 0; st.an = 0; st.cur = 0; st.err = 0; st.seg_dense = 1;
    TRY(write_state(h, &st));
    TRY(ensure_live(h, n));
    const size_t wb = (size_t)h->NW * 8;
    if (n > 0) {
        CU(cudaMemcpyAsync(h->z[0], z, n * wb, cudaMemcpyDefault, h->stream));
        CU(cudaMemcpyAsync(h->x[0], x, n * wb, cudaMemcpyDefault, h->stream));
        CU(cudaMemcpyAsync(h->c[0], c, n * 8, cudaMemcpyDefault, h->stream));
    }
    TRY(read_state(h, &st));
    st.n = n; st.cur = 0;
    if (!sorted && n > 1) {
        int in_t = 0;
        TRY(radix_sort_nw(h, h->z[0], h->x[0], h->c[0], h->z[1], h->x[1], h->c[1], n, &in_t));
        st.cur = in_t;
    }
    TRY(write_state(h, &st));
    return PP_OK;
}

extern "C" int pp_download(pp_spv *h, void *z, void *x, double *c, int64_t cap, int64_t *n) {
    if (!h) return fail(PP_ARGUMENT_ERROR, "null handle");
    DevState st;
    TRY(read_state(h, &st));
    const long long m = std::min<long long>(st.n, std::max<int64_t>(cap, 0));
    const size_t wb = (size_t)h->NW * 8;
    if (m > 0) {
        if (z) CU(cudaMemcpyAsync(z, h->z[st.cur], m * wb, cudaMemcpyDefault, h->stream));
        if (x) CU(cudaMemcpyAsync(x, h->x[st.cur], m * wb, cudaMemcpyDefault, h->stream));
        if (c) CU(cudaMemcpyAsync(c, h->c[st.cur], m * 8, cudaMemcpyDefault, h->stream));
        CU(cudaStreamSynchronize(h->stream));
    }
    if (n) *n = st.n;
    return PP_OK;
}

extern "C" int pp_length(pp_spv *h, int64_t *n) {
    if (!h || !n) return fail(PP_ARGUMENT_ERROR, "null argument");
    DevState st;
    TRY(read_state(h, &st));
    *n = st.n;
    return PP_OK;
}

extern "C" int pp_copy(pp_spv *h, pp_spv **out) {
    if (!h || !out) return fail(PP_ARGUMENT_ERROR, "null argument");
    DevState st;
    TRY(read_state(h, &st));
    pp_spv *o = nullptr;
    TRY(pp_create(h->N, st.n, st.acap_logical, &o));
    const size_t wb = (size_t)h->NW * 8;
    if (st.n > 0) {
        cudaMemcpyAsync(o->z[0], h->z[st.cur], st.n * wb, cudaMemcpyDeviceToDevice, o->stream);
        cudaMemcpyAsync(o->x[0], h->x[st.cur], st.n * wb, cudaMemcpyDeviceToDevice, o->stream);
        cudaMemcpyAsync(o->c[0], h->c[st.cur], st.n * 8, cudaMemcpyDeviceToDevice, o->stream);
    }
    DevState so;
    memset(&so, 0, sizeof so);
    so.n = st.n;
    so.acap_logical = st.acap_logical;
    so.seg_dense = 1;
    int r = write_state(o, &so);
    if (r) { pp_destroy(o); return r; }
    *out = o;
    return PP_OK;
}

static int ensure_gens(pp_spv *h, long long L) {
    if (L > h->gens_cap) {
        TRY(dalloc(h, &h->gens, L));
        h->gens_cap = L;
    }
    if (L > h->gens_h_cap) {
        if (h->gens_h) cudaFreeHost(h->gens_h);
        if (cudaMallocHost((void **)&h->gens_h, L * sizeof(GenRec)) != cudaSuccess)
            return fail(PP_OUT_OF_MEMORY, "cudaMallocHost");
        h->gens_h_cap = L;
    }
    return PP_OK;
}

// CUDA graph of `len` consecutive window-1 rotations (6 kernels each).  The
// kernels take only buffer pointers and read the rotation cursor, counts and
// parity from DevState, so one instantiated graph serves every chunk until a
// buffer is reallocated.
template <int NW>
static int struct_graph(pp_spv *h, int gi, int len) {
    if (h->gexec[gi] && h->gexec_gen[gi] == h->buf_gen) return PP_OK;
    if (h->gexec[gi]) { cudaGraphExecDestroy(h->gexec[gi]); h->gexec[gi] = nullptr; }
    Bufs B = make_bufs(h);
    cudaGraph_t graph = nullptr;
    CU(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    for (int r = 0; r < len; ++r) launch_struct_rotation<NW>(h, B);
    CU(cudaStreamEndCapture(h->stream, &graph));
    cudaError_t e = cudaGraphInstantiate(&h->gexec[gi], graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(PP_DEVICE_ERROR, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    h->gexec_gen[gi] = h->buf_gen;
    return PP_OK;
}

// Per-call accounting of launches and (when profiling) per-kernel device time.
struct RunProf {
    bool on = false;
    double t_rotate = 0, t_partition = 0, t_merge = 0;
    long long launches = 0;
    long long bk_rot = 0;          // rotations run on buckets
    double bk_bytes = 0;           // their algorithmic bytes B * (n_in + n_out)
};

// ------------------------------------------------------------------ bucketed window-1 rotations
// Window-1 rotations of a live set larger than k_small_run's shared memory run
// one k_bk_rotate launch each over a hash-bucketed copy of the live set
// (kernels_bucket.cuh); the sequence ends with a gather into a dense array and a
// radix sort, so the live set is dense and sorted between calls as before.
static int expect_dev(pp_spv *h, const u64 *k, double *out);
static constexpr int BK_MIN_ROT = 32;     // shorter sequences keep the sorted-merge kernels
// Internal status (never returned by the C ABI): a bucket layout for the live set
// would not fit in device memory; the sequence continues on the sorted-merge
// kernels from the rotation the device cursor is at.
static constexpr int BK_NOFIT = 0x4b4e4f46;

// PAULIPROP_WINDOW1_PATH=tiles selects the sorted-merge kernels instead (both
// give the same result; the switch exists for comparisons).
static bool bk_enabled() {
    const char *e = getenv("PAULIPROP_WINDOW1_PATH");
    return !(e && strcmp(e, "tiles") == 0);
}

// Compiled variants of k_bk_rotate: (bucket capacity, staged items per thread).
typedef void (*BkKernel)(BkArgs, int);
struct BkVariant {
    int cap, items;
    BkKernel k1, k2, kb;            // one- and two-word keys; batched instances (two-word)
    size_t smem1, smem2;
};

#define PP_BK_VARIANT(C, I)                                                                                 \
    { C, I, k_bk_rotate<1, C, I>, k_bk_rotate<2, C, I>, k_bk_rotate<2, C, I, true>, bk_smem_bytes<1, C, I>(),     \
      bk_smem_bytes<2, C, I>() }
static const BkVariant BK_VARIANTS[] = {PP_BK_VARIANT(128, 4), PP_BK_VARIANT(256, 4), PP_BK_VARIANT(512, 4),
                                        PP_BK_VARIANT(256, 8), PP_BK_VARIANT(512, 8), PP_BK_VARIANT(1024, 8)};
static constexpr int BK_NVAR = sizeof(BK_VARIANTS) / sizeof(BK_VARIANTS[0]);
#undef PP_BK_VARIANT

static const BkVariant *bk_variant(int cap, int items) {
    for (const BkVariant &v : BK_VARIANTS)
        if (v.cap == cap && v.items == items) return &v;
    return nullptr;
}

template <int NW>
static void bk_launch(pp_spv *h, const BkVariant *v, const BkArgs &A, int k) {
    // persistent grid: every resident CTA, or one per bucket pair (the kernel sizes its groups)
    const long long pairs = 1ll << (A.bits - 1);
    const auto &oc = h->bk_occ[v - BK_VARIANTS];
    const bool batch = NW == 2 && h->batch_on;
    const int occ = NW == 1 ? oc.occ1 : batch ? oc.occb : oc.occ2;
    const int grid = (int)std::min(pairs, (long long)h->nsm * occ);
    // programmatic dependent launch: the rotation's prologue overlaps the previous
    // rotation's tail (k_bk_rotate waits for its outputs in griddepcontrol.wait)
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(BK_THREADS);
    cfg.dynamicSmemBytes = NW == 1 ? v->smem1 : v->smem2;
    cfg.stream = h->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, NW == 1 ? v->k1 : batch ? v->kb : v->k2, A, k);
}

// Hash rows: fixed pseudo-random words (splitmix64 from a fixed seed), so the
// bucket of a key never depends on the call.
static void bk_rows_host(u64 *rows) {
    unsigned long long s = 0x5EEDB0C4E7ull;
    for (int i = 0; i < BK_ROWS * 4; ++i) {
        s += 0x9E3779B97F4A7C15ull;
        unsigned long long z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        rows[i] = z ^ (z >> 31);
    }
}

static int bk_rows_init(pp_spv *h) {
    if (h->bk_rows) return PP_OK;
    u64 rows[BK_ROWS * 4];
    bk_rows_host(rows);
    u64 *dr = nullptr;
    int *da = nullptr;
    TRY(dalloc(h, &dr, BK_ROWS * 4));
    int r = dalloc(h, &da, 2);
    if (r) { dfree(h, dr); return r; }
    h->bk_rows = dr;
    h->bk_aux = da;
    CU(cudaMemcpyAsync(h->bk_rows, rows, sizeof rows, cudaMemcpyHostToDevice, h->stream));
    for (int i = 0; i < BK_NVAR; ++i) {
        const BkVariant &v = BK_VARIANTS[i];
        CU(cudaFuncSetAttribute(v.k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem1));
        CU(cudaFuncSetAttribute(v.k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem2));
        CU(cudaFuncSetAttribute(v.k1, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared));
        CU(cudaFuncSetAttribute(v.k2, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared));
        int o = 0;
        CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, v.k1, BK_THREADS, v.smem1));
        h->bk_occ[i].occ1 = std::max(1, o);
        CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, v.k2, BK_THREADS, v.smem2));
        h->bk_occ[i].occ2 = std::max(1, o);
        CU(cudaFuncSetAttribute(v.kb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)v.smem2));
        CU(cudaFuncSetAttribute(v.kb, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared));
        CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, v.kb, BK_THREADS, v.smem2));
        h->bk_occ[i].occb = std::max(1, o);
    }
    return sync_check(h);
}

// Smallest bucket count for n terms at a mean load of at most cap / load_div.
static int bk_bits_for(long long n, int cap, int load_div) {
    int b = 1;
    while (b < BK_ROWS && ((long long)cap << b) < (long long)load_div * n) ++b;
    return b;
}

static BkArgs bk_args(pp_spv *h, const BkVariant *v, int bits, BkRec *rec) {
    BkArgs A;
    memset(&A, 0, sizeof A);
    for (int s = 0; s < 2; ++s) { A.z[s] = h->bkz[s]; A.x[s] = h->bkx[s]; A.c[s] = h->bkc[s]; A.cnt[s] = h->bkcnt[s]; }
    A.bits = bits;
    A.bits_cap = h->bk_bits_cap;
    A.rec_len = h->bk_rec_cap;
    A.rows = h->bk_rows;
    A.rec = rec;
    A.S = h->S;
    A.P = h->P;
    A.gens = h->gens;
    A.pref_forced = -1;
    if (h->batch_on) {
        A.bcos = h->bcos;
        A.bsin = h->bsin;
        A.bend = h->bend;
        A.ninst = h->ninst;
        A.ncol = h->ncol;
    }
    return A;
}

// Scatters (SZ, SX, SC) -- dense n terms, or the bucket set `from` of 2^sbits
// buckets -- into bucket set `to` with 2^bits buckets.  Returns the largest
// bucket count in *maxcnt, or -1 if a bucket overflowed.
template <int NW>
static int bk_scatter(pp_spv *h, const u64 *SZ, const u64 *SX, const double *SC, long long n, int from, int sbits,
                      int to, int bits, int *maxcnt) {
    cudaStream_t s = h->stream;
    const int cap = h->bk_cap;
    CU(cudaMemsetAsync(h->bkcnt[to], 0, sizeof(int) << bits, s));
    CU(cudaMemsetAsync(h->bk_aux, 0, 2 * sizeof(int), s));
    const long long slots = from >= 0 ? ((long long)cap << sbits) : n;
    const int grid = (int)std::max(1ll, std::min((slots + 255) / 256, (long long)h->nsm * 16));
    k_bk_scatter<NW><<<grid, 256, 0, s>>>(SZ, SX, SC, n, from >= 0 ? h->bkcnt[from] : nullptr, sbits, h->bkz[to],
                                          h->bkx[to], h->bkc[to], h->bkcnt[to], bits, cap, h->bk_rows, h->bk_aux,
                                          h->bk_aux + 1);
    int aux[2] = {0, 0};
    CU(cudaMemcpyAsync(aux, h->bk_aux, sizeof aux, cudaMemcpyDeviceToHost, s));
    TRY(sync_check(h));
    *maxcnt = (aux[1] & ERR_OVERFLOW) ? -1 : aux[0];
    return PP_OK;
}

// Bucket sets for 2^bits buckets of the tuned capacity.  Growing the allocation
// moves the live bucket set `*cur` (of 2^cur_bits buckets; cur_bits < 0: none)
// into the new set 0.  Every buffer is allocated before the old ones are freed.
template <int NW>
static int bk_reserve(pp_spv *h, int bits, int *cur, int cur_bits) {
    if (bits <= h->bk_bits_cap && h->bk_cap == h->tune.bucket_cap) return PP_OK;
    if (cur_bits >= 0 && h->bk_cap != h->tune.bucket_cap)
        return fail(PP_ERROR_EXCEPTION, "internal error: bucket capacity changed inside a call");
    const int cap = h->tune.bucket_cap;
    // the two bucket sets, and room to convert a full layout (at most slots / 2
    // terms before the next split) back to a dense sorted set, plus 4 GiB; one
    // split of headroom (2^(bits+1) buckets) when that fits, else 2^bits
    auto fits = [&](long long sl) {
        size_t freeb = 0, totalb = 0;
        if (cudaMemGetInfo(&freeb, &totalb) == cudaSuccess) {
            const double B = 16.0 * NW + 8.0;
            if (3.5 * (double)sl * B + 4.0 * (1ull << 30) > (double)freeb) return false;
        }
        const long long lim = g_bk_slot_limit.load();
        return !(lim > 0 && sl > lim);
    };
    int nbits = std::min(BK_ROWS, std::max(bits + 1, h->bk_cap == cap ? h->bk_bits_cap : 0));
    if (!fits((long long)cap << nbits)) nbits = bits;
    if (!fits((long long)cap << nbits)) return BK_NOFIT;
    const long long slots = (long long)cap << nbits;
    u64 *nz[2] = {nullptr, nullptr}, *nx[2] = {nullptr, nullptr};
    double *nc[2] = {nullptr, nullptr};
    int *nn[2] = {nullptr, nullptr};
    long long *noff = nullptr;
    auto drop = [&]() {
        for (int q = 0; q < 2; ++q) { dfree(h, nz[q]); dfree(h, nx[q]); dfree(h, nc[q]); dfree(h, nn[q]); }
        dfree(h, noff);
    };
    int r = 0;
    for (int q = 0; q < 2 && !r; ++q) {
        r = dalloc(h, &nz[q], slots * NW);
        if (!r) r = dalloc(h, &nx[q], slots * NW);
        if (!r) r = dalloc(h, &nc[q], slots);
        if (!r) r = dalloc(h, &nn[q], 1ll << nbits);
    }
    if (!r) r = dalloc(h, &noff, (1ll << nbits) + 1);
    if (r) { drop(); return r; }
    if (cur_bits >= 0 && h->bk_bits_cap >= 0) {
        // the live bucket set keeps its layout: copy it into new set 0
        const long long os = (long long)h->bk_cap << cur_bits;
        cudaStream_t s = h->stream;
        cudaError_t e = cudaMemcpyAsync(nz[0], h->bkz[*cur], os * NW * 8, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(nx[0], h->bkx[*cur], os * NW * 8, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(nc[0], h->bkc[*cur], os * 8, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(nn[0], h->bkcnt[*cur], sizeof(int) << cur_bits, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) { drop(); return fail(PP_DEVICE_ERROR, cudaGetErrorString(e)); }
        *cur = 0;
    }
    for (int q = 0; q < 2; ++q) {
        dfree(h, h->bkz[q]); dfree(h, h->bkx[q]); dfree(h, h->bkc[q]); dfree(h, h->bkcnt[q]);
        h->bkz[q] = nz[q]; h->bkx[q] = nx[q]; h->bkc[q] = nc[q]; h->bkcnt[q] = nn[q];
    }
    dfree(h, h->bk_off);
    h->bk_off = noff;
    h->bk_bits_cap = nbits;
    h->bk_cap = cap;
    return PP_OK;
}

// Frees the bucket sets (the live set is dense again).
static void bk_release(pp_spv *h) {
    for (int q = 0; q < 2; ++q) {
        dfree(h, h->bkz[q]); dfree(h, h->bkx[q]); dfree(h, h->bkc[q]); dfree(h, h->bkcnt[q]);
        h->bkz[q] = h->bkx[q] = nullptr;
        h->bkc[q] = nullptr;
        h->bkcnt[q] = nullptr;
    }
    dfree(h, h->bk_off);
    h->bk_off = nullptr;
    h->bk_bits_cap = -1;
    for (int q = 0; q < 2; ++q) { dfree(h, h->bkfcnt[q]); h->bkfcnt[q] = nullptr; }
    h->bkfcnt_bits = -1;
    h->buf_gen++;
}

// Moves the live bucket set *cur (2^*bits buckets) to a layout with more
// buckets, doubling until the largest bucket holds at most half its capacity
// (then no bucket of the next rotation's output can overflow).
template <int NW>
static int bk_regrid(pp_spv *h, int *cur, int *bits) {
    int nbits = *bits;
    for (;;) {
        if (nbits + 1 > BK_ROWS) return fail(PP_OUT_OF_MEMORY, "bucketed live set exceeds 2^26 buckets");
        ++nbits;
        TRY(bk_reserve<NW>(h, nbits, cur, *bits));
        int mx = 0;
        TRY(bk_scatter<NW>(h, h->bkz[*cur], h->bkx[*cur], h->bkc[*cur], 0, *cur, *bits, *cur ^ 1, nbits, &mx));
        if (mx >= 0 && mx <= h->bk_cap / 2) break;
    }
    *cur ^= 1;
    *bits = nbits;
    return PP_OK;
}

// Graph of `len` consecutive k_bk_rotate launches over 2^bits buckets.
template <int NW>
static int bk_graph(pp_spv *h, const BkVariant *v, int bits, int cls, int len, cudaGraphExec_t *out) {
    if (h->bk_graph_gen != h->buf_gen) {
        for (auto &kv : h->bk_graphs) cudaGraphExecDestroy(kv.second);
        h->bk_graphs.clear();
        h->bk_graph_gen = h->buf_gen;
    }
    const int key = bits * 4 + cls;
    auto it = h->bk_graphs.find(key);
    if (it != h->bk_graphs.end()) { *out = it->second; return PP_OK; }
    const BkArgs A = bk_args(h, v, bits, h->bk_rec);
    cudaGraph_t graph = nullptr;
    CU(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < len; ++k) bk_launch<NW>(h, v, A, k);
    CU(cudaStreamEndCapture(h->stream, &graph));
    cudaGraphExec_t ex = nullptr;
    cudaError_t e = cudaGraphInstantiate(&ex, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(PP_DEVICE_ERROR, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    h->bk_graphs[key] = ex;
    *out = ex;
    return PP_OK;
}

// Gathers the bucket set `cur` (2^bits buckets) into live set 0 and
// radix-sorts it: the live set is dense and sorted again.  Every allocation
// comes first, so a failure leaves the dense live set as it was.
template <int NW>
static int bk_to_dense(pp_spv *h, int cur, int bits) {
    const int nb = 1 << bits;
    cudaStream_t s = h->stream;
    k_bk_offsets<<<1, BKS_THREADS, 0, s>>>(h->bkcnt[cur], nb, h->bk_cap, h->bk_off);
    long long n = 0;
    CU(cudaMemcpyAsync(&n, h->bk_off + nb, sizeof n, cudaMemcpyDeviceToHost, s));
    TRY(sync_check(h));
    PP_TRACE("buckets -> dense: %lld terms (2^%d buckets)", n, bits);
    TRY(radix_reserve(h, n));
    TRY(ensure_live(h, n + 1, false));
    k_bk_gather<NW><<<std::max(1, std::min(h->nsm * 8, (nb + 7) / 8)), 256, 0, s>>>(
        h->bkz[cur], h->bkx[cur], h->bkc[cur], h->bkcnt[cur], nb, h->bk_cap, h->bk_off, h->z[0], h->x[0], h->c[0],
        h->cap, h->S);
    TRY(sync_check(h));
    int in_t = 0;
    TRY(radix_sort<NW>(h, h->z[0], h->x[0], h->c[0], h->z[1], h->x[1], h->c[1], n, &in_t));
    DevState st;
    TRY(read_state(h, &st));
    st.n = n;
    st.cur = in_t;
    st.seg_dense = 1;
    TRY(write_state(h, &st));
    return PP_OK;
}

// The window-1 sequence [start, L) on buckets.  The device cursor is at start.
// per_rot: per-rotation times were asked for (each launch bracketed by events,
// no graphs); otherwise the rotations replay from captured graphs, and a
// profiled call (prof->on) times each graph replay.
template <int NW>
static int run_bucket(pp_spv *h, long long start, long long L, pp_counters *ctr, RunProf *prof, bool per_rot) {
    TRY(ensure_dense(h));
    TRY(bk_rows_init(h));
    const BkVariant *var = bk_variant(h->tune.bucket_cap, h->tune.items_per_thread);
    if (!var) return fail(PP_ERROR_EXCEPTION, "internal error: no compiled bucket variant for the tuning");
    DevState st;
    TRY(read_state(h, &st));
    const long long n0 = st.n;
    // per-rotation records rec[start .. L]
    if (L + 1 > h->bk_rec_cap) {
        TRY(dalloc(h, &h->bk_rec, L + 1));
        h->bk_rec_cap = L + 1;
    }
    {
        BkRec r0;
        memset(&r0, 0, sizeof r0);
        r0.n_in = n0;
        r0.n_out = (unsigned long long)n0;
        r0.acap = st.acap_logical;
        CU(cudaMemcpyAsync(h->bk_rec + start, &r0, sizeof r0, cudaMemcpyHostToDevice, h->stream));
        CU(cudaMemsetAsync(h->bk_rec + start + 1, 0, (L - start) * sizeof(BkRec), h->stream));
    }
    // bucket the live set
    int bits = bk_bits_for(n0, h->tune.bucket_cap, h->tune.load_div), cur = 0;
    PP_TRACE("buckets: rotations [%lld, %lld), %lld live terms, 2^%d buckets of %d", start, L, n0, bits,
             h->tune.bucket_cap);
    // (when that layout does not fit, fewer and fuller buckets down to a mean load
    // of cap / 3, as long as no bucket is more than half full)
    const int bmin = bk_bits_for(n0, h->tune.bucket_cap, 3);
    bool lowered = false;
    for (;;) {
        const int rr = bk_reserve<NW>(h, bits, &cur, -1);
        if (rr == BK_NOFIT && bits > bmin) {
            --bits;
            lowered = true;
            continue;
        }
        if (rr) return rr;                  // BK_NOFIT: nothing changed, the dense set is the input
        int mx = 0;
        TRY(bk_scatter<NW>(h, h->z[st.cur], h->x[st.cur], h->c[st.cur], n0, -1, 0, 0, bits, &mx));
        if (mx >= 0 && mx <= h->bk_cap / 2) break;
        if (lowered) return BK_NOFIT;       // the fuller layout fails the half-full rule, a larger one does not fit
        if (++bits > BK_ROWS) return fail(PP_OUT_OF_MEMORY, "bucketed live set exceeds 2^26 buckets");
    }
    cudaStream_t s = h->stream;
    // totals and counters of rotations [start, upto) into the device state, and the
    // live set (bucket set cur) back to the dense sorted layout
    auto finish = [&](long long upto) -> int {
        std::vector<BkRec> rec((size_t)(upto - start + 1));
        CU(cudaMemcpyAsync(rec.data(), h->bk_rec + start, rec.size() * sizeof(BkRec), cudaMemcpyDeviceToHost, s));
        TRY(sync_check(h));
        TRY(read_state(h, &st));
        std::vector<long long> rr;
        if (h->rec_on) rr.assign((size_t)(4 * (upto - start)), 0);
        for (long long r = start; r < upto; ++r) {
            const BkRec &o = rec[(size_t)(r - start + 1)];
            const long long n = o.n_in, a = (long long)o.created, tot = (long long)o.n_out, np = (long long)o.np;
            st.live_in += n;
            st.created += a;
            st.merge_in += n + a;
            st.merge_out += tot;
            if (tot > st.peak) st.peak = tot;
            if (o.pref) st.early += 1;
            prof->bk_rot += 1;
            prof->bk_bytes += (double)(16 * NW + 8) * (double)(n + tot);
            if (h->rec_on) {
                // WindowCounters of the rotation (window = 1): an early boundary merges
                // n -> np first, the regular one np + a -> total
                long long *q = &rr[(size_t)(4 * (r - start))];
                q[0] = a;
                q[1] = (o.pref ? n + np : n) + a;
                q[2] = (o.pref ? np : 0) + tot;
                q[3] = o.pref ? 1 : 0;
            }
        }
        if (h->rec_on && upto > start)
            CU(cudaMemcpy(h->rec + 4 * start, rr.data(), rr.size() * sizeof(long long), cudaMemcpyHostToDevice));
        {
            // the early-merge capacity rule after the last rotation (as k_bk_rotate applies it)
            const BkRec &o = rec.back();
            long long acap = o.acap;
            if (o.pref && (long long)o.np > acap) acap = std::max(2 * acap, (long long)o.np);
            st.acap_logical = acap;
        }
        st.rot = upto;
        TRY(write_state(h, &st));
        return bk_to_dense<NW>(h, cur, bits);
    };
    cur = 0;
    long long done = start;
    const int chunk = h->tune.chunk;
    std::vector<cudaEvent_t> gev;      // event pairs around the graph replays of a chunk (profiled calls)
    struct GevGuard {
        std::vector<cudaEvent_t> &v;
        ~GevGuard() { for (auto e : v) cudaEventDestroy(e); }
    } gevg{gev};
    while (done < L) {
        const long long len = std::min((long long)chunk, L - done);
        if (bits < 1 || bits > h->bk_bits_cap || h->bk_cap != var->cap || L + 1 > h->bk_rec_cap || (cur & ~1))
            return fail(PP_ERROR_EXCEPTION, "internal error: inconsistent bucket layout before a launch");
        k_bk_begin<<<1, 1, 0, s>>>(h->S, done, cur, 1);
        prof->launches += 1;
        int ngraph = 0;
        if (!per_rot) {
            long long r = 0;
            while (r < len) {
                const int cls = (len - r >= chunk) ? 0 : (len - r >= 8) ? 1 : 2;
                const int cl = cls == 0 ? chunk : cls == 1 ? 8 : 1;
                if (r > 0) {
                    // a later graph of the chunk starts at rotation done + r
                    k_bk_begin<<<1, 1, 0, s>>>(h->S, done + r, (cur + (int)r) & 1, 0);
                    prof->launches += 1;
                }
                cudaGraphExec_t ex = nullptr;
                TRY(bk_graph<NW>(h, var, bits, cls, cl, &ex));
                if (prof->on) {
                    while ((int)gev.size() < 2 * (ngraph + 1)) {
                        cudaEvent_t e;
                        CU(cudaEventCreate(&e));
                        gev.push_back(e);
                    }
                    CU(cudaEventRecord(gev[2 * ngraph], s));
                }
                CU(cudaGraphLaunch(ex, s));
                if (prof->on) CU(cudaEventRecord(gev[2 * ngraph++ + 1], s));
                prof->launches += cl;
                r += cl;
            }
        } else {
            const BkArgs A = bk_args(h, var, bits, h->bk_rec);
            for (long long k = 0; k < len; ++k) {
                cudaEvent_t e0, e1;
                cudaEventCreate(&e0);
                cudaEventCreate(&e1);
                cudaEventRecord(e0, s);
                bk_launch<NW>(h, var, A, (int)k);
                cudaEventRecord(e1, s);
                TRY(sync_check(h));
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                cudaEventDestroy(e0);
                cudaEventDestroy(e1);
                const long long r = done + k;
                prof->t_merge += ms * 1e-3;
                prof->launches += 1;
                if (ctr && r < ctr->nwin && ctr->t_merge) ctr->t_merge[r] += ms * 1e-3;
            }
        }
        TRY(sync_check(h));
        for (int q = 0; q < ngraph; ++q) {
            float ms = 0.f;
            CU(cudaEventElapsedTime(&ms, gev[2 * q], gev[2 * q + 1]));
            prof->t_merge += ms * 1e-3;
        }
        TRY(read_state(h, &st));
        if (st.err & ~ERR_OVERFLOW) return check_err(h, st);   // the dense live set is the sequence's input
        const long long completed = (st.err & ERR_OVERFLOW) ? std::max(0ll, std::min(len, st.bk_fail - done)) : len;
        cur = (cur + (int)(completed & 1)) & 1;
        done += completed;
        BkRec last;
        CU(cudaMemcpyAsync(&last, h->bk_rec + done, sizeof last, cudaMemcpyDeviceToHost, s));
        TRY(sync_check(h));
        const bool over = (st.err & ERR_OVERFLOW) != 0;
        if (over) {
            st.err &= ~ERR_OVERFLOW;
            TRY(write_state(h, &st));
            CU(cudaMemsetAsync(h->bk_rec + done + 1, 0, sizeof(BkRec), s));
        }
        if (done < L && (over || last.maxcnt > h->bk_cap / 2)) {
            const int rr = bk_regrid<NW>(h, &cur, &bits);
            PP_TRACE("buckets: split at rotation %lld (largest bucket %d) -> 2^%d buckets%s", done, last.maxcnt, bits,
                     rr == BK_NOFIT ? ": does not fit, hand-over to the sorted-merge kernels" : "");
            if (rr == BK_NOFIT) {
                // no room for a larger layout: the rotations so far go back to the
                // dense sorted set, the bucket sets are freed, and the sorted-merge
                // kernels take the rest of the sequence
                TRY(finish(done));
                bk_release(h);
                return BK_NOFIT;
            }
            if (rr) return rr;
        }
    }
    TRY(finish(L));
    if (h->batch_on) return PP_OK;      // batched instances are measured per instance at their ends
    // <ket|O|ket> after the last rotation (GEN_MEASURE), on the sorted live set
    double ev = 0.0;
    TRY(expect_dev(h, h->Ph->ket, &ev));
    TRY(read_state(h, &st));
    st.expect_val = ev;
    st.measure_valid = 1;
    TRY(write_state(h, &st));
    return PP_OK;
}

// Structured window-1 sequence over rotations [start, L) (the device cursor
// S->rot is at start): chunks of CHUNK_ROT rotations between state read-backs; on
// ERR_OVERFLOW grow and resume at the rotation that stopped.  While the live set
// fits k_small_run's shared memory (and the call has no local truncation,
// correction or batched instances, and no per-rotation timing), one launch of it
// runs the rotations instead.
template <int NW>
static int run_struct(pp_spv *h, long long start, long long L, pp_counters *ctr, RunProf *prof, long long n_known = -1) {
    long long done = start;
    const bool per_rot = ctr && (ctr->t_rotate || ctr->t_merge);   // per-rotation times asked for
    const bool timed = prof->on || per_rot;
    std::vector<cudaEvent_t> ev;   // 5 per rotation when timed
    bool table = false;            // the device segment table describes the (dense) live set
    const bool small_ok = !per_rot && !h->batch_on && !h->Ph->local_active && h->Ph->corr_kind == 0;
    bool use_bk = bk_enabled() && h->Ph->corr_kind == 0;
    long long ncur = small_cap<NW>() + 1;   // live terms at the chunk's start (read when small_ok)
    bool dense = false;                      // the last state read showed a dense live set
    if (small_ok) {
        if (n_known >= 0) {
            ncur = n_known;
        } else {
            DevState st;
            TRY(read_state(h, &st));
            ncur = st.n;
        }
    }
    while (done < L) {
        if (small_ok && ncur <= small_cap<NW>()) {
            Bufs B = make_bufs(h);
            k_small_run<NW><<<1, SM_THREADS, small_smem<NW>(), h->stream>>>(B);
            prof->launches += 1;
            TRY(sync_check(h));
            DevState st;
            TRY(read_state(h, &st));
            if (st.err) { ensure_dense(h); return check_err(h, st); }
            table = false;
            ncur = st.n;
            dense = st.seg_dense != 0;
            if (st.rot == done) ncur = small_cap<NW>() + 1;   // no progress: leave it to the multi-kernel path
            done = st.rot;
            continue;
        }
        if (use_bk && L - done >= BK_MIN_ROT) {
            const int rb = run_bucket<NW>(h, done, L, ctr, prof, per_rot);
            if (rb != BK_NOFIT) return rb;
            bk_release(h);                  // their memory goes to the sorted-merge kernels
            PP_TRACE("buckets do not fit at rotation %lld: sorted-merge kernels for the rest of the call", done);
            // no room for buckets: the rest of the sequence on the sorted-merge kernels,
            // from the rotation the bucketed part reached
            use_bk = false;
            table = false;
            DevState st;
            TRY(read_state(h, &st));
            done = st.rot;
            ncur = small_ok ? st.n : small_cap<NW>() + 1;
            continue;
        }
        dense = false;                       // the merge kernels leave a segment table
        Bufs B = make_bufs(h);
        const long long end = std::min(L, done + CHUNK_ROT);
        cudaStream_t s = h->stream;
        if (!table) {
            k_segdense<<<h->nsm, 256, 0, s>>>(B);
            prof->launches += 1;
            table = true;
        }
        if (!timed) {
            // replay captured chunks: CHUNK_ROT, then 8, then single rotations
            long long r = done;
            while (r < end) {
                const int gi = (end - r >= CHUNK_ROT) ? 0 : (end - r >= 8) ? 1 : 2;
                const int len = gi == 0 ? CHUNK_ROT : gi == 1 ? 8 : 1;
                TRY(struct_graph<NW>(h, gi, len));
                CU(cudaGraphLaunch(h->gexec[gi], s));
                r += len;
                prof->launches += 6 * len;
            }
        }
        for (long long r = done; r < end && timed; ++r) {
            {
                cudaEvent_t e[5];
                for (int q = 0; q < 5; ++q) cudaEventCreate(&e[q]);
                cudaEventRecord(e[0], s);
                k_classify<NW><<<h->nsm * h->occA1, A_THREADS, 2 * NW * A_TILE * 8 + A_TILE, s>>>(B);
                k_tilescan<NW><<<1, S_THREADS, tilescan_smem<NW>(), s>>>(B);
                k_permute<NW><<<h->nsm * h->occA3, A_THREADS, 0, s>>>(B);
                cudaEventRecord(e[1], s);
                k_partition<NW, 0><<<h->nsm * 4, P_THREADS, 0, s>>>(B);
                cudaEventRecord(e[2], s);
                k_merge<NW, 0><<<h->nsm * h->occB, B_THREADS, merge_smem_bytes<NW>(), s>>>(B, 0);
                cudaEventRecord(e[3], s);
                k_commit<0><<<1, 256, 0, s>>>(B, 0);
                cudaEventRecord(e[4], s);
                for (int q = 0; q < 5; ++q) ev.push_back(e[q]);
            }
            prof->launches += 6;
        }
        TRY(sync_check(h));
        DevState st;
        TRY(read_state(h, &st));
        ncur = st.n;
        if (timed) {
            // rotations that ran are [done, st.rot); the rest were no-ops
            const long long base = (long long)ev.size() / 5 - (end - done);
            for (long long r = done; r < end; ++r) {
                cudaEvent_t *e = &ev[(base + (r - done)) * 5];
                if (r < st.rot) {
                    float a = 0, b = 0, c = 0, d = 0;
                    cudaEventElapsedTime(&a, e[0], e[1]);
                    cudaEventElapsedTime(&b, e[1], e[2]);
                    cudaEventElapsedTime(&c, e[2], e[3]);
                    cudaEventElapsedTime(&d, e[3], e[4]);
                    prof->t_rotate += a * 1e-3;
                    prof->t_partition += (b + d) * 1e-3;
                    prof->t_merge += c * 1e-3;
                    if (ctr && r < ctr->nwin) {
                        if (ctr->t_rotate) ctr->t_rotate[r] += a * 1e-3;
                        if (ctr->t_merge) ctr->t_merge[r] += (b + c + d) * 1e-3;
                    }
                }
                for (int q = 0; q < 5; ++q) cudaEventDestroy(e[q]);
            }
            ev.clear();
        }
        if (st.err & ERR_OVERFLOW) {
            st.err &= ~ERR_OVERFLOW;
            TRY(write_state(h, &st));
            TRY(ensure_live(h, std::max(st.need + st.need / 2, 3 * st.n)));
            table = false;
            done = st.rot;
            continue;
        }
        if (st.err) { ensure_dense(h); return check_err(h, st); }
        done = st.rot;
        // grow ahead of time: the merge's per-tile output slots need ~1.25 (n + a) <= 2.5 n
        // (3 n required, 6 n preferred while device memory allows)
        if (done < L && 3 * st.n > h->cap) {
            TRY(ensure_live(h, 3 * st.n, true, 6 * st.n));
            table = false;
        }
    }
    return dense ? PP_OK : ensure_dense(h);
}

// General path boundary: sort pending appends, merge (MODE 1).
template <int NW>
static int general_boundary(pp_spv *h, int flags, long long *n_in, long long *n_out) {
    DevState st;
    TRY(read_state(h, &st));
    const long long an = st.an;
    *n_in = st.n + an;
    TRY(ensure_live(h, st.n + an));
    TRY(read_state(h, &st));
    Bufs B = make_bufs(h);
    if (an > 0) {
        int in_t = 0;
        TRY(ensure_append(h, h->acap_phys, an));
        TRY(radix_sort<NW>(h, h->az, h->ax, h->ac, h->tz, h->tx, h->tc, an, &in_t));
        B = make_bufs(h);
        if (in_t) { B.vz = h->tz; B.vx = h->tx; B.vc = h->tc; }
    }
    launch_merge<NW, 1>(h, B, flags);
    TRY(sync_check(h));
    TRY(read_state(h, &st));
    TRY(check_err(h, st));
    *n_out = st.n;
    return PP_OK;
}

// <ket|O|ket> of the live set (the reduction of pp_expect_ket).
static int expect_dev(pp_spv *h, const u64 *k, double *out) {
    Bufs B = make_bufs(h);
    const int nb = std::min(4096, h->nsm * 8);
    if (h->NW == 1) k_expect<1><<<nb, 256, 0, h->stream>>>(B, k[0], k[1], h->epart);
    else k_expect<2><<<nb, 256, 0, h->stream>>>(B, k[0], k[1], h->epart);
    k_expect_final<<<1, 32, 0, h->stream>>>(h->epart, nb, h->eout);
    CU(cudaMemcpyAsync(out, h->eout, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    return sync_check(h);
}

// _apply!(v, ::AdaptiveTruncation) (spv_evolve.jl:103-114): with n > max_terms the
// clip threshold is the (max_terms + 1)-th largest |c| -- coeffs[end - max_terms]
// of the ascending sort -- found exactly by a radix select on the device;
// otherwise min_thresh.  Then coeff_clip! (drop |c| <= thresh, order kept).
static int adaptive_apply(pp_spv *h, long long max_terms, double min_thresh) {
    DevState st;
    TRY(read_state(h, &st));
    double thr = min_thresh;
    if (st.n > max_terms) {
        if (!h->sel64) TRY(dalloc(h, &h->sel64, 1));
        Select64 s0;
        memset(&s0, 0, sizeof s0);
        s0.remaining = max_terms + 1;
        CU(cudaMemcpyAsync(h->sel64, &s0, sizeof s0, cudaMemcpyHostToDevice, h->stream));
        const double *C = h->c[st.cur];
        for (int shift = 56; shift >= 0; shift -= 8) {
            k_abs_hist<<<h->nsm * 4, 256, 0, h->stream>>>(C, st.n, h->sel64, shift);
            k_sel64_pick<<<1, 32, 0, h->stream>>>(h->sel64, shift);
        }
        Select64 sf;
        CU(cudaMemcpyAsync(&sf, h->sel64, sizeof sf, cudaMemcpyDeviceToHost, h->stream));
        TRY(sync_check(h));
        memcpy(&thr, &sf.prefix, sizeof thr);
    }
    pp_filter f = NOFILTER_H;
    f.thresh = thr;
    compile_filter(&f, &h->Ph->clip);
    TRY(upload_params(h));
    TRY(read_state(h, &st));
    st.an = 0;
    TRY(write_state(h, &st));
    Bufs B = make_bufs(h);
    if (h->NW == 1) launch_merge<1, 2>(h, B, 0);
    else launch_merge<2, 2>(h, B, 0);
    TRY(sync_check(h));
    TRY(read_state(h, &st));
    return check_err(h, st);
}

// variance(O, ψ) of the live set (statistics.jl:6-22; see k_var_records).
template <int NW>
static int variance_nw(pp_spv *h, const u64 *ket, double *out) {
    DevState st;
    TRY(read_state(h, &st));
    const long long n = st.n;
    *out = 0.0;
    if (n == 0) return PP_OK;
    if (!h->vtmp) TRY(dalloc(h, &h->vtmp, 2));
    TRY(ensure_append(h, std::max(n, h->acap_phys), 0));
    Bufs B = make_bufs(h);
    cudaStream_t s = h->stream;
    k_var_records<NW><<<h->nsm * 8, 256, 0, s>>>(B, ket[0], ket[1], h->az, h->ax, h->ac);
    int in_t = 0;
    TRY(radix_sort<NW>(h, h->az, h->ax, h->ac, h->tz, h->tx, h->tc, n, &in_t));
    const u64 *RZ = in_t ? h->tz : h->az, *RX = in_t ? h->tx : h->ax;
    const double *RC = in_t ? h->tc : h->ac;
    double *gval = in_t ? h->ac : h->tc;
    CU(cudaMemsetAsync(h->vtmp, 0, 2 * sizeof(double), s));
    k_var_groups<NW><<<h->nsm * 8, 256, 0, s>>>(RZ, RX, RC, n, gval, h->vtmp);
    const int nb = std::min(4096, h->nsm * 8);
    k_sum_partials<<<nb, 256, 0, s>>>(gval, n, h->epart);
    k_expect_final<<<1, 32, 0, s>>>(h->epart, nb, h->eout);
    double e2 = 0.0, e1 = 0.0;
    CU(cudaMemcpyAsync(&e2, h->eout, sizeof(double), cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(&e1, h->vtmp, sizeof(double), cudaMemcpyDeviceToHost, s));
    TRY(sync_check(h));
    *out = e2 - e1 * e1;
    return PP_OK;
}

static int variance_dev(pp_spv *h, const u64 *ket, double *out) {
    return h->NW == 1 ? variance_nw<1>(h, ket, out) : variance_nw<2>(h, ket, out);
}

// Device scratch of one stochastic truncation call (freed on return).
struct Scratch {
    std::vector<void *> p;
    ~Scratch() { for (void *q : p) cudaFree(q); }
    template <typename T>
    int get(T **out, long long count) {
        void *q = nullptr;
        if (cudaMalloc(&q, (size_t)std::max(1ll, count) * sizeof(T)) != cudaSuccess) {
            cudaGetLastError();
            return fail(PP_OUT_OF_MEMORY, "cudaMalloc (scratch buffer)");
        }
        p.push_back(q);
        *out = (T *)q;
        return PP_OK;
    }
};

// Commits an order-preserving flag compaction of the live set into the other set.
static int flag_compact(pp_spv *h, DevState &st, const unsigned char *keep, const double *nc, const double *scale,
                        Scratch &sc) {
    const long long n = st.n;
    const long long ntiles = (n + FC_TILE - 1) / FC_TILE;
    int *cnt, *off;
    long long *total;
    TRY(sc.get(&cnt, ntiles));
    TRY(sc.get(&off, ntiles));
    TRY(sc.get(&total, 1));
    cudaStream_t s = h->stream;
    const int cur = st.cur;
    const int g = (int)std::min<long long>(ntiles, 8ll * h->nsm);
    k_flag_count<<<g, FC_THREADS, 0, s>>>(keep, n, cnt);
    k_flag_scan<<<1, 1024, 0, s>>>(ntiles, cnt, off, total);
    k_flag_write<<<g, FC_THREADS, 0, s>>>(keep, n, off, h->z[cur], h->x[cur], h->c[cur], nc, h->NW, scale,
                                          h->z[cur ^ 1], h->x[cur ^ 1], h->c[cur ^ 1]);
    long long kept = 0;
    CU(cudaMemcpyAsync(&kept, total, sizeof kept, cudaMemcpyDeviceToHost, s));
    TRY(sync_check(h));
    TRY(read_state(h, &st));
    st.n = kept;
    st.cur ^= 1;
    return write_state(h, &st);
}

// stochastic_clip!(v, eps) (spv_evolve.jl:35-52) with the counter-based generator.
static int stoch_clip_apply(pp_spv *h, double eps, unsigned long long seed) {
    DevState st;
    TRY(read_state(h, &st));
    const long long n = st.n;
    if (n == 0) return PP_OK;
    Scratch sc;
    unsigned char *keep;
    double *nc;
    TRY(sc.get(&keep, n));
    TRY(sc.get(&nc, n));
    k_stoch_clip_mark<<<h->nsm * 8, 256, 0, h->stream>>>(h->c[st.cur], n, eps, seed, keep, nc);
    return flag_compact(h, st, keep, nc, nullptr, sc);
}

// _apply!(v, ::StochasticSamplingTruncation) (spv_evolve.jl:69-99): the n_keep
// largest keys u^(1/|c|^2) (exact radix select; ties: the smaller index), then
// the norm-restoring scale.
static int stoch_sample_apply(pp_spv *h, long long n_keep, unsigned long long seed) {
    DevState st;
    TRY(read_state(h, &st));
    const long long n = st.n;
    if (n <= n_keep) return PP_OK;
    Scratch sc;
    unsigned long long *key;
    unsigned char *keep, *keyeq;
    int *tcnt, *toff;
    long long *ttot;
    Select64 *sel;
    double *pall, *pkept, *nrm;
    const long long ntiles = (n + FC_TILE - 1) / FC_TILE;
    const int nb = std::min(4096, h->nsm * 8);
    TRY(sc.get(&key, n));
    TRY(sc.get(&keep, n));
    TRY(sc.get(&keyeq, n));
    TRY(sc.get(&tcnt, ntiles));
    TRY(sc.get(&toff, ntiles));
    TRY(sc.get(&ttot, 1));
    TRY(sc.get(&sel, 1));
    TRY(sc.get(&pall, nb));
    TRY(sc.get(&pkept, nb));
    TRY(sc.get(&nrm, 3));
    cudaStream_t s = h->stream;
    const double *C = h->c[st.cur];
    k_stoch_sample_keys<<<h->nsm * 8, 256, 0, s>>>(C, n, seed, key);
    Select64 s0;
    memset(&s0, 0, sizeof s0);
    s0.remaining = n_keep;
    CU(cudaMemcpyAsync(sel, &s0, sizeof s0, cudaMemcpyHostToDevice, s));
    for (int shift = 56; shift >= 0; shift -= 8) {
        k_key64_hist<<<h->nsm * 4, 256, 0, s>>>(key, n, sel, shift);
        k_sel64_pick<<<1, 32, 0, s>>>(sel, shift);
    }
    k_stoch_sample_mark<<<h->nsm * 8, 256, 0, s>>>(key, n, sel, keep, keyeq);
    const int g = (int)std::min<long long>(ntiles, 8ll * h->nsm);
    k_flag_count<<<g, FC_THREADS, 0, s>>>(keyeq, n, tcnt);
    k_flag_scan<<<1, 1024, 0, s>>>(ntiles, tcnt, toff, ttot);
    k_stoch_sample_ties<<<g, FC_THREADS, 0, s>>>(n, sel, keyeq, toff, keep);
    k_norm_partials<<<nb, 256, 0, s>>>(C, keep, n, pall, pkept);
    k_expect_final<<<1, 32, 0, s>>>(pall, nb, nrm);
    k_expect_final<<<1, 32, 0, s>>>(pkept, nb, nrm + 1);
    k_norm_scale<<<1, 32, 0, s>>>(nrm, nrm + 1, nrm + 2);
    return flag_compact(h, st, keep, nullptr, nrm + 2, sc);
}

// Truncations that run as a separate step after an unfiltered merge
// (_boundary!, spv_evolve.jl:258-284): AdaptiveTruncation (_apply!), and any
// truncation under EnergyVarianceCorrection (_needs_merged_measure: merge with
// NOFILTER, measure, compact with the strict filter, measure).  The energy (and
// variance) change the step causes is accumulated.
struct AdaptSpec {
    bool on = false;
    int kind = 0;                     // 0 compiled strict filter, 1 Adaptive, 2 StochasticCoeff, 3 StochasticSampling
    bool adaptive = false;            // kind == 1
    double epsilon = 0.0;             // kind 2
    unsigned long long seed = 0;      // kinds 2, 3: each application draws from seed + its index
    long long napp = 0;
    long long max_terms = 0;
    double min_thresh = 0.0;
    pp_filter strict = NOFILTER_H;
    bool corr = false;                // EnergyCorrection or EnergyVarianceCorrection
    bool var = false;                 // EnergyVarianceCorrection
    u64 ket[2] = {0, 0};
    double var_acc = 0.0;             // accumulated variance change of this call
};

static int compact_with(pp_spv *h, const pp_filter &f) {
    compile_filter(&f, &h->Ph->clip);
    TRY(upload_params(h));
    DevState st;
    TRY(read_state(h, &st));
    st.an = 0;
    TRY(write_state(h, &st));
    Bufs B = make_bufs(h);
    if (h->NW == 1) launch_merge<1, 2>(h, B, 0);
    else launch_merge<2, 2>(h, B, 0);
    TRY(sync_check(h));
    TRY(read_state(h, &st));
    return check_err(h, st);
}

static int adapt_step(pp_spv *h, AdaptSpec &A) {
    double before = 0.0, after = 0.0, vb = 0.0, va = 0.0;
    if (A.corr) TRY(expect_dev(h, A.ket, &before));
    if (A.var) TRY(variance_dev(h, A.ket, &vb));
    const unsigned long long sd = A.seed + 0xD1B54A32D192ED03ull * (unsigned long long)(A.napp++);
    if (A.kind == 1) TRY(adaptive_apply(h, A.max_terms, A.min_thresh));
    else if (A.kind == 2) TRY(stoch_clip_apply(h, A.epsilon, sd));
    else if (A.kind == 3) TRY(stoch_sample_apply(h, A.max_terms, sd));
    else TRY(compact_with(h, A.strict));
    if (A.corr) {
        TRY(expect_dev(h, A.ket, &after));
        DevState st;
        TRY(read_state(h, &st));
        st.corr_energy += after - before;
        TRY(write_state(h, &st));
    }
    if (A.var) {
        TRY(variance_dev(h, A.ket, &va));
        A.var_acc += va - vb;
    }
    return PP_OK;
}

// General path: the sequence driver of spv_evolve.jl:352-385 with host decisions.
// `period` > 0 makes every period-th rotation end a separate evolve! call (the
// window count restarts and a boundary closes the layer), which is the
// semantics of a loop "evolve!(v, layer; ...); channel!(v, p)".
template <int NW>
static int run_general(pp_spv *h, const std::vector<GenRec> &G, long long window, pp_counters *ctr, int last_flags,
                       long long period, int chan_flags, RunProf *prof, AdaptSpec &A) {
    const long long L = (long long)G.size();
    long long since = 0;
    for (long long i = 1; i <= L; ++i) {
        const long long w = (i + window - 1) / window;
        const long long irel = period > 0 ? (i - 1) % period + 1 : i;
        DevState st;
        TRY(read_state(h, &st));
        if (2 * st.an + st.n > st.acap_logical) {
            long long ni, no;
            TRY(general_boundary<NW>(h, 0, &ni, &no));
            if (A.on) TRY(adapt_step(h, A));
            since = 0;
            TRY(read_state(h, &st));
            if (ctr && w <= ctr->nwin) {
                if (ctr->early_merges) ctr->early_merges[w - 1] += 1;
                if (ctr->merge_in) ctr->merge_in[w - 1] += ni;
                if (ctr->merge_out) ctr->merge_out[w - 1] += no;
            }
            if (st.n > st.acap_logical) {
                st.acap_logical = std::max(2 * st.acap_logical, st.n);
                TRY(write_state(h, &st));
            }
        }
        TRY(ensure_append(h, std::max(st.acap_logical, 2 * st.an + st.n), st.an));
        TRY(alloc_merge_ws(h, h->cap, h->acap_phys));
        Bufs B = make_bufs(h);
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (ctr && ctr->t_rotate) { cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventRecord(e0, h->stream); }
        const long long an_before = st.an;
        const int ntiles = (int)std::max(1ll, (st.n + st.an + G_TILE - 1) / G_TILE);
        k_rotate_general<NW><<<std::min(ntiles, h->nsm * h->occG), G_THREADS, 0, h->stream>>>(B, G[i - 1]);
        k_rotate_commit<<<1, 1, 0, h->stream>>>(B);
        if (e1) cudaEventRecord(e1, h->stream);
        TRY(sync_check(h));
        TRY(read_state(h, &st));
        TRY(check_err(h, st));
        if (ctr && w <= ctr->nwin) {
            if (ctr->terms_created) ctr->terms_created[w - 1] += st.an - an_before;
            if (e0) { float ms = 0; cudaEventElapsedTime(&ms, e0, e1); ctr->t_rotate[w - 1] += ms * 1e-3; }
        }
        if (e0) { cudaEventDestroy(e0); cudaEventDestroy(e1); }
        since++;
        prof->launches += 2;
        const bool layer_end = period > 0 && irel == period;
        if (irel % window == 0 || layer_end || i == L) {
            long long ni, no;
            cudaEvent_t m0 = nullptr, m1 = nullptr;
            if (ctr && ctr->t_merge) { cudaEventCreate(&m0); cudaEventCreate(&m1); cudaEventRecord(m0, h->stream); }
            const int fl = (i == L ? last_flags : 0) | (layer_end ? chan_flags : 0);
            if (!A.on) {
                TRY(general_boundary<NW>(h, fl, &ni, &no));
            } else {
                // merge unfiltered, then the strategy, then the layer's channel, then <ket|O|ket>
                TRY(general_boundary<NW>(h, 0, &ni, &no));
                TRY(adapt_step(h, A));
                if (fl & GEN_CHANNEL) {
                    Bufs Bc = make_bufs(h);
                    k_channel<NW><<<h->nsm * 8, 256, 0, h->stream>>>(Bc);
                    TRY(sync_check(h));
                }
                if (fl & GEN_MEASURE) {
                    double e = 0.0;
                    const u64 *kk = h->Ph->ket;
                    TRY(expect_dev(h, kk, &e));
                    DevState s2;
                    TRY(read_state(h, &s2));
                    s2.expect_val = e;
                    s2.measure_valid = 1;
                    TRY(write_state(h, &s2));
                }
            }
            prof->launches += 3;
            if (m0) {
                cudaEventRecord(m1, h->stream);
                cudaEventSynchronize(m1);
                float ms = 0;
                cudaEventElapsedTime(&ms, m0, m1);
                if (w <= ctr->nwin) ctr->t_merge[w - 1] += ms * 1e-3;
                cudaEventDestroy(m0); cudaEventDestroy(m1);
            }
            if (ctr && w <= ctr->nwin) {
                if (ctr->merge_in) ctr->merge_in[w - 1] += ni;
                if (ctr->merge_out) ctr->merge_out[w - 1] += no;
            }
            since = 0;
        }
    }
    return PP_OK;
}

static int evolve_impl(pp_spv *h, const void *gz, const void *gx, const double *cosv, const double *sinv, int64_t L,
                       const pp_evolve_opts *o) {
    pp_evolve_opts def;
    memset(&def, 0, sizeof def);
    def.window = 1;
    def.chan_kind = -1;
    const pp_evolve_opts &O = o ? *o : def;
    if (O.window < 1) return fail(PP_ARGUMENT_ERROR, "window must be >= 1");
    if (L < 0) return fail(PP_DIMENSION_MISMATCH, "generators and angles must have same length");
    if (L > 0 && (!gz || !gx || !cosv || !sinv)) return fail(PP_ARGUMENT_ERROR, "null generator arrays");
    if (O.strict_kind < 0 || O.strict_kind > 3) return fail(PP_ARGUMENT_ERROR, "unknown strict_kind");
    AdaptSpec A;
    if (O.strict_kind != 0 || O.corr_kind == 2) {
        if ((O.strict_kind == 1 || O.strict_kind == 3) && O.adapt_max_terms < 0)
            return fail(PP_ARGUMENT_ERROR, "max_terms / n_keep must be >= 0");
        A.on = true;
        A.kind = O.strict_kind;
        A.adaptive = O.strict_kind == 1;
        A.epsilon = O.adapt_min_thresh;
        A.seed = O.seed;
        A.max_terms = O.adapt_max_terms;
        A.min_thresh = O.adapt_min_thresh;
        if (O.strict_kind == 0 && O.strict) A.strict = *O.strict;
        A.corr = O.corr_kind == 1 || O.corr_kind == 2;
        A.var = O.corr_kind == 2;
        load_word(O.ket, h->NW, A.ket);
    }
    if (O.corr_kind < 0 || O.corr_kind > 2) return fail(PP_ARGUMENT_ERROR, "unknown corr_kind");
    // parameters (a separate truncation step merges unfiltered and measures itself)
    DevParams *P = h->Ph;
    compile_filter(A.on ? nullptr : O.strict, &P->strict);
    compile_filter(O.local, &P->local);
    P->local_active = filter_is_nofilter(O.local) ? 0 : 1;
    P->corr_kind = A.on ? 0 : O.corr_kind;
    load_word(O.ket, h->NW, P->ket);
    P->chan_kind = -1;
    if (O.chan_kind >= 0) TRY(build_channel(h, O.chan_kind, O.chan_prm, O.chan_mask, P));
    if (L == 0) {
        if (O.chan_kind >= 0) {
            TRY(upload_params(h));
            Bufs B = make_bufs(h);
            if (h->NW == 1) k_channel<1><<<h->nsm * 8, 256, 0, h->stream>>>(B);
            else k_channel<2><<<h->nsm * 8, 256, 0, h->stream>>>(B);
            TRY(sync_check(h));
        }
        return PP_OK;
    }
    TRY(upload_params(h));
    // generators
    TRY(ensure_gens(h, L));
    std::vector<GenRec> G((size_t)L);
    bool all_struct = true;
    const size_t wb = (size_t)h->NW * 8;
    for (long long i = 0; i < L; ++i) {
        u64 wz[2] = {0, 0}, wx[2] = {0, 0};
        memcpy(wz, (const char *)gz + i * wb, wb);
        memcpy(wx, (const char *)gx + i * wb, wb);
        bool st = true;
        make_gen(h, wz, wx, cosv[i], sinv[i], &G[i], &st);
        all_struct = all_struct && st;
    }
    const bool chan = O.chan_kind >= 0;
    const long long period = (chan && O.chan_every > 0) ? O.chan_every : 0;
    const int last_flags = GEN_MEASURE | ((chan && period == 0) ? GEN_CHANNEL : 0);
    G[L - 1].flags |= last_flags;
    if (period > 0)
        for (long long i = period - 1; i < L; i += period) G[i].flags |= GEN_CHANNEL;
    memcpy(h->gens_h, G.data(), L * sizeof(GenRec));
    CU(cudaMemcpyAsync(h->gens, h->gens_h, L * sizeof(GenRec), cudaMemcpyHostToDevice, h->stream));
    // state for this call
    DevState st;
    TRY(read_state(h, &st));
    st.rot = 0; st.rot_end = L;
    st.created = st.merge_in = st.merge_out = st.early = 0;
    st.npref = 0;
    st.live_in = 0;
    st.peak = 0;
    st.corr_energy = O.corr_energy ? *O.corr_energy : 0.0;
    st.measure_valid = 0;
    st.b_tile_ctr = 0; st.g_tile_ctr = 0;
    TRY(write_state(h, &st));
    pp_counters *ctr = O.counters;
    RunProf prof;
    prof.on = O.profile != 0;
    if (O.window == 1 && all_struct && !A.on) {
        TRY(ensure_live(h, 3 * st.n + 2 * SEG));
        const bool want_rec = ctr && ctr->nwin > 0;
        if (want_rec && L > h->rec_cap) {
            TRY(dalloc(h, &h->rec, 4 * L));
            h->rec_cap = L;
        }
        if (want_rec != h->rec_on) { h->rec_on = want_rec; h->buf_gen++; }
        if (h->NW == 1) TRY(run_struct<1>(h, 0, L, ctr, &prof, st.n));
        else TRY(run_struct<2>(h, 0, L, ctr, &prof, st.n));
        if (want_rec) {
            std::vector<long long> rec((size_t)(4 * L));
            CU(cudaMemcpy(rec.data(), h->rec, 4 * L * sizeof(long long), cudaMemcpyDeviceToHost));
            for (long long r = 0; r < L && r < ctr->nwin; ++r) {
                if (ctr->terms_created) ctr->terms_created[r] += rec[4 * r];
                if (ctr->merge_in) ctr->merge_in[r] += rec[4 * r + 1];
                if (ctr->merge_out) ctr->merge_out[r] += rec[4 * r + 2];
                if (ctr->early_merges) ctr->early_merges[r] += rec[4 * r + 3];
            }
        }
    } else {
        if (h->NW == 1) TRY(run_general<1>(h, G, O.window, ctr, last_flags, period, GEN_CHANNEL, &prof, A));
        else TRY(run_general<2>(h, G, O.window, ctr, last_flags, period, GEN_CHANNEL, &prof, A));
    }
    TRY(read_state(h, &st));
    TRY(check_err(h, st));
    if (O.corr_energy) *O.corr_energy = st.corr_energy;
    if (O.corr_variance) *O.corr_variance += A.var_acc;
    if (O.expect_out) *O.expect_out = st.expect_val;
    if (O.stats_out) {
        double *so = O.stats_out;
        for (int i = 0; i < PP_STATS_LEN; ++i) so[i] = 0.0;
        so[PP_STAT_TERMS_IN] = (double)st.live_in;
        so[PP_STAT_CREATED] = (double)st.created;
        so[PP_STAT_MERGE_IN] = (double)st.merge_in;
        so[PP_STAT_MERGE_OUT] = (double)st.merge_out;
        so[PP_STAT_PEAK] = (double)st.peak;
        so[PP_STAT_EARLY] = (double)st.early;
        so[PP_STAT_T_ROTATE] = prof.t_rotate;
        so[PP_STAT_T_MERGE] = prof.t_merge;
        so[PP_STAT_LAUNCHES] = (double)prof.launches;
        so[PP_STAT_BUCKET_ROT] = (double)prof.bk_rot;
        so[PP_STAT_BUCKET_BYTES] = prof.bk_bytes;
        so[PP_STAT_T_PARTITION] = prof.t_partition;
    }
    return PP_OK;
}

extern "C" int pp_evolve(pp_spv *h, const void *gz, const void *gx, const double *cosv, const double *sinv, int64_t L,
                         const pp_evolve_opts *opts) {
    if (!h) return fail(PP_ARGUMENT_ERROR, "null handle");
    return evolve_impl(h, gz, gx, cosv, sinv, L, opts);
}

extern "C" int pp_evolve1(pp_spv *h, const void *gz, const void *gx, double cos_theta, double sin_theta) {
    if (!h) return fail(PP_ARGUMENT_ERROR, "null handle");
    // evolve!(O, G, θ): grow the append capacity to n + 2an first (spv_evolve.jl:231),
    // which is what the early-merge rule of later sequence calls sees.
    DevState st;
    TRY(read_state(h, &st));
    if (st.n + 2 * st.an > st.acap_logical) {
        st.acap_logical = std::max(2 * st.acap_logical, st.n + 2 * st.an);
        TRY(write_state(h, &st));
    }
    pp_evolve_opts o;
    memset(&o, 0, sizeof o);
    o.window = 1;
    o.chan_kind = -1;
    return evolve_impl(h, gz, gx, &cos_theta, &sin_theta, 1, &o);
}

extern "C" int pp_compact(pp_spv *h, const pp_filter *f) {
    if (!h) return fail(PP_ARGUMENT_ERROR, "null handle");
    compile_filter(f, &h->Ph->clip);
    TRY(upload_params(h));
    DevState st;
    TRY(read_state(h, &st));
    st.an = 0;
    TRY(write_state(h, &st));
    Bufs B = make_bufs(h);
    if (h->NW == 1) launch_merge<1, 2>(h, B, 0);
    else launch_merge<2, 2>(h, B, 0);
    TRY(sync_check(h));
    TRY(read_state(h, &st));
    return check_err(h, st);
}

extern "C" int pp_adaptive(pp_spv *h, int64_t max_terms, double min_thresh) {
    if (!h) return fail(PP_ARGUMENT_ERROR, "null handle");
    if (max_terms < 0) return fail(PP_ARGUMENT_ERROR, "max_terms must be >= 0");
    return adaptive_apply(h, max_terms, min_thresh);
}

extern "C" int pp_channel(pp_spv *h, int32_t kind, const double *prm, const void *qubit_mask) {
    if (!h) return fail(PP_ARGUMENT_ERROR, "null handle");
    TRY(build_channel(h, kind, prm, qubit_mask, h->Ph));
    TRY(upload_params(h));
    Bufs B = make_bufs(h);
    if (h->NW == 1) k_channel<1><<<h->nsm * 8, 256, 0, h->stream>>>(B);
    else k_channel<2><<<h->nsm * 8, 256, 0, h->stream>>>(B);
    return sync_check(h);
}

extern "C" int pp_expect_ket(pp_spv *h, const void *ket, double *out) {
    if (!h || !out) return fail(PP_ARGUMENT_ERROR, "null argument");
    u64 k[2];
    load_word(ket, h->NW, k);
    Bufs B = make_bufs(h);
    const int nb = std::min(4096, h->nsm * 8);
    if (h->NW == 1) k_expect<1><<<nb, 256, 0, h->stream>>>(B, k[0], k[1], h->epart);
    else k_expect<2><<<nb, 256, 0, h->stream>>>(B, k[0], k[1], h->epart);
    k_expect_final<<<1, 32, 0, h->stream>>>(h->epart, nb, h->eout);
    CU(cudaMemcpyAsync(out, h->eout, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    return sync_check(h);
}

extern "C" int pp_check(pp_spv *h, int32_t *ok) {
    if (!h || !ok) return fail(PP_ARGUMENT_ERROR, "null argument");
    DevState st;
    TRY(read_state(h, &st));
    st.err &= ~ERR_CHECK;
    TRY(write_state(h, &st));
    Bufs B = make_bufs(h);
    if (h->NW == 1) k_check<1><<<h->nsm * 8, 256, 0, h->stream>>>(B);
    else k_check<2><<<h->nsm * 8, 256, 0, h->stream>>>(B);
    TRY(sync_check(h));
    TRY(read_state(h, &st));
    *ok = (!(st.err & ERR_CHECK) && st.n <= h->cap && st.an == 0) ? 1 : 0;
    st.err &= ~ERR_CHECK;
    TRY(write_state(h, &st));
    return PP_OK;
}

extern "C" int pp_stream(pp_spv *h, void **stream) {
    if (!h || !stream) return fail(PP_ARGUMENT_ERROR, "null argument");
    *stream = (void *)h->stream;
    return PP_OK;
}

#ifdef PP_PHASE_TIMERS
extern "C" int pp_debug_phase_cycles(unsigned long long *out, int reset) {
    cudaMemcpyFromSymbol(out, pp_phase_cycles, sizeof(unsigned long long) * 8);
    if (reset) {
        unsigned long long z[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        cudaMemcpyToSymbol(pp_phase_cycles, z, sizeof z);
    }
    return PP_OK;
}
#endif

// ------------------------------------------------------------------ tuning
extern "C" int pp_set_tuning(pp_spv *h, const pp_tuning *t) {
    if (!h || !t) return fail(PP_ARGUMENT_ERROR, "pp_set_tuning: null argument");
    if (!bk_variant(t->bucket_cap, t->items_per_thread))
        return fail(PP_ARGUMENT_ERROR, "pp_set_tuning: (bucket_cap, items_per_thread) must be one of (128, 4), "
                                       "(256, 4), (512, 4), (256, 8), (512, 8), (1024, 8)");
    if (t->load_div < 3 || t->load_div > 16) return fail(PP_ARGUMENT_ERROR, "pp_set_tuning: load_div must be in 3..16");
    if (t->chunk < 8 || t->chunk > 256) return fail(PP_ARGUMENT_ERROR, "pp_set_tuning: chunk must be in 8..256");
    if (t->bucket_cap != h->tune.bucket_cap || t->items_per_thread != h->tune.items_per_thread ||
        t->chunk != h->tune.chunk) {
        for (auto &kv : h->bk_graphs) cudaGraphExecDestroy(kv.second);
        h->bk_graphs.clear();
    }
    h->tune = *t;
    return PP_OK;
}

extern "C" int pp_get_tuning(pp_spv *h, pp_tuning *t) {
    if (!h || !t) return fail(PP_ARGUMENT_ERROR, "pp_get_tuning: null argument");
    *t = h->tune;
    return PP_OK;
}

extern "C" int pp_device_info(pp_spv *h, int32_t *sm_count, int32_t *cc_major, int32_t *cc_minor) {
    if (!h || !sm_count || !cc_major || !cc_minor) return fail(PP_ARGUMENT_ERROR, "pp_device_info: null argument");
    int ma = 0, mi = 0;
    CU(cudaDeviceGetAttribute(&ma, cudaDevAttrComputeCapabilityMajor, h->dev));
    CU(cudaDeviceGetAttribute(&mi, cudaDevAttrComputeCapabilityMinor, h->dev));
    *sm_count = h->nsm;
    *cc_major = ma;
    *cc_minor = mi;
    return PP_OK;
}

// ------------------------------------------------------------------ test hooks
extern "C" int pp_debug_fail_alloc(int64_t after) {
    g_fail_alloc_after.store(after > 0 ? after : 0);
    return PP_OK;
}

extern "C" int pp_debug_bucket_limit(int64_t slots) {
    g_bk_slot_limit.store(slots > 0 ? slots : 0);
    return PP_OK;
}

// A look-back status that nothing publishes: tile 1's bounded wait on tile 0
// must give up after `limit` polls and report ERR_TIMEOUT.
static __device__ u64 g_dbg_status[2];
static __device__ int g_dbg_err;

__global__ void k_debug_lookback(long long limit) {
    lookback_warp(g_dbg_status, 1, 1u, 7u, &g_dbg_err, limit);
}

extern "C" int pp_debug_lookback_timeout(int64_t limit) {
    if (limit < 1 || limit > SPIN_LIMIT) return fail(PP_ARGUMENT_ERROR, "limit must be in 1..2^22");
    const u64 zs[2] = {0, 0};
    const int ze = 0;
    CU(cudaMemcpyToSymbol(g_dbg_status, zs, sizeof zs));
    CU(cudaMemcpyToSymbol(g_dbg_err, &ze, sizeof ze));
    k_debug_lookback<<<1, 32>>>((long long)limit);
    CU(cudaGetLastError());
    CU(cudaDeviceSynchronize());
    int e = 0;
    CU(cudaMemcpyFromSymbol(&e, g_dbg_err, sizeof e));
    if (e & ERR_TIMEOUT) return fail(PP_TIMEOUT, "a device-side look-back wait timed out (test hook: nothing publishes)");
    return fail(PP_ERROR_EXCEPTION, "the look-back wait did not report its timeout");
}

extern "C" int pp_device_bytes(pp_spv *h, int64_t *bytes) {
    if (!h || !bytes) return fail(PP_ARGUMENT_ERROR, "null argument");
    *bytes = h->bytes;
    return PP_OK;
}

// ------------------------------------------------------------------ batched instances
template <typename T>
static int ensure_buf(pp_spv *h, T **p, long long need, long long *cap) {
    if (need <= *cap && *p) return PP_OK;
    TRY(dalloc(h, p, need));
    *cap = need;
    return PP_OK;
}

static int batch_impl(pp_spv *h, const void *gz, const void *gx, long long L, const pp_batch *b,
                      const pp_evolve_opts &O, long long *acap_saved) {
    const long long ninst = b->ninst;
    const int ncol = b->ncol, nq = b->nq;
    std::vector<long long> ends((size_t)ninst);
    for (long long i = 0; i < ninst; ++i) {
        ends[i] = b->rot_end[i];
        if (ends[i] < 0 || ends[i] > L) return fail(PP_ARGUMENT_ERROR, "rot_end must lie in 0..L");
    }
    // parameters: strict filter over the instance word, no local filter, channel on the instance qubits
    DevParams *P = h->Ph;
    compile_filter(O.strict, &P->strict);
    P->strict.wlow = 1;
    compile_filter(nullptr, &P->local);
    P->local_active = 0;
    compile_filter(nullptr, &P->clip);   // the harvest compaction keeps every term of running instances
    P->corr_kind = 0;
    load_word(O.ket, 2, P->ket);
    P->ket[1] = 0;
    P->chan_kind = -1;
    if (O.chan_kind >= 0) {
        u64 m[2] = {nq == 64 ? ~0ull : ((1ull << nq) - 1ull), 0ull};
        if (O.chan_mask) {
            load_word(O.chan_mask, 2, m);
            m[1] = 0;
        }
        TRY(build_channel(h, O.chan_kind, O.chan_prm, m, P));
    }
    TRY(upload_params(h));
    // instance tables and harvest workspaces
    long long tcap = h->btab_cap, icap = h->binst_cap;
    TRY(ensure_buf(h, &h->bcos, ninst * ncol, &tcap));
    tcap = h->btab_cap;
    TRY(ensure_buf(h, &h->bsin, ninst * ncol, &tcap));
    h->btab_cap = tcap;
    if (ninst > h->binst_cap || !h->bend) {
        TRY(dalloc(h, &h->bend, ninst));
        TRY(dalloc(h, &h->hfin, ninst));
        TRY(dalloc(h, &h->hpart, ninst * HV_CHUNKS));
        TRY(dalloc(h, &h->heout, ninst));
        TRY(dalloc(h, &h->hrange, 2 * ninst));
        TRY(dalloc(h, &h->hnout, ninst));
        icap = ninst;
    }
    h->binst_cap = icap;
    CU(cudaMemcpyAsync(h->bcos, b->cosv, ninst * ncol * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CU(cudaMemcpyAsync(h->bsin, b->sinv, ninst * ncol * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CU(cudaMemcpyAsync(h->bend, ends.data(), ninst * sizeof(long long), cudaMemcpyHostToDevice, h->stream));
    h->batch_on = true;
    h->ninst = ninst;
    h->ncol = ncol;
    h->rec_on = false;
    h->buf_gen++;
    // generators: the instance qubits only; the angle column of each rotation
    if (L > 0) {
        TRY(ensure_gens(h, L));
        std::vector<GenRec> G((size_t)L);
        for (long long i = 0; i < L; ++i) {
            u64 wz[2] = {0, 0}, wx[2] = {0, 0};
            memcpy(wz, (const char *)gz + i * 16, 16);
            memcpy(wx, (const char *)gx + i * 16, 16);
            if (wz[1] || wx[1] || (nq < 64 && ((wz[0] | wx[0]) >> nq)))
                return fail(PP_ARGUMENT_ERROR, "generators must act on the instance qubits only");
            if (b->acol[i] < 0 || b->acol[i] >= ncol) return fail(PP_ARGUMENT_ERROR, "acol out of range");
            bool st = true;
            TRY(make_gen(h, wz, wx, 1.0, 0.0, &G[i], &st));
            if (!st) return fail(PP_NOT_IMPLEMENTED, "batched instances need generators of at most 16 mask levels");
            G[i].acol = b->acol[i];
        }
        if (O.chan_kind >= 0) {
            if (O.chan_every > 0) {
                for (long long i = O.chan_every - 1; i < L; i += O.chan_every) G[i].flags |= GEN_CHANNEL;
            } else {
                G[L - 1].flags |= GEN_CHANNEL;
            }
        }
        memcpy(h->gens_h, G.data(), L * sizeof(GenRec));
        CU(cudaMemcpyAsync(h->gens, h->gens_h, L * sizeof(GenRec), cudaMemcpyHostToDevice, h->stream));
    }
    // state: no early merges (every instance has an unbounded append capacity)
    DevState st;
    TRY(read_state(h, &st));
    *acap_saved = st.acap_logical;
    st.acap_logical = 1ll << 62;
    st.rot = 0;
    st.rot_end = 0;
    st.created = st.merge_in = st.merge_out = st.early = 0;
    st.npref = 0;
    st.live_in = 0;
    st.peak = 0;
    st.measure_valid = 0;
    st.b_tile_ctr = 0;
    st.g_tile_ctr = 0;
    TRY(write_state(h, &st));
    TRY(ensure_live(h, 3 * st.n + 2 * SEG));
    // harvest points: the distinct instance ends, in order
    std::vector<long long> pts(ends);
    std::sort(pts.begin(), pts.end());
    pts.erase(std::unique(pts.begin(), pts.end()), pts.end());
    std::vector<cudaEvent_t> ev(pts.size() + 1);
    for (auto &e : ev) cudaEventCreate(&e);
    struct EvGuard {
        std::vector<cudaEvent_t> &v;
        ~EvGuard() { for (auto e : v) cudaEventDestroy(e); }
    } evg{ev};
    RunProf prof;
    prof.on = O.profile != 0;
    CU(cudaEventRecord(ev[0], h->stream));
    long long done = 0;
    std::vector<int> fin;
    fin.reserve((size_t)ninst);
    for (size_t k = 0; k < pts.size(); ++k) {
        const long long r = pts[k];
        if (r > done) {
            TRY(read_state(h, &st));
            st.rot_end = r;
            TRY(write_state(h, &st));
            TRY(run_struct<2>(h, done, r, nullptr, &prof));
            done = r;
        }
        fin.clear();
        for (long long i = 0; i < ninst; ++i) if (ends[i] == r) fin.push_back((int)i);
        const int nfin = (int)fin.size();
        CU(cudaMemcpyAsync(h->hfin, fin.data(), nfin * sizeof(int), cudaMemcpyHostToDevice, h->stream));
        Bufs B = make_bufs(h);
        k_harvest_part<<<dim3(HV_CHUNKS, nfin), HV_THREADS, 0, h->stream>>>(B, h->hfin, h->hpart, h->hrange);
        k_harvest_fin<<<(nfin + 127) / 128, 128, 0, h->stream>>>(h->hfin, nfin, h->hpart, h->hrange, h->heout,
                                                                 h->hnout);
        prof.launches += 2;
        if (!b->keep_finished) {
            TRY(read_state(h, &st));
            st.an = 0;
            TRY(write_state(h, &st));
            launch_merge<2, 2>(h, B, GEN_HARVEST);
            prof.launches += 3;
        }
        CU(cudaEventRecord(ev[k + 1], h->stream));
        TRY(sync_check(h));
        TRY(read_state(h, &st));
        TRY(check_err(h, st));
    }
    if (b->expect_out)
        CU(cudaMemcpyAsync(b->expect_out, h->heout, ninst * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (b->n_final)
        CU(cudaMemcpyAsync(b->n_final, h->hnout, ninst * sizeof(long long), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    if (b->t_done) {
        for (long long i = 0; i < ninst; ++i) {
            const size_t k = std::lower_bound(pts.begin(), pts.end(), ends[i]) - pts.begin();
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[0], ev[k + 1]);
            b->t_done[i] = ms * 1e-3;
        }
    }
    TRY(read_state(h, &st));
    if (O.stats_out) {
        double *so = O.stats_out;
        for (int i = 0; i < PP_STATS_LEN; ++i) so[i] = 0.0;
        so[PP_STAT_TERMS_IN] = (double)st.live_in;
        so[PP_STAT_CREATED] = (double)st.created;
        so[PP_STAT_MERGE_IN] = (double)st.merge_in;
        so[PP_STAT_MERGE_OUT] = (double)st.merge_out;
        so[PP_STAT_PEAK] = (double)st.peak;
        so[PP_STAT_T_ROTATE] = prof.t_rotate;
        so[PP_STAT_T_MERGE] = prof.t_merge;
        so[PP_STAT_LAUNCHES] = (double)prof.launches;
        so[PP_STAT_BUCKET_ROT] = (double)prof.bk_rot;
        so[PP_STAT_BUCKET_BYTES] = prof.bk_bytes;
        so[PP_STAT_T_PARTITION] = prof.t_partition;
    }
    return PP_OK;
}

extern "C" int pp_evolve_batch(pp_spv *h, const void *gz, const void *gx, int64_t L, const pp_batch *b,
                               const pp_evolve_opts *opts) {
    if (!h || !b) return fail(PP_ARGUMENT_ERROR, "null argument");
    if (h->NW != 2) return fail(PP_ARGUMENT_ERROR, "batched instances need a handle with 128-bit words (N > 64)");
    if (L < 0 || b->ninst < 1 || b->ninst > (1ll << 30) || b->ncol < 1 || b->nq < 1 || b->nq > 64)
        return fail(PP_ARGUMENT_ERROR, "need L >= 0, 1 <= ninst <= 2^30, ncol >= 1, 1 <= nq <= 64");
    if ((L > 0 && (!gz || !gx || !b->acol)) || !b->cosv || !b->sinv || !b->rot_end)
        return fail(PP_ARGUMENT_ERROR, "null array");
    pp_evolve_opts O;
    memset(&O, 0, sizeof O);
    O.window = 1;
    O.chan_kind = -1;
    if (opts) O = *opts;
    if (O.window != 1) return fail(PP_ARGUMENT_ERROR, "batched instances run at window = 1");
    if (!filter_is_nofilter(O.local)) return fail(PP_ARGUMENT_ERROR, "batched instances take no local_truncation");
    if (O.strict_kind != 0 || O.corr_kind != 0)
        return fail(PP_NOT_IMPLEMENTED, "batched instances support compiled truncations and NoCorrection only");
    long long acap = -1;
    int r = batch_impl(h, gz, gx, L, b, O, &acap);
    // back to a plain vector whatever happened
    h->batch_on = false;
    h->buf_gen++;
    if (acap >= 0) {
        DevState st;
        if (read_state(h, &st) == PP_OK) {
            st.acap_logical = acap;
            write_state(h, &st);
        }
    }
    return r;
}

// ------------------------------------------------------------------ key-sharded runs
// One rank of a window-1 evolution whose live set is split over 2^rank_bits ranks
// by owner(P) (bk_owner: GF(2)-linear, so a term's sin branch P xor M is owned by
// owner(P) xor owner(M)).  Per rotation r the caller (one process per GPU, or one
// process driving several handles) runs, on every rank:
//   pp_shard_send   the local terms whose sin branches the partner rank owns;
//   (exchange them with the partner rank r xor owner(M); nothing when equal)
//   pp_shard_recv   the partner's terms, as foreign terms of this rank's buckets;
//   pp_shard_rotate one k_bk_rotate launch: own outputs of local terms, sin
//                   branches of foreign terms whose partner is absent here;
// and agrees on the global counts (early-merge rule, splits) between rotations.
// All ranks use the same bucket count, so a bucket never holds more than cap/2
// local plus cap/2 foreign terms.

static int shard_fcnt(pp_spv *h) {
    // foreign counts for the current bucket capacity, zeroed
    if (h->bkfcnt_bits < h->bk_bits_cap || !h->bkfcnt[0]) {
        int *f0 = nullptr, *f1 = nullptr;
        TRY(dalloc(h, &f0, 1ll << h->bk_bits_cap));
        int r = dalloc(h, &f1, 1ll << h->bk_bits_cap);
        if (r) { dfree(h, f0); return r; }
        dfree(h, h->bkfcnt[0]);
        dfree(h, h->bkfcnt[1]);
        h->bkfcnt[0] = f0;
        h->bkfcnt[1] = f1;
        h->bkfcnt_bits = h->bk_bits_cap;
    }
    CU(cudaMemsetAsync(h->bkfcnt[0], 0, sizeof(int) << h->bkfcnt_bits, h->stream));
    CU(cudaMemsetAsync(h->bkfcnt[1], 0, sizeof(int) << h->bkfcnt_bits, h->stream));
    return PP_OK;
}

extern "C" int pp_shard_owner(int32_t nw, const void *z, const void *x, int64_t n, int32_t rank_bits, int32_t *owner) {
    if (nw < 1 || nw > 2 || n < 0 || rank_bits < 0 || rank_bits > 8)
        return fail(PP_ARGUMENT_ERROR, "need nw in 1..2, n >= 0, rank_bits in 0..8");
    if (n > 0 && (!z || !x || !owner)) return fail(PP_ARGUMENT_ERROR, "null array");
    u64 rows[BK_ROWS * 4];
    bk_rows_host(rows);
    for (int64_t i = 0; i < n; ++i) {
        u64 kz[2] = {0, 0}, kx[2] = {0, 0};
        memcpy(kz, (const char *)z + i * nw * 8, nw * 8);
        memcpy(kx, (const char *)x + i * nw * 8, nw * 8);
        owner[i] = (int32_t)(nw == 1 ? bk_owner<1>(kz, kx, rows, rank_bits) : bk_owner<2>(kz, kx, rows, rank_bits));
    }
    return PP_OK;
}

template <int NW>
static int shard_begin_impl(pp_spv *h, int bits, int32_t *maxcnt) {
    TRY(ensure_dense(h));
    TRY(bk_rows_init(h));
    DevState st;
    TRY(read_state(h, &st));
    int cur = 0;
    const int rr = bk_reserve<NW>(h, bits, &cur, -1);
    if (rr == BK_NOFIT) return fail(PP_OUT_OF_MEMORY, "the bucket layout of this shard does not fit in device memory");
    if (rr) return rr;
    int mx = 0;
    TRY(bk_scatter<NW>(h, h->z[st.cur], h->x[st.cur], h->c[st.cur], st.n, -1, 0, 0, bits, &mx));
    if (mx < 0) mx = h->bk_cap + 1;       // a full bucket: more buckets needed
    TRY(shard_fcnt(h));
    *maxcnt = mx;
    return PP_OK;
}

extern "C" int pp_shard_begin(pp_spv *h, int32_t rank_bits, int32_t rank, const void *gz, const void *gx,
                              const double *cosv, const double *sinv, int64_t L, const pp_evolve_opts *opts,
                              int32_t bits, int32_t *maxcnt) {
    if (!h || !maxcnt) return fail(PP_ARGUMENT_ERROR, "null argument");
    if (rank_bits < 0 || rank_bits > 8 || rank < 0 || rank >= (1 << rank_bits))
        return fail(PP_ARGUMENT_ERROR, "need rank_bits in 0..8 and 0 <= rank < 2^rank_bits");
    if (bits < 1 || bits + rank_bits > BK_ROWS) return fail(PP_ARGUMENT_ERROR, "need 1 <= bits <= 26 - rank_bits");
    if (L < 1 || !gz || !gx || !cosv || !sinv) return fail(PP_ARGUMENT_ERROR, "need L >= 1 generators");
    if (h->batch_on) return fail(PP_ARGUMENT_ERROR, "a batched handle cannot be a shard");
    pp_evolve_opts O;
    memset(&O, 0, sizeof O);
    O.window = 1;
    O.chan_kind = -1;
    if (opts) O = *opts;
    if (O.window != 1 || O.strict_kind != 0 || O.corr_kind != 0 || O.counters)
        return fail(PP_NOT_IMPLEMENTED, "key-sharded runs take window 1, a compiled truncation, no correction and "
                                        "no WindowCounters");
    DevParams *P = h->Ph;
    compile_filter(O.strict, &P->strict);
    compile_filter(O.local, &P->local);
    P->local_active = filter_is_nofilter(O.local) ? 0 : 1;
    P->corr_kind = 0;
    load_word(O.ket, h->NW, P->ket);
    P->chan_kind = -1;
    if (O.chan_kind >= 0) TRY(build_channel(h, O.chan_kind, O.chan_prm, O.chan_mask, P));
    TRY(upload_params(h));
    TRY(ensure_gens(h, L));
    std::vector<GenRec> G((size_t)L);
    const size_t wb = (size_t)h->NW * 8;
    for (long long i = 0; i < L; ++i) {
        u64 wz[2] = {0, 0}, wx[2] = {0, 0};
        memcpy(wz, (const char *)gz + i * wb, wb);
        memcpy(wx, (const char *)gx + i * wb, wb);
        bool stc = true;
        make_gen(h, wz, wx, cosv[i], sinv[i], &G[i], &stc);
    }
    if (O.chan_kind >= 0) {
        if (O.chan_every > 0) {
            for (long long i = O.chan_every - 1; i < L; i += O.chan_every) G[i].flags |= GEN_CHANNEL;
        } else {
            G[L - 1].flags |= GEN_CHANNEL;
        }
    }
    memcpy(h->gens_h, G.data(), L * sizeof(GenRec));
    CU(cudaMemcpyAsync(h->gens, h->gens_h, L * sizeof(GenRec), cudaMemcpyHostToDevice, h->stream));
    DevState st;
    TRY(read_state(h, &st));
    st.rot = 0;
    st.rot_end = L;
    st.created = st.merge_in = st.merge_out = st.early = 0;
    st.npref = st.live_in = st.peak = 0;
    st.measure_valid = 0;
    st.err = 0;
    TRY(write_state(h, &st));
    if (L + 1 > h->bk_rec_cap) {
        TRY(dalloc(h, &h->bk_rec, L + 1));
        h->bk_rec_cap = L + 1;
    }
    {
        BkRec r0;
        memset(&r0, 0, sizeof r0);
        r0.n_in = st.n;
        r0.n_out = (unsigned long long)st.n;
        r0.acap = 1ll << 62;
        CU(cudaMemcpyAsync(h->bk_rec, &r0, sizeof r0, cudaMemcpyHostToDevice, h->stream));
        CU(cudaMemsetAsync(h->bk_rec + 1, 0, L * sizeof(BkRec), h->stream));
    }
    if (!h->shard_cnt) TRY(dalloc(h, &h->shard_cnt, 1));
    TRY(h->NW == 1 ? shard_begin_impl<1>(h, bits, maxcnt) : shard_begin_impl<2>(h, bits, maxcnt));
    h->shard_on = true;
    h->shard_rank_bits = rank_bits;
    h->shard_rank = rank;
    h->shard_cur = 0;
    h->shard_bits = bits;
    h->shard_L = L;
    return PP_OK;
}

static int shard_partner(pp_spv *h, int64_t r, int32_t *partner) {
    if (!h->shard_on) return fail(PP_ARGUMENT_ERROR, "no key-sharded run in progress (pp_shard_begin)");
    if (r < 0 || r >= h->shard_L) return fail(PP_ARGUMENT_ERROR, "rotation index out of range");
    u64 rows[BK_ROWS * 4];
    bk_rows_host(rows);
    const GenRec &g = h->gens_h[r];
    const unsigned o = h->NW == 1 ? bk_owner<1>(g.gz, g.gx, rows, h->shard_rank_bits)
                                  : bk_owner<2>(g.gz, g.gx, rows, h->shard_rank_bits);
    *partner = h->shard_rank ^ (int32_t)o;
    return PP_OK;
}

extern "C" int pp_shard_send(pp_spv *h, int64_t r, int32_t pref, void *zout, void *xout, double *cout, int64_t cap,
                             int64_t *n_out, int32_t *partner) {
    if (!h || !n_out || !partner) return fail(PP_ARGUMENT_ERROR, "null argument");
    TRY(shard_partner(h, r, partner));
    *n_out = 0;
    if (*partner == h->shard_rank) return PP_OK;
    if (cap > 0 && (!zout || !xout || !cout)) return fail(PP_ARGUMENT_ERROR, "null output buffer");
    cudaStream_t s = h->stream;
    CU(cudaMemsetAsync(h->shard_cnt, 0, sizeof(unsigned long long), s));
    const int cur = h->shard_cur, bits = h->shard_bits, cap_b = h->bk_cap;
    const long long slots = (long long)cap_b << bits;
    const int grid = (int)std::max(1ll, std::min((slots + 255) / 256, (long long)h->nsm * 16));
    if (h->NW == 1)
        k_bk_send<1><<<grid, 256, 0, s>>>(h->bkz[cur], h->bkx[cur], h->bkc[cur], h->bkcnt[cur], bits, cap_b,
                                          h->gens + r, pref ? 1 : 0, h->P, (u64 *)zout, (u64 *)xout, cout, cap,
                                          h->shard_cnt, h->S);
    else
        k_bk_send<2><<<grid, 256, 0, s>>>(h->bkz[cur], h->bkx[cur], h->bkc[cur], h->bkcnt[cur], bits, cap_b,
                                          h->gens + r, pref ? 1 : 0, h->P, (u64 *)zout, (u64 *)xout, cout, cap,
                                          h->shard_cnt, h->S);
    unsigned long long n = 0;
    CU(cudaMemcpyAsync(&n, h->shard_cnt, sizeof n, cudaMemcpyDeviceToHost, s));
    TRY(sync_check(h));
    DevState st;
    TRY(read_state(h, &st));
    if (st.err & ERR_OVERFLOW) {
        st.err &= ~ERR_OVERFLOW;
        TRY(write_state(h, &st));
        return fail(PP_OUT_OF_MEMORY, "pp_shard_send: " + std::to_string(n) + " terms to send, buffer holds " +
                                          std::to_string(cap));
    }
    TRY(check_err(h, st));
    *n_out = (int64_t)n;
    return PP_OK;
}

extern "C" int pp_shard_recv(pp_spv *h, const void *z, const void *x, const double *c, int64_t n) {
    if (!h) return fail(PP_ARGUMENT_ERROR, "null handle");
    if (!h->shard_on) return fail(PP_ARGUMENT_ERROR, "no key-sharded run in progress (pp_shard_begin)");
    if (n < 0 || (n > 0 && (!z || !x || !c))) return fail(PP_ARGUMENT_ERROR, "need n >= 0 received terms");
    if (n == 0) return PP_OK;
    cudaStream_t s = h->stream;
    const int cur = h->shard_cur, bits = h->shard_bits;
    const int grid = (int)std::max(1ll, std::min((long long)(n + 255) / 256, (long long)h->nsm * 16));
    if (h->NW == 1)
        k_bk_absorb<1><<<grid, 256, 0, s>>>((const u64 *)z, (const u64 *)x, c, n, h->bkz[cur], h->bkx[cur], h->bkc[cur],
                                            h->bkcnt[cur], h->bkfcnt[cur], bits, h->bk_cap, h->bk_rows, h->S);
    else
        k_bk_absorb<2><<<grid, 256, 0, s>>>((const u64 *)z, (const u64 *)x, c, n, h->bkz[cur], h->bkx[cur], h->bkc[cur],
                                            h->bkcnt[cur], h->bkfcnt[cur], bits, h->bk_cap, h->bk_rows, h->S);
    TRY(sync_check(h));
    DevState st;
    TRY(read_state(h, &st));
    if (st.err & ERR_OVERFLOW) return fail(PP_OUT_OF_MEMORY, "pp_shard_recv: a bucket would exceed its capacity");
    return check_err(h, st);
}

template <int NW>
static int shard_rotate_impl(pp_spv *h, int64_t r, int pref, int remote, int64_t *out) {
    const BkVariant *var = bk_variant(h->tune.bucket_cap, h->tune.items_per_thread);
    if (!var || var->cap != h->bk_cap) return fail(PP_ERROR_EXCEPTION, "internal error: bucket variant changed");
    cudaStream_t s = h->stream;
    BkArgs A = bk_args(h, var, h->shard_bits, h->bk_rec);
    A.fcnt[0] = h->bkfcnt[0];
    A.fcnt[1] = h->bkfcnt[1];
    A.remote = remote;
    A.pref_forced = pref ? 1 : 0;
    k_bk_begin<<<1, 1, 0, s>>>(h->S, r, h->shard_cur, 1);
    bk_launch<NW>(h, var, A, 0);
    BkRec o;
    CU(cudaMemcpyAsync(&o, h->bk_rec + r + 1, sizeof o, cudaMemcpyDeviceToHost, s));
    TRY(sync_check(h));
    DevState st;
    TRY(read_state(h, &st));
    if (st.err & ERR_OVERFLOW) return fail(PP_OUT_OF_MEMORY, "pp_shard_rotate: a bucket would exceed its capacity");
    TRY(check_err(h, st));
    h->shard_cur ^= 1;
    st.live_in += o.n_in;
    st.created += (long long)o.created;
    st.merge_in += o.n_in + (long long)o.created;
    st.merge_out += (long long)o.n_out;
    if ((long long)o.n_out > st.peak) st.peak = (long long)o.n_out;
    if (pref) st.early += 1;
    st.rot = r + 1;
    TRY(write_state(h, &st));
    out[0] = o.n_in;
    out[1] = (int64_t)o.n_out;
    out[2] = (int64_t)o.created;
    out[3] = (int64_t)o.np;
    out[4] = o.maxcnt;
    return PP_OK;
}

extern "C" int pp_shard_rotate(pp_spv *h, int64_t r, int32_t pref, int64_t *stats5) {
    if (!h || !stats5) return fail(PP_ARGUMENT_ERROR, "null argument");
    int32_t partner = 0;
    TRY(shard_partner(h, r, &partner));
    const int remote = partner != h->shard_rank ? 1 : 0;
    return h->NW == 1 ? shard_rotate_impl<1>(h, r, pref, remote, stats5) : shard_rotate_impl<2>(h, r, pref, remote, stats5);
}

template <int NW>
static int shard_regrid_impl(pp_spv *h, int bits, int32_t *maxcnt) {
    int cur = h->shard_cur;
    const int rr = bk_reserve<NW>(h, bits, &cur, h->shard_bits);
    if (rr == BK_NOFIT) return fail(PP_OUT_OF_MEMORY, "the bucket layout of this shard does not fit in device memory");
    if (rr) return rr;
    int mx = 0;
    TRY(bk_scatter<NW>(h, h->bkz[cur], h->bkx[cur], h->bkc[cur], 0, cur, h->shard_bits, cur ^ 1, bits, &mx));
    if (mx < 0) mx = h->bk_cap + 1;
    h->shard_cur = cur ^ 1;
    h->shard_bits = bits;
    TRY(shard_fcnt(h));
    *maxcnt = mx;
    return PP_OK;
}

extern "C" int pp_shard_regrid(pp_spv *h, int32_t bits, int32_t *maxcnt) {
    if (!h || !maxcnt) return fail(PP_ARGUMENT_ERROR, "null argument");
    if (!h->shard_on) return fail(PP_ARGUMENT_ERROR, "no key-sharded run in progress (pp_shard_begin)");
    if (bits < 1 || bits + h->shard_rank_bits > BK_ROWS) return fail(PP_ARGUMENT_ERROR, "need 1 <= bits <= 26 - rank_bits");
    return h->NW == 1 ? shard_regrid_impl<1>(h, bits, maxcnt) : shard_regrid_impl<2>(h, bits, maxcnt);
}

extern "C" int pp_shard_end(pp_spv *h, double *expect_partial, double *stats_out) {
    if (!h) return fail(PP_ARGUMENT_ERROR, "null handle");
    if (!h->shard_on) return fail(PP_ARGUMENT_ERROR, "no key-sharded run in progress (pp_shard_begin)");
    h->shard_on = false;
    TRY(h->NW == 1 ? bk_to_dense<1>(h, h->shard_cur, h->shard_bits) : bk_to_dense<2>(h, h->shard_cur, h->shard_bits));
    double ev = 0.0;
    TRY(expect_dev(h, h->Ph->ket, &ev));
    DevState st;
    TRY(read_state(h, &st));
    st.expect_val = ev;
    st.measure_valid = 1;
    TRY(write_state(h, &st));
    if (expect_partial) *expect_partial = ev;
    if (stats_out) {
        for (int i = 0; i < PP_STATS_LEN; ++i) stats_out[i] = 0.0;
        stats_out[PP_STAT_TERMS_IN] = (double)st.live_in;
        stats_out[PP_STAT_CREATED] = (double)st.created;
        stats_out[PP_STAT_MERGE_IN] = (double)st.merge_in;
        stats_out[PP_STAT_MERGE_OUT] = (double)st.merge_out;
        stats_out[PP_STAT_PEAK] = (double)st.peak;
        stats_out[PP_STAT_EARLY] = (double)st.early;
    }
    return PP_OK;
}

// ------------------------------------------------------------------ learned truncation
static_assert(sizeof(pp_feature_ctx) == sizeof(FeatCtx), "pp_feature_ctx mirrors FeatCtx");
static_assert(PP_MLP_NPARAM == MLP_NPARAM, "parameter count");

struct pp_mlp {
    int dev = 0, nsm = 148;
    cudaStream_t stream = nullptr;
    MlpDev *W = nullptr;
    float *p = nullptr, *m = nullptr, *v = nullptr, *g = nullptr;   // master params, Adam moments, grad (+loss)
    float *gpart = nullptr;
    float *feat = nullptr, *target = nullptr, *out = nullptr;
    long long ndata = 0, data_cap = 0, out_cap = 0;
    int *idx = nullptr;
    long long idx_cap = 0;
    float *loss_log = nullptr;
    long long loss_cap = 0;
    FeatCtx *ctx = nullptr;
    int *err = nullptr;
    long long step = 0;
    // selection workspaces (used with a pp_spv's stream)
    float *score = nullptr;
    long long score_cap = 0;
    SelectState *sel = nullptr;
    int *cgt = nullptr, *ceq = nullptr, *tie_off = nullptr, *out_off = nullptr;
    long long *total = nullptr;
    long long tiles_cap = 0;
};

#define MCU(call)                                                                            \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(e_ == cudaErrorMemoryAllocation ? PP_OUT_OF_MEMORY : PP_DEVICE_ERROR, \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                 \
    } while (0)

// New buffer first, then the old one freed: a failure leaves *p as it was.
template <typename T>
static int malloc_n(T **p, long long n) {
    T *q = nullptr;
    MCU(cudaMalloc((void **)&q, (size_t)std::max(1ll, n) * sizeof(T)));
    if (*p) cudaFree(*p);
    *p = q;
    return PP_OK;
}

static int mlp_check(pp_mlp *m) {
    MCU(cudaStreamSynchronize(m->stream));
    int e = 0;
    MCU(cudaMemcpy(&e, m->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        cudaMemset(m->err, 0, sizeof(int));
        return fail(e & ERR_TIMEOUT ? PP_TIMEOUT : PP_ERROR_EXCEPTION, "learned-truncation kernel error flag set");
    }
    return PP_OK;
}

extern "C" int pp_mlp_create(pp_mlp **out) {
    if (!out) return fail(PP_ARGUMENT_ERROR, "null argument");
    pp_mlp *m = new pp_mlp();
    auto bail = [&](int r) { pp_mlp_destroy(m); return r; };
    int r;
    if (cudaGetDevice(&m->dev) != cudaSuccess) return bail(fail(PP_DEVICE_ERROR, "no CUDA device"));
    cudaDeviceGetAttribute(&m->nsm, cudaDevAttrMultiProcessorCount, m->dev);
    if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(PP_DEVICE_ERROR, "stream"));
    if ((r = malloc_n(&m->W, 1)) || (r = malloc_n(&m->p, MLP_NPARAM)) || (r = malloc_n(&m->m, MLP_NPARAM)) ||
        (r = malloc_n(&m->v, MLP_NPARAM)) || (r = malloc_n(&m->g, MLP_NPARAM + 1)) ||
        (r = malloc_n(&m->gpart, (long long)m->nsm * (MLP_NPARAM + 1))) || (r = malloc_n(&m->ctx, 1)) ||
        (r = malloc_n(&m->err, 1)) || (r = malloc_n(&m->sel, 1)) || (r = malloc_n(&m->total, 1)))
        return bail(r);
    cudaMemset(m->W, 0, sizeof(MlpDev));
    cudaMemset(m->p, 0, MLP_NPARAM * 4);
    cudaMemset(m->m, 0, MLP_NPARAM * 4);
    cudaMemset(m->v, 0, MLP_NPARAM * 4);
    cudaMemset(m->err, 0, 4);
    if (cudaFuncSetAttribute(k_mlp_fwd<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MLP_FWD_SMEM) ||
        cudaFuncSetAttribute(k_mlp_fwd<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MLP_FWD_SMEM) ||
        cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MLP_GRAD_SMEM))
        return bail(fail(PP_DEVICE_ERROR, "cudaFuncSetAttribute (shared memory)"));
    if (cudaDeviceSynchronize() != cudaSuccess) return bail(fail(PP_DEVICE_ERROR, "device"));
    *out = m;
    return PP_OK;
}

extern "C" int pp_mlp_destroy(pp_mlp *m) {
    if (!m) return PP_OK;
    if (m->stream) cudaStreamSynchronize(m->stream);
    void *ptrs[] = {m->W, m->p, m->m, m->v, m->g, m->gpart, m->feat, m->target, m->out, m->idx, m->loss_log,
                    m->ctx, m->err, m->score, m->sel, m->cgt, m->ceq, m->tie_off, m->out_off, m->total};
    for (void *q : ptrs) if (q) cudaFree(q);
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return PP_OK;
}

extern "C" int pp_mlp_set_params(pp_mlp *m, const float *params) {
    if (!m || !params) return fail(PP_ARGUMENT_ERROR, "null argument");
    MCU(cudaMemcpyAsync(m->p, params, MLP_NPARAM * 4, cudaMemcpyDefault, m->stream));
    MCU(cudaMemsetAsync(m->m, 0, MLP_NPARAM * 4, m->stream));
    MCU(cudaMemsetAsync(m->v, 0, MLP_NPARAM * 4, m->stream));
    k_mlp_set<<<(MLP_NPARAM + 255) / 256, 256, 0, m->stream>>>(m->p, m->W);
    m->step = 0;
    return mlp_check(m);
}

extern "C" int pp_mlp_get_params(pp_mlp *m, float *params) {
    if (!m || !params) return fail(PP_ARGUMENT_ERROR, "null argument");
    MCU(cudaMemcpyAsync(params, m->p, MLP_NPARAM * 4, cudaMemcpyDefault, m->stream));
    return mlp_check(m);
}

static int mlp_stage(pp_mlp *m, const float *feat, const float *target, long long n) {
    if (n > m->data_cap) {
        TRY(malloc_n(&m->feat, n * MLP_F));
        TRY(malloc_n(&m->target, n));
        m->data_cap = n;
    }
    if (n > 0) {
        MCU(cudaMemcpyAsync(m->feat, feat, n * MLP_F * 4, cudaMemcpyDefault, m->stream));
        if (target) MCU(cudaMemcpyAsync(m->target, target, n * 4, cudaMemcpyDefault, m->stream));
    }
    m->ndata = n;
    return PP_OK;
}

extern "C" int pp_mlp_forward(pp_mlp *m, const float *feat, int64_t n, float *out) {
    if (!m || n < 0 || (n > 0 && (!feat || !out))) return fail(PP_ARGUMENT_ERROR, "bad argument");
    TRY(mlp_stage(m, feat, nullptr, n));
    if (n > m->out_cap) {
        TRY(malloc_n(&m->out, n));
        m->out_cap = n;
    }
    if (n == 0) return PP_OK;
    const long long tiles = (n + MLP_ROWS - 1) / MLP_ROWS;
    const int grid = (int)std::min<long long>(tiles, 4ll * m->nsm);
    k_mlp_fwd<0><<<grid, MLP_ROWS, MLP_FWD_SMEM, m->stream>>>(m->feat, nullptr, nullptr, nullptr, n, nullptr, m->W,
                                                              m->out, nullptr, m->err);
    MCU(cudaGetLastError());
    MCU(cudaMemcpyAsync(out, m->out, n * 4, cudaMemcpyDefault, m->stream));
    return mlp_check(m);
}

// One gradient of mean((y - t)^2) over idx[0, B) of the staged data into m->g.
static int mlp_grad_launch(pp_mlp *m, const int *idx, long long B) {
    const long long tiles = (B + MLP_ROWS - 1) / MLP_ROWS;
    const int grid = (int)std::min<long long>(tiles, m->nsm);
    k_mlp_grad<<<grid, MLP_ROWS, MLP_GRAD_SMEM, m->stream>>>(m->feat, m->target, idx, B, m->W, m->gpart, m->err);
    k_mlp_reduce<<<(MLP_NPARAM + 1 + 255) / 256, 256, 0, m->stream>>>(m->gpart, grid, m->g);
    MCU(cudaGetLastError());
    return PP_OK;
}

static int mlp_ensure_idx(pp_mlp *m, long long n) {
    if (n > m->idx_cap) {
        TRY(malloc_n(&m->idx, n));
        m->idx_cap = n;
    }
    return PP_OK;
}

extern "C" int pp_mlp_grad(pp_mlp *m, const float *feat, const float *target, int64_t n, float *grad, float *loss) {
    if (!m || n <= 0 || !feat || !target || !grad) return fail(PP_ARGUMENT_ERROR, "bad argument");
    if (n > (1ll << 31) - 1) return fail(PP_ARGUMENT_ERROR, "n too large");
    TRY(mlp_stage(m, feat, target, n));
    TRY(mlp_ensure_idx(m, n));
    std::vector<int> id((size_t)n);
    for (long long i = 0; i < n; ++i) id[i] = (int)i;
    MCU(cudaMemcpyAsync(m->idx, id.data(), n * 4, cudaMemcpyHostToDevice, m->stream));
    TRY(mlp_grad_launch(m, m->idx, n));
    std::vector<float> g(MLP_NPARAM + 1);
    MCU(cudaMemcpyAsync(g.data(), m->g, (MLP_NPARAM + 1) * 4, cudaMemcpyDeviceToHost, m->stream));
    TRY(mlp_check(m));
    memcpy(grad, g.data(), MLP_NPARAM * 4);
    if (loss) *loss = g[MLP_NPARAM] / (float)n;
    return PP_OK;
}

extern "C" int pp_mlp_load_data(pp_mlp *m, const float *feat, const float *target, int64_t n) {
    if (!m || n <= 0 || !feat || !target) return fail(PP_ARGUMENT_ERROR, "bad argument");
    if (n > (1ll << 31) - 1) return fail(PP_ARGUMENT_ERROR, "n too large");
    TRY(mlp_stage(m, feat, target, n));
    return mlp_check(m);
}

static inline uint64_t splitmix64(uint64_t *s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

extern "C" int pp_mlp_train(pp_mlp *m, int64_t steps, int64_t batch, float lr, uint64_t seed, float *loss_out) {
    if (!m || steps < 0 || batch < 1 || !(lr > 0.0f)) return fail(PP_ARGUMENT_ERROR, "bad argument");
    const long long nd = m->ndata;
    if (nd < 1) return fail(PP_ARGUMENT_ERROR, "no training data loaded (pp_mlp_load_data)");
    batch = std::min<long long>(batch, nd);
    TRY(mlp_ensure_idx(m, nd));
    if (steps > m->loss_cap) {
        TRY(malloc_n(&m->loss_log, steps));
        m->loss_cap = steps;
    }
    std::vector<int> perm((size_t)nd);
    for (long long i = 0; i < nd; ++i) perm[i] = (int)i;
    uint64_t st = seed;
    long long pos = nd;   // forces a shuffle first
    for (long long s = 0; s < steps; ++s) {
        if (pos + batch > nd) {
            for (long long i = nd - 1; i > 0; --i) std::swap(perm[i], perm[splitmix64(&st) % (uint64_t)(i + 1)]);
            MCU(cudaMemcpyAsync(m->idx, perm.data(), nd * 4, cudaMemcpyHostToDevice, m->stream));
            MCU(cudaStreamSynchronize(m->stream));
            pos = 0;
        }
        TRY(mlp_grad_launch(m, m->idx + pos, batch));
        m->step += 1;
        k_mlp_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, m->stream>>>(m->p, m->m, m->v, m->g, (int)m->step, lr, m->W,
                                                                    m->loss_log + s, batch);
        pos += batch;
    }
    MCU(cudaGetLastError());
    if (loss_out && steps > 0) MCU(cudaMemcpyAsync(loss_out, m->loss_log, steps * 4, cudaMemcpyDeviceToHost, m->stream));
    return mlp_check(m);
}

extern "C" int pp_features(pp_spv *h, const pp_feature_ctx *ctx, float *out, int64_t cap, int64_t *n_out) {
    if (!h || !ctx || !n_out) return fail(PP_ARGUMENT_ERROR, "null argument");
    if (h->NW != 1) return fail(PP_ARGUMENT_ERROR, "term features need N <= 64");
    DevState st;
    TRY(read_state(h, &st));
    *n_out = st.n;
    const long long n = std::min<long long>(st.n, std::max<int64_t>(cap, 0));
    if (n == 0) return PP_OK;
    if (!out) return fail(PP_ARGUMENT_ERROR, "null output");
    FeatCtx *dctx = nullptr;
    float *dout = nullptr;
    CU(cudaMalloc((void **)&dctx, sizeof(FeatCtx)));
    cudaError_t e = cudaMalloc((void **)&dout, (size_t)n * MLP_F * 4);
    if (e != cudaSuccess) { cudaFree(dctx); return fail(PP_OUT_OF_MEMORY, "features buffer"); }
    cudaMemcpyAsync(dctx, ctx, sizeof(FeatCtx), cudaMemcpyHostToDevice, h->stream);
    k_features<<<h->nsm * 8, 256, 0, h->stream>>>(h->z[st.cur], h->x[st.cur], h->c[st.cur], n, dctx, dout);
    e = cudaMemcpyAsync(out, dout, (size_t)n * MLP_F * 4, cudaMemcpyDefault, h->stream);
    cudaStreamSynchronize(h->stream);
    cudaFree(dctx);
    cudaFree(dout);
    if (e != cudaSuccess) return fail(PP_DEVICE_ERROR, cudaGetErrorString(e));
    return sync_check(h);
}

extern "C" int pp_learned_truncate(pp_spv *h, pp_mlp *m, const pp_feature_ctx *ctx, int64_t budget,
                                   float *cut_score, pp_drop_sample *sample) {
    if (!h || !m || !ctx || budget < 0) return fail(PP_ARGUMENT_ERROR, "bad argument");
    if (h->NW != 1) return fail(PP_ARGUMENT_ERROR, "learned truncation needs N <= 64");
    DevState st;
    TRY(read_state(h, &st));
    if (cut_score) *cut_score = -INFINITY;
    const long long n = st.n;
    if (sample) {
        sample->n = 0;
        sample->n_dropped = std::max(0ll, n - (long long)budget);
        if (sample->cap < 0 || (sample->cap > 0 && (!sample->z || !sample->x || !sample->c)))
            return fail(PP_ARGUMENT_ERROR, "bad drop-sample buffers");
    }
    if (n <= budget) return PP_OK;
    MCU(cudaStreamSynchronize(m->stream));   // the network's last update is visible to h's stream
    if (n > m->score_cap) {
        TRY(malloc_n(&m->score, n));
        m->score_cap = n;
    }
    const long long ntiles = (n + SL_TILE - 1) / SL_TILE;
    if (ntiles > m->tiles_cap) {
        TRY(malloc_n(&m->cgt, ntiles));
        TRY(malloc_n(&m->ceq, ntiles));
        TRY(malloc_n(&m->tie_off, ntiles));
        TRY(malloc_n(&m->out_off, ntiles));
        m->tiles_cap = ntiles;
    }
    cudaStream_t s = h->stream;
    SelectState s0;
    memset(&s0, 0, sizeof s0);
    s0.remaining = budget;
    CU(cudaMemcpyAsync(m->ctx, ctx, sizeof(FeatCtx), cudaMemcpyHostToDevice, s));
    CU(cudaMemcpyAsync(m->sel, &s0, sizeof s0, cudaMemcpyHostToDevice, s));
    const int cur = st.cur;
    const long long rtiles = (n + MLP_ROWS - 1) / MLP_ROWS;
    k_mlp_fwd<1><<<(int)std::min<long long>(rtiles, 4ll * m->nsm), MLP_ROWS, MLP_FWD_SMEM, s>>>(
        nullptr, h->z[cur], h->x[cur], h->c[cur], n, m->ctx, m->W, m->score, m->sel, m->err);
    k_sel_pick<<<1, 32, 0, s>>>(m->sel, 24);
    for (int shift = 16; shift >= 0; shift -= 8) {
        k_sel_hist<<<h->nsm * 4, 256, 0, s>>>(m->score, n, m->sel, shift);
        k_sel_pick<<<1, 32, 0, s>>>(m->sel, shift);
    }
    const int g = (int)std::min<long long>(ntiles, 8ll * h->nsm);
    k_sel_count<<<g, SL_THREADS, 0, s>>>(m->score, n, m->sel, m->cgt, m->ceq);
    k_sel_scan<<<1, 1024, 0, s>>>(ntiles, m->sel, m->cgt, m->ceq, m->tie_off, m->out_off, m->total);
    k_sel_write<<<g, SL_THREADS, 0, s>>>(m->score, n, m->sel, m->tie_off, m->out_off, h->z[cur], h->x[cur], h->c[cur],
                                         h->z[cur ^ 1], h->x[cur ^ 1], h->c[cur ^ 1]);
    Scratch sample_buf;             // the drop sample's device buffer, freed on every return
    u64 *sbuf = nullptr;
    unsigned long long *scnt = nullptr;
    long long scap = sample ? sample->cap : 0;
    if (scap > 0) {
        // acceptance probability 0.9 cap / dropped keeps the sample under its cap
        const double pacc = std::min(1.0, 0.9 * (double)scap / (double)(n - budget));
        const unsigned long long thr =
            pacc >= 1.0 ? ~0ull : (unsigned long long)(pacc * 18446744073709551616.0);
        TRY(sample_buf.get(&sbuf, 3 * scap + 1));     // z, x, c words of the sample, then its counter
        scnt = reinterpret_cast<unsigned long long *>(sbuf + 3 * scap);
        CU(cudaMemsetAsync(scnt, 0, 8, s));
        k_sel_sample<<<h->nsm * 4, 256, 0, s>>>(m->score, n, m->sel, sample->seed, thr, h->z[cur], h->x[cur],
                                               h->c[cur], sbuf, sbuf + scap, reinterpret_cast<double *>(sbuf + 2 * scap),
                                               scap, scnt);
    }
    CU(cudaGetLastError());
    long long kept = 0;
    SelectState sf;
    CU(cudaMemcpyAsync(&kept, m->total, sizeof kept, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(&sf, m->sel, sizeof sf, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (scap > 0) {
        unsigned long long got = 0;
        cudaMemcpy(&got, scnt, 8, cudaMemcpyDeviceToHost);
        const long long ns = std::min<long long>((long long)got, scap);
        cudaMemcpy(sample->z, sbuf, ns * 8, cudaMemcpyDefault);
        cudaMemcpy(sample->x, sbuf + scap, ns * 8, cudaMemcpyDefault);
        cudaMemcpy(sample->c, sbuf + 2 * scap, ns * 8, cudaMemcpyDefault);
        sample->n = ns;
    }
    int e = 0;
    CU(cudaMemcpy(&e, m->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        cudaMemset(m->err, 0, sizeof(int));
        return fail(PP_TIMEOUT, "learned truncation: a tensor-core wait timed out");
    }
    if (kept != budget) return fail(PP_ERROR_EXCEPTION, "learned truncation kept a count other than the budget");
    TRY(read_state(h, &st));
    st.n = kept;
    st.cur ^= 1;
    TRY(write_state(h, &st));
    if (cut_score) {
        const uint32_t k = sf.prefix;
        const uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
        float f;
        memcpy(&f, &u, 4);
        *cut_score = f;
    }
    return PP_OK;
}

extern "C" int pp_sample_terms(pp_spv *h, int32_t nbins, double lg_lo, double lg_hi, int64_t per_bin, uint64_t seed,
                               void *z, void *x, double *c, int64_t cap, int64_t *n_out) {
    if (!h || !n_out || nbins < 1 || nbins > 64 || !(lg_hi > lg_lo) || per_bin < 0 || cap < 0 ||
        (cap > 0 && (!z || !x || !c)))
        return fail(PP_ARGUMENT_ERROR, "bad argument");
    if (h->NW != 1) return fail(PP_ARGUMENT_ERROR, "term sampling needs N <= 64");
    DevState st;
    TRY(read_state(h, &st));
    *n_out = 0;
    const long long n = st.n;
    if (n == 0 || cap == 0) return PP_OK;
    cudaStream_t s = h->stream;
    const int cur = st.cur;
    unsigned long long *dbuf = nullptr;
    CU(cudaMalloc((void **)&dbuf, (size_t)(2 * 64 + 1 + 3 * cap) * 8));
    unsigned long long *hist = dbuf, *thr = dbuf + 64, *cnt = dbuf + 128;
    u64 *sz = dbuf + 129, *sx = sz + cap;
    double *sc = reinterpret_cast<double *>(sx + cap);
    cudaMemsetAsync(dbuf, 0, 129 * 8, s);
    k_lgc_hist<<<h->nsm * 4, 256, 0, s>>>(h->c[cur], n, lg_lo, lg_hi, nbins, hist);
    unsigned long long hh[64], th[64];
    cudaMemcpyAsync(hh, hist, nbins * 8, cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { cudaFree(dbuf); return fail(PP_DEVICE_ERROR, cudaGetErrorString(e)); }
    // acceptance 0.9 per_bin / count keeps the sample under its cap with high probability
    for (int b = 0; b < nbins; ++b) {
        const double p = hh[b] ? std::min(1.0, 0.9 * (double)per_bin / (double)hh[b]) : 0.0;
        th[b] = p >= 1.0 ? ~0ull : (unsigned long long)(p * 18446744073709551616.0);
    }
    cudaMemcpyAsync(thr, th, nbins * 8, cudaMemcpyHostToDevice, s);
    k_lgc_sample<<<h->nsm * 4, 256, 0, s>>>(h->z[cur], h->x[cur], h->c[cur], n, lg_lo, lg_hi, nbins, thr, seed, sz,
                                             sx, sc, cap, cnt);
    unsigned long long got = 0;
    cudaMemcpyAsync(&got, cnt, 8, cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    const long long ns = std::min<long long>((long long)got, cap);
    if (e == cudaSuccess && ns > 0) {
        cudaMemcpy(z, sz, ns * 8, cudaMemcpyDefault);
        cudaMemcpy(x, sx, ns * 8, cudaMemcpyDefault);
        e = cudaMemcpy(c, sc, ns * 8, cudaMemcpyDefault);
    }
    cudaFree(dbuf);
    if (e != cudaSuccess) return fail(PP_DEVICE_ERROR, cudaGetErrorString(e));
    *n_out = ns;
    return PP_OK;
}

extern "C" int pp_variance(pp_spv *h, const void *ket, double *out) {
    if (!h || !out) return fail(PP_ARGUMENT_ERROR, "null argument");
    u64 k[2];
    load_word(ket, h->NW, k);
    return variance_dev(h, k, out);
}

extern "C" int pp_stochastic_clip(pp_spv *h, double epsilon, uint64_t seed) {
    if (!h) return fail(PP_ARGUMENT_ERROR, "null handle");
    return stoch_clip_apply(h, epsilon, seed);
}

extern "C" int pp_stochastic_sample(pp_spv *h, int64_t n_keep, uint64_t seed) {
    if (!h) return fail(PP_ARGUMENT_ERROR, "null handle");
    if (n_keep < 0) return fail(PP_ARGUMENT_ERROR, "n_keep must be >= 0");
    return stoch_sample_apply(h, n_keep, seed);
}

// ------------------------------------------------------------------ SPV algebra (spv_ops.jl), real coefficients
// Unfiltered merge of the handle's live set with the sorted run (VZ, VX, VC)[0, m)
// as its appends: equal keys summed live first, zeros kept (_merge_spv!(v, m,
// NOFILTER), spv_kernels.jl:326-386).
template <int NW>
static int merge_run(pp_spv *h, u64 *VZ, u64 *VX, double *VC, long long m) {
    DevState st;
    TRY(read_state(h, &st));
    TRY(ensure_live(h, st.n + m));
    DevParams *P = h->Ph;
    compile_filter(nullptr, &P->strict);
    P->corr_kind = 0;
    P->chan_kind = -1;
    TRY(upload_params(h));
    TRY(read_state(h, &st));
    st.an = m;
    TRY(write_state(h, &st));
    Bufs B = make_bufs(h);
    B.vz = VZ;
    B.vx = VX;
    B.vc = VC;
    launch_merge<NW, 1>(h, B, 0);
    TRY(sync_check(h));
    TRY(read_state(h, &st));
    return check_err(h, st);
}

static int same_kind(pp_spv *a, pp_spv *b) {
    if (!a || !b) return fail(PP_ARGUMENT_ERROR, "null handle");
    if (a->N != b->N) return fail(PP_DIMENSION_MISMATCH, "operands have different qubit counts");
    return PP_OK;
}

extern "C" int pp_scale(pp_spv *h, double a) {
    if (!h) return fail(PP_ARGUMENT_ERROR, "null handle");
    DevState st;
    TRY(read_state(h, &st));
    if (st.n > 0) k_scale<<<h->nsm * 8, 256, 0, h->stream>>>(h->c[st.cur], st.n, a);
    return sync_check(h);
}

extern "C" int pp_norm(pp_spv *h, double p, double *out) {
    if (!h || !out) return fail(PP_ARGUMENT_ERROR, "null argument");
    DevState st;
    TRY(read_state(h, &st));
    *out = 0.0;
    if (st.n == 0) return PP_OK;
    Scratch sc;
    const int nb = std::min(4096, h->nsm * 8);
    double *part, *res;
    TRY(sc.get(&part, nb));
    TRY(sc.get(&res, 1));
    cudaStream_t s = h->stream;
    const double *C = h->c[st.cur];
    if (std::isinf(p)) {
        k_absmax<<<nb, 256, 0, s>>>(C, st.n, part);
        k_max_final<<<1, 32, 0, s>>>(part, nb, res);
    } else {
        double *val;
        TRY(sc.get(&val, st.n));
        k_norm_terms<<<h->nsm * 8, 256, 0, s>>>(C, st.n, p, val);
        k_sum_partials<<<nb, 256, 0, s>>>(val, st.n, part);
        k_expect_final<<<1, 32, 0, s>>>(part, nb, res);
    }
    double r = 0.0;
    CU(cudaMemcpyAsync(&r, res, sizeof r, cudaMemcpyDeviceToHost, s));
    TRY(sync_check(h));
    *out = std::isinf(p) ? r : p == 2.0 ? std::sqrt(r) : p == 1.0 ? r : std::pow(r, 1.0 / p);
    return PP_OK;
}

extern "C" int pp_trace(pp_spv *h, double *out) {
    if (!h || !out) return fail(PP_ARGUMENT_ERROR, "null argument");
    DevState st;
    TRY(read_state(h, &st));
    // 2^N is the reference's Int64 power: it wraps for N >= 63
    const double pow2 = h->N < 63 ? std::ldexp(1.0, h->N) : h->N == 63 ? -std::ldexp(1.0, 63) : 0.0;
    *out = 0.0;
    if (st.n == 0) return PP_OK;
    u64 z[2] = {0, 0}, x[2] = {0, 0};
    double c = 0.0;
    CU(cudaMemcpyAsync(z, h->z[st.cur], h->NW * 8, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaMemcpyAsync(x, h->x[st.cur], h->NW * 8, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaMemcpyAsync(&c, h->c[st.cur], 8, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    if ((z[0] | z[1] | x[0] | x[1]) == 0) *out = c * pow2;
    return PP_OK;
}

extern "C" int pp_sum(pp_spv *h, pp_spv *o, double sign) {
    TRY(same_kind(h, o));
    if (sign != 1.0 && sign != -1.0) return fail(PP_ARGUMENT_ERROR, "sign must be +1 or -1");
    DevState so, sh;
    TRY(read_state(o, &so));
    TRY(read_state(h, &sh));
    if (sh.an != 0) return fail(PP_ERROR_EXCEPTION, "sum! on a SparsePauliVector with pending appends");
    const long long m = so.n;
    if (m == 0) return PP_OK;
    TRY(ensure_append(h, std::max(m, h->acap_phys), 0));
    TRY(cudaStreamSynchronize(o->stream) == cudaSuccess ? PP_OK : fail(PP_DEVICE_ERROR, "stream"));
    k_copy_terms<<<h->nsm * 8, 256, 0, h->stream>>>(o->z[so.cur], o->x[so.cur], o->c[so.cur], m, h->NW, sign, h->az,
                                                     h->ax, h->ac);
    return h->NW == 1 ? merge_run<1>(h, h->az, h->ax, h->ac, m) : merge_run<2>(h, h->az, h->ax, h->ac, m);
}

extern "C" int pp_inner_product(pp_spv *a, pp_spv *b, double *out) {
    TRY(same_kind(a, b));
    if (!out) return fail(PP_ARGUMENT_ERROR, "null argument");
    DevState sa, sb;
    TRY(read_state(a, &sa));
    TRY(read_state(b, &sb));
    *out = 0.0;
    if (sa.n == 0 || sb.n == 0) return PP_OK;
    CU(cudaStreamSynchronize(b->stream));
    Scratch sc;
    const int nb = std::min(4096, a->nsm * 8);
    double *val, *part, *res;
    TRY(sc.get(&val, sa.n));
    TRY(sc.get(&part, nb));
    TRY(sc.get(&res, 1));
    cudaStream_t s = a->stream;
    if (a->NW == 1)
        k_inner_terms<1><<<a->nsm * 8, 256, 0, s>>>(a->z[sa.cur], a->x[sa.cur], a->c[sa.cur], sa.n, b->z[sb.cur],
                                                     b->x[sb.cur], b->c[sb.cur], sb.n, val);
    else
        k_inner_terms<2><<<a->nsm * 8, 256, 0, s>>>(a->z[sa.cur], a->x[sa.cur], a->c[sa.cur], sa.n, b->z[sb.cur],
                                                     b->x[sb.cur], b->c[sb.cur], sb.n, val);
    k_sum_partials<<<nb, 256, 0, s>>>(val, sa.n, part);
    k_expect_final<<<1, 32, 0, s>>>(part, nb, res);
    CU(cudaMemcpyAsync(out, res, sizeof(double), cudaMemcpyDeviceToHost, s));
    return sync_check(a);
}

template <int NW>
static int product_nw(pp_spv *out, pp_spv *a, pp_spv *b, int kind) {
    DevState sa, sb;
    TRY(read_state(a, &sa));
    TRY(read_state(b, &sb));
    const long long tot = sa.n * sb.n;
    if (tot > 0x7fffffffll - 8192) return fail(PP_OUT_OF_MEMORY, "more than 2^31 term pairs");
    CU(cudaStreamSynchronize(a->stream));
    CU(cudaStreamSynchronize(b->stream));
    TRY(ensure_append(out, std::max(tot, out->acap_phys), 0));
    Scratch sc;
    unsigned char *keep;
    int *err;
    TRY(sc.get(&keep, tot));
    TRY(sc.get(&err, 1));
    cudaStream_t s = out->stream;
    CU(cudaMemsetAsync(err, 0, sizeof(int), s));
    if (tot > 0)
        k_pairs<NW><<<out->nsm * 8, 256, 0, s>>>(a->z[sa.cur], a->x[sa.cur], a->c[sa.cur], sa.n, b->z[sb.cur],
                                                  b->x[sb.cur], b->c[sb.cur], sb.n, kind, out->az, out->ax, out->ac,
                                                  keep, err);
    int e = 0;
    CU(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (e) return fail(PP_ERROR_EXCEPTION, "InexactError: the product has imaginary coefficients; "
                                           "use a complex coefficient type");
    // keep the surviving pairs in generation order (anticommutator), then sort stably by key
    u64 *PZ = out->az, *PX = out->ax;
    double *PC = out->ac;
    long long m = tot;
    if (kind == 1 && tot > 0) {
        const long long ntiles = (tot + FC_TILE - 1) / FC_TILE;
        int *cnt, *off;
        long long *total;
        TRY(sc.get(&cnt, ntiles));
        TRY(sc.get(&off, ntiles));
        TRY(sc.get(&total, 1));
        const int g = (int)std::min<long long>(ntiles, 8ll * out->nsm);
        k_flag_count<<<g, FC_THREADS, 0, s>>>(keep, tot, cnt);
        k_flag_scan<<<1, 1024, 0, s>>>(ntiles, cnt, off, total);
        k_flag_write<<<g, FC_THREADS, 0, s>>>(keep, tot, off, out->az, out->ax, out->ac, nullptr, NW, nullptr, out->tz,
                                              out->tx, out->tc);
        CU(cudaMemcpyAsync(&m, total, sizeof m, cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
        PZ = out->tz; PX = out->tx; PC = out->tc;
    }
    int in_t = 0;
    u64 *QZ = PZ == out->az ? out->tz : out->az, *QX = PX == out->ax ? out->tx : out->ax;
    double *QC = PC == out->ac ? out->tc : out->ac;
    TRY(radix_sort<NW>(out, PZ, PX, PC, QZ, QX, QC, m, &in_t));
    if (in_t) { PZ = QZ; PX = QX; PC = QC; }
    // result = the sorted triples summed by key (_triples_to_live!, spv_ops.jl:234-255)
    DevState so;
    TRY(read_state(out, &so));
    so.n = 0;
    so.an = 0;
    so.seg_dense = 1;
    TRY(write_state(out, &so));
    return merge_run<NW>(out, PZ, PX, PC, m);
}

extern "C" int pp_product(pp_spv *out, pp_spv *a, pp_spv *b, int32_t kind) {
    TRY(same_kind(a, b));
    TRY(same_kind(out, a));
    if (kind < 0 || kind > 2) return fail(PP_ARGUMENT_ERROR, "kind: 0 product, 1 anticommutator, 2 commutator");
    if (kind == 2)
        return fail(PP_ERROR_EXCEPTION, "commutator coefficients are imaginary; use a complex coefficient type "
                                        "(T=ComplexF64)");
    return out->NW == 1 ? product_nw<1>(out, a, b, kind) : product_nw<2>(out, a, b, kind);
}
