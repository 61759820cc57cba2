// gnss_b200.cu -- host side of the B200 pseudospectral step: context,
// launch orchestration and the C ABI declared in include/gnss_b200.h.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <type_traits>
#include <mutex>
#include <string>
#include <vector>

#include "gnss_b200.h"
#include "internal.h"
#include "kernels.cuh"
#include "zreg.cuh"
#include "passreg.cuh"
#include "passtc.cuh"
#include "diag.cuh"

using namespace gnss;

// ============================================================== context
struct gnss_ctx {
    gnss_config cfg{};
    Geom g{};
    size_t nspec = 0;       // complex elements per field
    size_t elem = 0;        // bytes per complex element
    void *tw[3] = {nullptr, nullptr, nullptr};   // twiddle tables for nx, ny, nz
    void *scratch = nullptr;                      // nscratch fields
    int nscratch = 0;
    bool scratch_ext = false;                     // scratch attached by the caller (not owned)
    double *stat_part = nullptr;                  // STAT_BLOCKS x STAT_SUMS
    double *stat_dev = nullptr;                   // STAT_SUMS
    double *stat_host = nullptr;                  // pinned STAT_SUMS
    double *turb_part = nullptr;                  // STAT_BLOCKS x TURB_SUMS (gnss_turb_stats)
    double *turb_dev = nullptr;                   // TURB_SUMS + 1 sums, then 5 * ny profile values
    double *turb_host = nullptr;                  // pinned copy of turb_dev
    void *res = nullptr;                          // resident state + history for gnss_run_host (2 * nf fields)
    double *run_sums = nullptr;                   // gnss_run_host: STAT_SUMS per step, summed by the update
    double *run_sums_host = nullptr;              // pinned copy of run_sums
    int run_sums_cap = 0;                         // steps run_sums holds
    cudaStream_t side = nullptr;                  // gnss_run_host: download of the modes outside the kept box
    cudaEvent_t side_ev[2] = {nullptr, nullptr};  // state ready / side copies done
    size_t owned_bytes = 0;
    // fused step layout (set_recipes): x-inverse outputs P, y-inverse outputs
    // (the raw quantities of the z pass) Q, physical quantities, products
    int n_xout = 0, n_raw = 0, n_phys = 0, nnl = 0;
    // kept box of the spherical truncation and the compact internal layouts:
    //   P fields [x][kept ky][ncp], Q fields [x][y][ncp], R (in Q) [kept ky][kept kx][ncp]
    KeepMap kx_keep{}, ky_keep{};
    int nkz = 0, ncp = 0;
    // kept Nyquist modes whose velocity the reference's transform round trip projects onto its Hermitian part
    // (k_herm): the ky Nyquist row and the kx Nyquist column of the kz = 0 plane, the kz = nz/2 plane
    int herm_row = 0, herm_col = 0, herm_plane = 0;
    size_t p_elems = 0, q_elems = 0;
    int zvariant = GNSS_VARIANT_AUTO;             // z kernel choice (gnss_set_option)
    int pvariant = GNSS_VARIANT_AUTO;             // x / y pass kernel choice
    long long n_sphere = 0;                       // kept-box modes inside the dealiasing sphere
    int n_xin = 0;                                // x-inverse inputs (state fields; s twice with alpha)
    signed char xvar_in[6]{}, xvar_n[6]{}, xvar_mul[6][2]{}, xvar_out[6][2]{};
    signed char yvar_n[MAXF]{}, yvar_mul[MAXF][2]{}, yvar_out[MAXF][2]{};
    ZRecipeSet zrec{};
    std::string err;
    long long launches = 0;                       // kernels launched by this context
    unsigned *d_err = nullptr;                    // [0] error word set by bounded waits that time out,
                                                  // [1] wait control (GNSS_OPT_TEST_WAIT; 0 normally)
    int test_wait = 0;                            // GNSS_OPT_TEST_WAIT
    double2 *mean64 = nullptr;                    // FP32 contexts: FP64 mean-profile line (kx = kz = 0) of the
                                                  // state and history, [2][5][ny] (k_update)
    int nsm = 148;                                // SMs of the device
    bool profiling = false;
    std::vector<cudaEvent_t> ev_pool;             // profiling events, reused
    std::vector<std::pair<int, std::pair<int, int>>> ev_rec;   // (stage, (start event, end event))
};

// Records an event pair around one stage launch when profiling is on.
struct StageTimer {
    gnss_ctx *c;
    cudaStream_t s;
    int stage, e0 = -1;
    StageTimer(gnss_ctx *c_, cudaStream_t s_, int st) : c(c_), s(s_), stage(st) {
        c->launches++;
        if (c->profiling) {
            e0 = take();
            cudaEventRecord(c->ev_pool[e0], s);
        }
    }
    ~StageTimer() {
        if (e0 >= 0) {
            int e1 = take();
            cudaEventRecord(c->ev_pool[e1], s);
            c->ev_rec.push_back({stage, {e0, e1}});
        }
    }
    int take() {
        size_t used = 2 * c->ev_rec.size() + (e0 >= 0 ? 1 : 0);
        while (c->ev_pool.size() <= used) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            c->ev_pool.push_back(e);
        }
        return (int)used;
    }
};

static gnss_status fail(gnss_ctx *c, gnss_status st, const char *fmt, ...) {
    if (c) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        c->err = buf;
    }
    return st;
}

#define CK(ctx, call)                                                                                  \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            return fail(ctx, GNSS_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),    \
                        __FILE__, __LINE__);                                                           \
    } while (0)

#define LAUNCH_CK(ctx)                                                                                 \
    do {                                                                                               \
        cudaError_t e_ = cudaGetLastError();                                                           \
        if (e_ != cudaSuccess)                                                                         \
            return fail(ctx, GNSS_ERR_CUDA, "kernel launch failed: %s (%s:%d)", cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                                           \
    } while (0)

static bool size_ok(int n) {
    switch (n) {
        case 8: case 12: case 16: case 24: case 32: case 48: case 64: case 96:
        case 128: case 192: case 256: case 384: case 512:
            return true;
        default:
            return false;
    }
}

static inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// every device pointer must be aligned to one complex element of the context
static bool al(const gnss_ctx *c, const void *p) {
    return p == nullptr || (reinterpret_cast<uintptr_t>(p) % c->elem) == 0;
}
static bool al_fields(const gnss_ctx *c, const gnss_fields *f) {
    return !f || (al(c, f->u) && al(c, f->v) && al(c, f->w) && al(c, f->s) && al(c, f->c));
}
static inline int grid_for(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    long long cap = 148LL * 16;
    return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

// Dynamic shared memory above 48 KB needs an opt-in, and the largest carveout
// lets several blocks share an SM.
template <class K> static cudaError_t prep_smem(K kern, int bytes) {
    if (bytes > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) return e;
    }
    if (bytes > 0)
        return cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    (int)cudaSharedmemCarveoutMaxShared);
    return cudaSuccess;
}

// ============================================================== per-size launchers
template <class K> static int blocks_per_sm(K kern, int threads, int smem) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        n = 1;
    }
    return n < 1 ? 1 : n;
}

// Line lengths at which GNSS_VARIANT_AUTO takes the register kernels, as
// measured on B200 (ensembles of 16 x 64^3 .. 2 x 192^3 and single jets at
// 256^3, 512^3): the z kernel at every length it serves; the passes at
// N = 96 .. 512 in FP32 (at N = 64 the staged pass: 8 931 against 7 759
// Mpoint-steps/s for 16 x 64^3) and at N = 256, 512 in FP64 (below, staged:
// 7 542 against 6 743 for 2 x 192^3).
__host__ __device__ constexpr bool zr_auto_z(int n) { return zr_size(n); }
__host__ __device__ constexpr bool zr_auto_pass(int n, bool fp64) {
    return zr_size(n) && (fp64 ? n >= 256 : n != 64);
}

template <typename T> static const V2<T> *pass_twiddles(const PassPtrs<T> &, const void *tw) {
    return reinterpret_cast<const V2<T> *>(tw);
}

// Launch of a kernel of the step.  Within a PdlScope that allows it, the
// launch carries programmatic stream serialization: the kernel may start its
// prologue on SMs the previous kernel in the stream has left and waits
// (pdl_wait) before it touches the memory of the step.  Inside stream capture
// the dependency becomes a programmatic graph edge.  Measured per step (FP32,
// one scalar): 64^3 53.5 -> 40.9 us, 96^3 118.7 -> 107.3 us, 128^3 195.3 ->
// 181.7 us, 192^3 579 -> 565 us.  Steps of more than 2^23 points launch
// plainly: with programmatic launches the 256^3 and 512^3 FP64 steps measured
// 0.5 - 2% slower.
static thread_local bool t_pdl = false;
struct PdlScope {
    bool prev;
    explicit PdlScope(bool on) : prev(t_pdl) { t_pdl = on; }
    ~PdlScope() { t_pdl = prev; }
};
constexpr long long PDL_MAX_POINTS = 1LL << 23;
template <typename... KA, typename... A>
static cudaError_t launch_dep(void (*kern)(KA...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A &&...args) {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.attrs = at;
    cfg.numAttrs = t_pdl ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

// A persistent pass launch: one block per SM times the blocks that fit
// (looked up once per kernel, from any host thread), at most one per work item.
template <class K, class PP>
static cudaError_t launch_persistent(K kern, std::atomic<int> &per_sm, int nt, int smem, int nsm, long long nitems,
                                     cudaStream_t s, const PP &P, const PassSpec &sp, const void *tw,
                                     unsigned *err = nullptr, bool with_err = false) {
    cudaError_t e = prep_smem(kern, smem);
    if (e != cudaSuccess) return e;
    int ps = per_sm.load(std::memory_order_relaxed);
    if (ps == 0) {
        ps = blocks_per_sm(kern, nt, smem);
        per_sm.store(ps, std::memory_order_relaxed);
    }
    long long grid = (long long)ps * nsm;
    if (grid > nitems) grid = nitems;
    if (with_err) {
        if constexpr (std::is_invocable_v<K, PP, PassSpec, const float2 *, unsigned *>)
            return launch_dep(kern, dim3((unsigned)grid), dim3(nt), smem, s, P, sp, reinterpret_cast<const float2 *>(tw),
                              err);
    } else {
        if constexpr (!std::is_invocable_v<K, PP, PassSpec, const float2 *, unsigned *>)
            return launch_dep(kern, dim3((unsigned)grid), dim3(nt), smem, s, P, sp, pass_twiddles(P, tw));
    }
    return cudaGetLastError();
}

template <typename T, int N> struct Launch {
    // Members of a batch (sp.nmem > 1) run the MB instantiations, which exist for the register lengths
    // (N = 64 .. 512); other lengths return cudaErrorNotSupported for a batch.
    static cudaError_t pass(int sign, const PassPtrs<T> &P, const PassSpec &sp, const void *tw, int nsm,
                            cudaStream_t s, int pvariant, unsigned *err) {
        const bool mb = sp.nmem > 1;
        const int ci = (sign < 0 ? 0 : 1) + (mb ? 2 : 0);   // occupancy cache index
        if constexpr (sizeof(T) == 4 && ptc_size(N)) {
            // split-TF32 DFT-GEMM transforms on the tensor cores (tiles of 8 columns)
            if (pvariant == GNSS_VARIANT_TENSOR) {
                using C = PTCfg<N>;
                auto kern = mb ? (sign < 0 ? k_passtc<N, -1, true> : k_passtc<N, +1, true>)
                               : (sign < 0 ? k_passtc<N, -1> : k_passtc<N, +1>);
                static std::atomic<int> per_sm[4];
                PassSpec s8 = sp;
                const int cols = sp.ncols > sp.out_ncols ? sp.ncols : sp.out_ncols;
                s8.ncolblk = (cols + C::NB - 1) / C::NB;
                const long long nitems = (long long)s8.nmem * s8.nin * s8.outer.count() * s8.ncolblk;
                return launch_persistent(kern, per_sm[ci], C::NT, C::SMEM, nsm, nitems, s,
                                         reinterpret_cast<const PassPtrs<float> &>(P), s8, tw, err, true);
            }
        }
        const long long nitems = (long long)sp.nmem * sp.nin * sp.outer.count() * sp.ncolblk;
        if constexpr (zr_size(N)) {
            // register-resident column transforms where they measured faster (512^3 FP32 step 7.34 against
            // 8.39 ms, FP64 10.1 against 8.9 Gpoint-steps/s; 256^3 1.23 against 1.28 ms; N = 96 .. 192 with
            // lane shuffles)
            const bool reg = pvariant == GNSS_VARIANT_REGISTER ||
                             ((pvariant == GNSS_VARIANT_AUTO || pvariant == GNSS_VARIANT_TENSOR) &&
                              zr_auto_pass(N, sizeof(T) == 8));
            if (reg) {
                using C = PRCfg<T, N>;
                auto kern = mb ? (sign < 0 ? k_passr<T, N, -1, true> : k_passr<T, N, +1, true>)
                               : (sign < 0 ? k_passr<T, N, -1> : k_passr<T, N, +1>);
                static std::atomic<int> per_sm[4];
                return launch_persistent(kern, per_sm[ci], C::NT, C::SMEM, nsm, nitems, s, P, sp, tw);
            }
        }
        using C = PassCfg<T, N>;
        static std::atomic<int> per_sm[4];
        if (mb) {
            if constexpr (zr_size(N)) {
                auto kern = sign < 0 ? k_pass<T, N, -1, true> : k_pass<T, N, +1, true>;
                return launch_persistent(kern, per_sm[ci], C::NT, C::SMEM, nsm, nitems, s, P, sp, tw);
            } else {
                return cudaErrorNotSupported;
            }
        }
        auto kern = sign < 0 ? k_pass<T, N, -1> : k_pass<T, N, +1>;
        return launch_persistent(kern, per_sm[ci], C::NT, C::SMEM, nsm, nitems, s, P, sp, tw);
    }
    static cudaError_t zpass(int dir, const FieldSet<T> &f, int nfields, long long nlines, int nz2, T scale,
                             const void *tw, cudaStream_t s) {
        using C = ZCfg<T, N>;
        long long npairs = (nlines + 1) / 2;
        dim3 grid((unsigned)((npairs + ZWARPS - 1) / ZWARPS), (unsigned)nfields);
        const V2<T> *t = reinterpret_cast<const V2<T> *>(tw);
        auto kern = dir < 0 ? k_zpass<T, N, -1> : k_zpass<T, N, +1>;
        cudaError_t e = prep_smem(kern, C::SMEM);
        if (e != cudaSuccess) return e;
        kern<<<grid, ZWARPS * 32, C::SMEM, s>>>(f, nlines, nz2, scale, t);
        return cudaGetLastError();
    }
    template <int NPH, int NRAW, bool PP>
    static cudaError_t zphys_k(const FieldSet<T> &f, const ZRecipeSet &zr, int nout, long long nlines, int ncp,
                               int nkz, T scale, T alpha, double dkz, const void *tw, unsigned *err, int nsm,
                               cudaStream_t s, int nmem, long long ms) {
        if (nmem > 1) return cudaErrorNotSupported;   // batches run the register z kernel
        using C = ZPCfg<T, N>;
        const int pipe_b = C::pipe_bytes(NPH, NRAW, ncp, PP);
        const int pipe = pipe_b <= C::SMEM_MAX ? 1 : 0;
        const int smem = pipe ? pipe_b : C::work_bytes(NPH, PP);
        auto kern = k_zphys<T, N, NPH, NRAW, PP>;
        cudaError_t e = prep_smem(kern, smem);
        if (e != cudaSuccess) return e;
        int per_sm = blocks_per_sm(kern, NPH * 32, smem);
        const long long mpairs = nlines / 2, npairs = mpairs * nmem;
        long long grid = (long long)per_sm * nsm;
        if (grid > npairs) grid = npairs;
        return launch_dep(kern, dim3((unsigned)grid), dim3(NPH * 32), smem, s, f, zr, nout, npairs, ncp, nkz, pipe,
                          scale, alpha, dkz, reinterpret_cast<const V2<T> *>(tw), err, mpairs, ms);
    }
    // ping-pong banks when they fit next to the staging area, else in place
    template <int NPH, int NRAW>
    static cudaError_t zphys_n(const FieldSet<T> &f, const ZRecipeSet &zr, int nout, long long nlines, int ncp,
                               int nkz, T scale, T alpha, double dkz, const void *tw, unsigned *err, int nsm,
                               cudaStream_t s, int nmem, long long ms) {
        using C = ZPCfg<T, N>;
        if (C::pipe_bytes(NPH, NRAW, ncp, true) <= C::SMEM_MAX)
            return zphys_k<NPH, NRAW, true>(f, zr, nout, nlines, ncp, nkz, scale, alpha, dkz, tw, err, nsm, s, nmem,
                                            ms);
        return zphys_k<NPH, NRAW, false>(f, zr, nout, nlines, ncp, nkz, scale, alpha, dkz, tw, err, nsm, s, nmem, ms);
    }
    // register-resident line transforms (N = 64 .. 512, zr_size) when their shared memory fits
    // diag != nullptr: the instantiation that also writes per-block vorticity sums there
    template <int NPH, int NRAW>
    static cudaError_t zreg_k(const FieldSet<T> &f, const ZRecipeSet &zr, int nout, long long nlines, int ncp, int nkz,
                              T scale, T alpha, double dkz, const void *tw, unsigned *err, int nsm, cudaStream_t s,
                              double *diag, int nmem, long long ms) {
        if constexpr (zr_size(N)) {
            const int smem = ZRCfg<T, N>::smem_bytes(NPH, NRAW, ncp);
            if (smem > ZPCfg<T, N>::SMEM_MAX) return cudaErrorNotSupported;
            auto kern = diag ? k_zreg<T, N, NPH, NRAW, true>
                             : (nmem > 1 ? k_zreg<T, N, NPH, NRAW, false, true> : k_zreg<T, N, NPH, NRAW, false>);
            cudaError_t e = prep_smem(kern, smem);
            if (e != cudaSuccess) return e;
            const int per_sm = blocks_per_sm(kern, NPH * 32, smem);
            const long long mpairs = nlines / 2, npairs = mpairs * nmem;
            long long grid = (long long)per_sm * nsm;
            if (grid > npairs) grid = npairs;
            if (diag && grid > STAT_BLOCKS) grid = STAT_BLOCKS;   // one row of sums per block
            return launch_dep(kern, dim3((unsigned)grid), dim3(NPH * 32), smem, s, f, zr, nout, npairs, ncp, nkz, scale,
                              alpha, dkz, reinterpret_cast<const V2<T> *>(tw), err, diag, mpairs, ms);
        } else {
            (void)f; (void)zr; (void)nout; (void)nlines; (void)ncp; (void)nkz; (void)scale; (void)alpha; (void)dkz;
            (void)tw; (void)err; (void)nsm; (void)s; (void)diag; (void)nmem; (void)ms;
            return cudaErrorNotSupported;
        }
    }
    // warp-specialised register z kernel (N = 256, 512; FP32 with 9 quantities and 4 products, FP64 with 9 and 4
    // or 12 and 5)
    static constexpr bool zws_size() { return N == 256 || N == 512; }
    template <int NPH, int NRAW>
    static cudaError_t zws_kt(const FieldSet<T> &f, const ZRecipeSet &zr, int nout, long long nlines, int ncp,
                              int nkz, T scale, T alpha, double dkz, const void *tw, unsigned *err, int nsm,
                              cudaStream_t s, int nmem, long long ms) {
        if (nmem > 1) return cudaErrorNotSupported;   // batches run the register z kernel
        if constexpr (zws_size()) {
            constexpr int NOUT = zws_nout<NPH>();
            const int smem = ZRCfg<T, N>::smem_bytes_ws(NPH, NOUT, NRAW, ncp);
            auto kern = k_zws<T, N, NPH, NRAW>;
            cudaError_t e = prep_smem(kern, smem);
            if (e != cudaSuccess) return e;
            const int nt = (NPH + NOUT) * 32;
            const int per_sm = blocks_per_sm(kern, nt, smem);
            const long long mpairs = nlines / 2, npairs = mpairs * nmem;
            long long grid = (long long)per_sm * nsm;
            if (grid > npairs) grid = npairs;
            return launch_dep(kern, dim3((unsigned)grid), dim3(nt), smem, s, f, zr, nout, npairs, ncp, nkz, scale, alpha,
                              dkz, reinterpret_cast<const V2<T> *>(tw), err, mpairs, ms);
        } else {
            (void)f; (void)zr; (void)nout; (void)nlines; (void)ncp; (void)nkz; (void)scale; (void)alpha; (void)dkz;
            (void)tw; (void)err; (void)nsm; (void)s; (void)nmem; (void)ms;
            return cudaErrorNotSupported;
        }
    }
    static cudaError_t zws_k(const FieldSet<T> &f, const ZRecipeSet &zr, int nph, int nraw, int nout, long long nlines,
                             int ncp, int nkz, T scale, T alpha, double dkz, const void *tw, unsigned *err, int nsm,
                             cudaStream_t s, int nmem, long long ms) {
        if (nph == 9 && nraw == 10)
            return zws_kt<9, 10>(f, zr, nout, nlines, ncp, nkz, scale, alpha, dkz, tw, err, nsm, s, nmem, ms);
        if (nph == 12 && nraw == 13)
            return zws_kt<12, 13>(f, zr, nout, nlines, ncp, nkz, scale, alpha, dkz, tw, err, nsm, s, nmem, ms);
        return cudaErrorNotSupported;
    }
    static bool zws_fits(int nph, int nraw, int nout, int ncp) {
        if constexpr (zws_size()) {
            const bool fp32 = sizeof(T) == 4 && nph == 9 && nraw == 10 && nout == 4;
            const bool fp64 = sizeof(T) == 8 && ((nph == 9 && nraw == 10 && nout == 4) ||
                                                 (nph == 12 && nraw == 13 && nout == 5));
            return (fp32 || fp64) && ZRCfg<T, N>::smem_bytes_ws(nph, nout, nraw, ncp) <= ZPCfg<T, N>::SMEM_MAX;
        } else {
            return false;
        }
    }
    static bool zreg_fits(int nph, int nraw, int ncp) {
        if constexpr (zr_size(N))
            return ZRCfg<T, N>::smem_bytes(nph, nraw, ncp) <= ZPCfg<T, N>::SMEM_MAX;
        else
            return false;
    }
    // the z kernel a variant option selects: GNSS_VARIANT_WARPSPEC, _REGISTER or _STAGED
    // AUTO: the warp-specialised kernel in FP64 where it fits (17 or 13 warps per SM against k_zreg's 12 or 9;
    // measured at 512^3 with two scalars: z 6.18 -> 5.53 ms, one scalar 5.48 -> 4.59 ms; 256^3 0.95 -> 0.80 ms),
    // the register kernel in FP32 (there k_zws measured slower: 2.52 -> 2.70 ms at 512^3)
    static int zkernel(int zvariant, int nph, int nraw, int nout, int ncp) {
        const bool ws = zvariant == GNSS_VARIANT_WARPSPEC || (zvariant == GNSS_VARIANT_AUTO && sizeof(T) == 8);
        if (ws && zws_fits(nph, nraw, nout, ncp)) return GNSS_VARIANT_WARPSPEC;
        const bool reg = zvariant == GNSS_VARIANT_REGISTER || zvariant == GNSS_VARIANT_WARPSPEC ||
                         (zvariant == GNSS_VARIANT_AUTO && zr_auto_z(N));
        return reg && zreg_fits(nph, nraw, ncp) ? GNSS_VARIANT_REGISTER : GNSS_VARIANT_STAGED;
    }
    // diag != nullptr: the register kernel with the fused vorticity sums (cudaErrorNotSupported where it does
    // not exist)
    static cudaError_t zphys(const FieldSet<T> &f, const ZRecipeSet &zr, int nph, int nraw, int nout,
                             long long nlines, int ncp, int nkz, T scale, T alpha, double dkz, const void *tw,
                             unsigned *err, int nsm, cudaStream_t s, int zvariant, double *diag = nullptr,
                             int nmem = 1, long long ms = 0) {
        if (diag) {
            if (!zreg_fits(nph, nraw, ncp)) return cudaErrorNotSupported;
            if (nph == 9 && nraw == 10)
                return zreg_k<9, 10>(f, zr, nout, nlines, ncp, nkz, scale, alpha, dkz, tw, err, nsm, s, diag, 1, 0);
            if (nph == 12 && nraw == 13)
                return zreg_k<12, 13>(f, zr, nout, nlines, ncp, nkz, scale, alpha, dkz, tw, err, nsm, s, diag, 1, 0);
            if (nph == 14 && nraw == 14)
                return zreg_k<14, 14>(f, zr, nout, nlines, ncp, nkz, scale, alpha, dkz, tw, err, nsm, s, diag, 1, 0);
            return cudaErrorInvalidValue;
        }
        const int kern = zkernel(zvariant, nph, nraw, nout, ncp);
        if (kern == GNSS_VARIANT_WARPSPEC)
            return zws_k(f, zr, nph, nraw, nout, nlines, ncp, nkz, scale, alpha, dkz, tw, err, nsm, s, nmem, ms);
        if (kern == GNSS_VARIANT_REGISTER) {
            if (nph == 9 && nraw == 10)
                return zreg_k<9, 10>(f, zr, nout, nlines, ncp, nkz, scale, alpha, dkz, tw, err, nsm, s, nullptr, nmem,
                                     ms);
            if (nph == 12 && nraw == 13)
                return zreg_k<12, 13>(f, zr, nout, nlines, ncp, nkz, scale, alpha, dkz, tw, err, nsm, s, nullptr, nmem,
                                      ms);
            if (nph == 14 && nraw == 14)
                return zreg_k<14, 14>(f, zr, nout, nlines, ncp, nkz, scale, alpha, dkz, tw, err, nsm, s, nullptr, nmem,
                                      ms);
            return cudaErrorInvalidValue;
        }
        if (nph == 9 && nraw == 10)
            return zphys_n<9, 10>(f, zr, nout, nlines, ncp, nkz, scale, alpha, dkz, tw, err, nsm, s, nmem, ms);
        if (nph == 12 && nraw == 13)
            return zphys_n<12, 13>(f, zr, nout, nlines, ncp, nkz, scale, alpha, dkz, tw, err, nsm, s, nmem, ms);
        if (nph == 14 && nraw == 14)
            return zphys_n<14, 14>(f, zr, nout, nlines, ncp, nkz, scale, alpha, dkz, tw, err, nsm, s, nmem, ms);
        return cudaErrorInvalidValue;
    }
};

#define GNSS_SIZE_SWITCH(n, EXPR) GNSS_SIZE_SWITCH_OR(n, EXPR, return cudaErrorInvalidValue)
#define GNSS_SIZE_SWITCH_OR(n, EXPR, DEFAULT)       \
    switch (n) {                                    \
        case 8: { constexpr int NN_ = 8; EXPR; }    \
        case 12: { constexpr int NN_ = 12; EXPR; }  \
        case 16: { constexpr int NN_ = 16; EXPR; }  \
        case 24: { constexpr int NN_ = 24; EXPR; }  \
        case 32: { constexpr int NN_ = 32; EXPR; }  \
        case 48: { constexpr int NN_ = 48; EXPR; }  \
        case 64: { constexpr int NN_ = 64; EXPR; }  \
        case 96: { constexpr int NN_ = 96; EXPR; }  \
        case 128: { constexpr int NN_ = 128; EXPR; } \
        case 192: { constexpr int NN_ = 192; EXPR; } \
        case 256: { constexpr int NN_ = 256; EXPR; } \
        case 384: { constexpr int NN_ = 384; EXPR; } \
        case 512: { constexpr int NN_ = 512; EXPR; } \
        default: DEFAULT;                           \
    }

template <typename T>
static cudaError_t launch_pass(int n, int sign, const PassPtrs<T> &P, const PassSpec &sp, const void *tw, int nsm,
                               cudaStream_t s, int pvariant, unsigned *err) {
    GNSS_SIZE_SWITCH(n, return (Launch<T, NN_>::pass(sign, P, sp, tw, nsm, s, pvariant, err)));
}
template <typename T>
static cudaError_t launch_zpass(int n, int dir, const FieldSet<T> &f, int nfields, long long nlines, int nz2, T scale,
                                const void *tw, cudaStream_t s) {
    GNSS_SIZE_SWITCH(n, return (Launch<T, NN_>::zpass(dir, f, nfields, nlines, nz2, scale, tw, s)));
}
template <typename T>
static cudaError_t launch_zphys(int n, const FieldSet<T> &f, const ZRecipeSet &zr, int nph, int nraw, int nout,
                                long long nlines, int ncp, int nkz, T scale, T alpha, double dkz, const void *tw,
                                unsigned *err, int nsm, cudaStream_t s, int zvariant, double *diag = nullptr,
                                int nmem = 1, long long ms = 0) {
    GNSS_SIZE_SWITCH(n, return (Launch<T, NN_>::zphys(f, zr, nph, nraw, nout, nlines, ncp, nkz, scale, alpha, dkz, tw,
                                                      err, nsm, s, zvariant, diag, nmem, ms)));
}

template <typename T> static int pass_nb(int n) {
    switch (n) {
        case 8: return PassCfg<T, 8>::NB; case 12: return PassCfg<T, 12>::NB;
        case 16: return PassCfg<T, 16>::NB; case 24: return PassCfg<T, 24>::NB;
        case 32: return PassCfg<T, 32>::NB; case 48: return PassCfg<T, 48>::NB;
        case 64: return PassCfg<T, 64>::NB; case 96: return PassCfg<T, 96>::NB;
        case 128: return PassCfg<T, 128>::NB; case 192: return PassCfg<T, 192>::NB;
        case 256: return PassCfg<T, 256>::NB; case 384: return PassCfg<T, 384>::NB;
        default: return PassCfg<T, 512>::NB;
    }
}

// ============================================================== helpers
template <typename T> static V2<T> *fld(void *base, size_t nspec, int i) {
    return reinterpret_cast<V2<T> *>(base) + nspec * (size_t)i;
}

static gnss_status ensure_scratch(gnss_ctx *c, int nfields) {
    if (c->nscratch >= nfields) return GNSS_OK;
    if (c->scratch_ext)
        return fail(c, GNSS_ERR_NOMEM, "attached scratch holds %d fields, %d needed", c->nscratch, nfields);
    if (c->scratch) {
        cudaFree(c->scratch);
        c->owned_bytes -= (size_t)c->nscratch * c->nspec * c->elem;
        c->scratch = nullptr;
        c->nscratch = 0;
    }
    size_t bytes = (size_t)nfields * c->nspec * c->elem;
    if (cudaMalloc(&c->scratch, bytes) != cudaSuccess) {
        cudaGetLastError();
        c->scratch = nullptr;
        return fail(c, GNSS_ERR_NOMEM, "cannot allocate %zu bytes of scratch", bytes);
    }
    c->nscratch = nfields;
    c->owned_bytes += bytes;
    return GNSS_OK;
}

// Scratch of the fused step: n_xout P fields, n_raw Q fields (and, for the
// IF-RK3 scheme, the history after them, full reference-layout fields).
static size_t step_scratch_elems(const gnss_ctx *c) {
    size_t e = c->p_elems * (size_t)c->n_xout + c->q_elems * (size_t)c->n_raw;
    if (c->cfg.scheme == GNSS_SCHEME_RK3IF) e += c->nspec * (size_t)(3 + c->cfg.n_scalars);
    return e;
}
static gnss_status ensure_scratch_step(gnss_ctx *c) {
    const size_t need = step_scratch_elems(c);
    const int nf = (int)((need + c->nspec - 1) / c->nspec);   // in units of full fields
    return ensure_scratch(c, nf);
}

// Pass geometries of the full 3D transforms (gnss_forward / gnss_inverse):
// x passes read / write the spectral layout [y][x][kz] on one side and
// [x][y][kz] on the other; y passes work on [x][y][kz]; every index kept.
enum PassKind { X_INV, X_FWD, Y_PASS };
static KeepMap keep_all(int n) { return KeepMap{n, -1}; }

template <typename T> static PassSpec base_spec(const gnss_ctx *c, int nrow_fft, int nin) {
    const Geom &g = c->g;
    PassSpec p{};
    p.nmem = 1;
    const int nb = pass_nb<T>(nrow_fft);
    p.ncols = g.nz2;
    p.out_ncols = g.nz2;
    p.ncolblk = (g.nz2 + nb - 1) / nb;
    p.nin = nin;
    p.n_col = g.nz;
    p.dk_col = g.dkz;
    p.kmax2 = g.kmax2;
    p.mask = 0;
    for (int i = 0; i < nin; ++i) {   // default: one plain output per input, same index
        p.nvar[i] = 1;
        p.vmul[i][0] = V_ONE;
        p.vout[i][0] = (signed char)i;
    }
    return p;
}

template <typename T> static PassSpec pass_spec(const gnss_ctx *c, PassKind kind, int nin) {
    const Geom &g = c->g;
    const long long nz2 = g.nz2;
    PassSpec p = base_spec<T>(c, kind == Y_PASS ? g.ny : g.nx, nin);
    switch (kind) {
        case X_INV:   // rows = kx, outer = ky: spectral -> [x][y][kz]
            p.s_row = nz2; p.s_out = (long long)g.nx * nz2; p.d_row = (long long)g.ny * nz2; p.d_out = nz2;
            p.row_in = p.row_out = keep_all(g.nx); p.outer = keep_all(g.ny);
            p.n_row = g.nx; p.n_out = g.ny; p.dk_row = g.dkx; p.dk_out = g.dky;
            break;
        case X_FWD:   // rows = x, outer = y: [x][y][kz] -> spectral
            p.s_row = (long long)g.ny * nz2; p.s_out = nz2; p.d_row = nz2; p.d_out = (long long)g.nx * nz2;
            p.row_in = p.row_out = keep_all(g.nx); p.outer = keep_all(g.ny);
            p.n_row = g.nx; p.n_out = 0; p.dk_row = g.dkx;
            break;
        case Y_PASS:  // rows = ky (or y), outer = x
            p.s_row = nz2; p.s_out = (long long)g.ny * nz2; p.d_row = nz2; p.d_out = (long long)g.ny * nz2;
            p.row_in = p.row_out = keep_all(g.ny); p.outer = keep_all(g.nx);
            p.n_row = g.ny; p.n_out = 0; p.dk_row = g.dky;
            break;
    }
    return p;
}

// Passes of the fused step on the compact layouts (see gnss_ctx):
//   X_INV_STEP  state [y][x][kz] (kept kx rows, kept ky, kz < nkz) -> P [x][kyc][ncp]
//   Y_INV_STEP  P [x][kyc][ncp] (rows = y, kept rows only)          -> Q [x][y][ncp]
//   Y_FWD_STEP  Q [x][y][ncp]                                      -> P [x][kyc][ncp] (kept ky rows)
//   X_FWD_STEP  P [x][kyc][ncp] (rows = x, outer = kept ky)        -> R [kyc][kxc][ncp] (kept kx rows)
enum StepPass { X_INV_STEP, Y_INV_STEP, Y_FWD_STEP, X_FWD_STEP };
template <typename T> static PassSpec step_spec(const gnss_ctx *c, StepPass kind, int nin) {
    const Geom &g = c->g;
    const long long ncp = c->ncp;
    const int nky = c->ky_keep.count(), nkx = c->kx_keep.count();
    const bool ypass = kind == Y_INV_STEP || kind == Y_FWD_STEP;
    PassSpec p = base_spec<T>(c, ypass ? g.ny : g.nx, nin);
    const int nb = pass_nb<T>(ypass ? g.ny : g.nx);
    p.ncols = (int)ncp;
    p.out_ncols = (int)ncp;
    p.ncolblk = (int)(ncp / nb);
    switch (kind) {
        case X_INV_STEP:
            p.s_row = g.nz2; p.s_out = (long long)g.nx * g.nz2;                 // state, expanded ky
            p.ncols = c->nkz;
            p.row_in = c->kx_keep; p.row_in_compact = 0;
            p.row_out = keep_all(g.nx);
            p.outer = c->ky_keep; p.outer_in_compact = 0; p.outer_out_compact = 1;
            p.d_row = (long long)nky * ncp; p.d_out = ncp;
            p.n_row = g.nx; p.n_out = g.ny; p.dk_row = g.dkx; p.dk_out = g.dky;
            p.mask = 1;
            break;
        case Y_INV_STEP:
            p.s_row = ncp; p.s_out = (long long)nky * ncp;
            p.row_in = c->ky_keep; p.row_in_compact = 1;
            p.row_out = keep_all(g.ny);
            p.outer = keep_all(g.nx);
            p.d_row = ncp; p.d_out = (long long)g.ny * ncp;
            p.n_row = g.ny; p.n_out = 0; p.dk_row = g.dky;
            break;
        case Y_FWD_STEP:
            p.s_row = ncp; p.s_out = (long long)g.ny * ncp;
            p.row_in = keep_all(g.ny);
            p.row_out = c->ky_keep; p.row_out_compact = 1;
            p.outer = keep_all(g.nx);
            p.d_row = ncp; p.d_out = (long long)nky * ncp;
            p.n_row = g.ny; p.n_out = 0; p.dk_row = g.dky;
            break;
        case X_FWD_STEP:
            p.s_row = (long long)nky * ncp; p.s_out = ncp;
            p.row_in = keep_all(g.nx);
            p.row_out = c->kx_keep; p.row_out_compact = 1;
            p.outer = c->ky_keep; p.outer_in_compact = 1; p.outer_out_compact = 1;
            p.d_row = ncp; p.d_out = (long long)nkx * ncp;
            p.n_row = g.nx; p.n_out = 0; p.dk_row = g.dkx;
            break;
    }
    return p;
}

// ============================================================== transforms
template <typename T> static gnss_status forward_t(gnss_ctx *c, void *f, cudaStream_t s) {
    gnss_status st = ensure_scratch(c, 1);
    if (st) return st;
    const Geom &g = c->g;
    FieldSet<T> F{};
    F.p[0] = reinterpret_cast<V2<T> *>(f);
    V2<T> *X = fld<T>(c->scratch, c->nspec, 0);
    const long long nlines = (long long)g.nx * g.ny;
    c->launches += 3;
    CK(c, launch_zpass<T>(g.nz, -1, F, 1, nlines, g.nz2, T(1), c->tw[2], s));
    PassPtrs<T> P{};
    P.in[0] = F.p[0];
    P.out[0] = X;
    CK(c, launch_pass<T>(g.ny, -1, P, pass_spec<T>(c, Y_PASS, 1), c->tw[1], c->nsm, s, c->pvariant, c->d_err));
    P.in[0] = X;
    P.out[0] = F.p[0];
    CK(c, launch_pass<T>(g.nx, -1, P, pass_spec<T>(c, X_FWD, 1), c->tw[0], c->nsm, s, c->pvariant, c->d_err));
    return GNSS_OK;
}

template <typename T> static gnss_status inverse_t(gnss_ctx *c, void *f, cudaStream_t s) {
    gnss_status st = ensure_scratch(c, 1);
    if (st) return st;
    const Geom &g = c->g;
    FieldSet<T> F{};
    F.p[0] = reinterpret_cast<V2<T> *>(f);
    V2<T> *X = fld<T>(c->scratch, c->nspec, 0);
    const long long nlines = (long long)g.nx * g.ny;
    const T scale = (T)(1.0 / ((double)g.nx * g.ny * g.nz));
    c->launches += 3;
    PassPtrs<T> P{};
    P.in[0] = F.p[0];
    P.out[0] = X;
    CK(c, launch_pass<T>(g.nx, +1, P, pass_spec<T>(c, X_INV, 1), c->tw[0], c->nsm, s, c->pvariant, c->d_err));
    P.in[0] = X;
    P.out[0] = F.p[0];
    CK(c, launch_pass<T>(g.ny, +1, P, pass_spec<T>(c, Y_PASS, 1), c->tw[1], c->nsm, s, c->pvariant, c->d_err));
    CK(c, launch_zpass<T>(g.nz, +1, F, 1, nlines, g.nz2, scale, c->tw[2], s));
    return GNSS_OK;
}

// ============================================================== fused step
// One evaluation of the nonlinear term followed by the spectral update.
//   1 x inverse of the dealiased state: X[f] and X[i kx f]                (state -> P)
//   2 y inverse: Y[.] and Y[i ky .]                                        (P -> Q)
//   3 z: kz factors and vorticity combinations, C2R, products, R2C        (Q -> Q[0..nnl))
//      (physical space stays on chip)
//   4 y forward of the products (in place)                                 (Q)
//   5 x forward of the products into the spectral layout                   (Q -> P)
//   6 projection, dealias and time update                                  (P, state, hist)
// A batch: nmem members of one geometry stepped by the same launches (the
// ensemble's size groups).  Member m's state and history fields lie ms_sh
// elements after member 0's, its step scratch ms_scr elements after the
// batch scratch `scratch`; mc holds the members' update coefficients.
struct Batch {
    int nmem = 1;
    long long ms_sh = 0, ms_scr = 0;
    void *scratch = nullptr;
    const MemberCoef *mc = nullptr;
};

template <typename T>
static gnss_status nonlinear_and_update(gnss_ctx *c, const gnss_fields *state, void *hist_base, const gnss_fields *hist,
                                        const UpdCoef &uc, cudaStream_t s, double *stats_dst = nullptr,
                                        double *diag = nullptr, const Batch &bt = Batch{}) {
    const Geom &g = c->g;
    const int np = c->n_xout, nq = c->n_raw, nnl = c->nnl;
    if (!bt.scratch) {
        gnss_status st = ensure_scratch_step(c);
        if (st) return st;
    }
    const PdlScope pdl((long long)g.nx * g.ny * g.nz <= PDL_MAX_POINTS);
    V2<T> *Pb = reinterpret_cast<V2<T> *>(bt.scratch ? bt.scratch : c->scratch);
    V2<T> *Qb = Pb + c->p_elems * (size_t)np;
    auto Pf = [&](int q) { return Pb + c->p_elems * (size_t)q; };
    auto Qf = [&](int q) { return Qb + c->q_elems * (size_t)q; };
    FieldSet<T> SF{}, Q{}, R{}, H{};
    void *sp[5] = {state->u, state->v, state->w, state->s, state->c};
    for (int q = 0; q < 5; ++q) SF.p[q] = reinterpret_cast<V2<T> *>(sp[q]);
    for (int q = 0; q < nq; ++q) Q.p[q] = Qf(q);
    for (int q = 0; q < nnl; ++q) R.p[q] = Qf(q);   // x forward output reuses Q storage
    if (hist) {
        void *hp[5] = {hist->u, hist->v, hist->w, hist->s, hist->c};
        for (int q = 0; q < 5; ++q) H.p[q] = reinterpret_cast<V2<T> *>(hp[q]);
    } else {
        for (int q = 0; q < 5; ++q) H.p[q] = fld<T>(hist_base, c->nspec, q);
    }
    const long long nlines = (long long)g.nx * g.ny;
    const T scale = (T)(1.0 / ((double)g.nx * g.ny * g.nz));
    if (uc.scheme == GNSS_SCHEME_CNAB2 && (c->herm_row || c->herm_col || c->herm_plane)) {
        // the Hermitian part of the velocity at kept Nyquist modes, as the reference's round trip leaves it
        MemberCoef mc{};
        if (bt.nmem > 1) mc = *bt.mc;
        else mc.mean[0] = c->mean64;
        const long long n = ((c->herm_row ? g.nx : 0) + (c->herm_col ? g.ny : 0) +
                             (c->herm_plane ? (long long)g.nx * g.ny : 0)) * bt.nmem;
        CK(c, launch_dep(k_herm<T>, dim3((unsigned)std::min<long long>((n + 255) / 256, 4LL * c->nsm)), dim3(256), 0, s,
                         SF, g, c->herm_row, c->herm_col, c->herm_plane, mc, bt.nmem, bt.ms_sh));
        c->launches++;
    }
    {
        StageTimer t(c, s, 0);
        PassPtrs<T> P{};
        const int nxi = c->n_xin;
        for (int q = 0; q < nxi; ++q) P.in[q] = SF.p[c->xvar_in[q]];
        for (int q = 0; q < np; ++q) P.out[q] = Pf(q);
        PassSpec spx = step_spec<T>(c, X_INV_STEP, nxi);
        for (int i = 0; i < nxi; ++i) {
            spx.nvar[i] = c->xvar_n[i];
            for (int v = 0; v < 2; ++v) { spx.vmul[i][v] = c->xvar_mul[i][v]; spx.vout[i][v] = c->xvar_out[i][v]; }
        }
        spx.nmem = bt.nmem; spx.ms_in = bt.ms_sh; spx.ms_out = bt.ms_scr;
        CK(c, launch_pass<T>(g.nx, +1, P, spx, c->tw[0], c->nsm, s, c->pvariant, c->d_err));
    }
    {
        StageTimer t(c, s, 1);
        PassPtrs<T> P{};
        for (int q = 0; q < np; ++q) P.in[q] = Pf(q);
        for (int q = 0; q < nq; ++q) P.out[q] = Qf(q);
        PassSpec spy = step_spec<T>(c, Y_INV_STEP, np);
        for (int i = 0; i < np; ++i) {
            spy.nvar[i] = c->yvar_n[i];
            for (int v = 0; v < 2; ++v) { spy.vmul[i][v] = c->yvar_mul[i][v]; spy.vout[i][v] = c->yvar_out[i][v]; }
        }
        spy.nmem = bt.nmem; spy.ms_in = spy.ms_out = bt.ms_scr;
        CK(c, launch_pass<T>(g.ny, +1, P, spy, c->tw[1], c->nsm, s, c->pvariant, c->d_err));
    }
    {
        StageTimer t(c, s, 2);
        CK(c, launch_zphys<T>(g.nz, Q, c->zrec, c->n_phys, nq, nnl, nlines, c->ncp, c->nkz, scale, (T)c->cfg.alpha,
                              g.dkz, c->tw[2], c->d_err, c->nsm, s, c->zvariant, diag, bt.nmem, bt.ms_scr));
    }
    {
        StageTimer t(c, s, 3);
        PassPtrs<T> P{};
        for (int q = 0; q < nnl; ++q) { P.in[q] = Qf(q); P.out[q] = Pf(q); }
        PassSpec sp3 = step_spec<T>(c, Y_FWD_STEP, nnl);
        sp3.nmem = bt.nmem; sp3.ms_in = sp3.ms_out = bt.ms_scr;
        CK(c, launch_pass<T>(g.ny, -1, P, sp3, c->tw[1], c->nsm, s, c->pvariant, c->d_err));
    }
    {
        StageTimer t(c, s, 4);
        PassPtrs<T> P{};
        for (int q = 0; q < nnl; ++q) { P.in[q] = Pf(q); P.out[q] = R.p[q]; }
        PassSpec sp4 = step_spec<T>(c, X_FWD_STEP, nnl);
        sp4.nmem = bt.nmem; sp4.ms_in = sp4.ms_out = bt.ms_scr;
        CK(c, launch_pass<T>(g.nx, -1, P, sp4, c->tw[0], c->nsm, s, c->pvariant, c->d_err));
    }
    {
        StageTimer t(c, s, 5);
        // one warp per kept (ky, kx) row; 8 blocks of 8 warps per SM
        const long long nrows = (long long)c->ky_keep.count() * c->kx_keep.count() * bt.nmem;
        const int full_rows = (uc.scheme == GNSS_SCHEME_CNAB2 && uc.euler) ? 1 : 0;
        long long nblk = std::min<long long>((nrows + 7) / 8, 8LL * c->nsm);
        if (bt.nmem > 1) {   // a batch (no statistics): per-member coefficients and mean lines
            auto kb = uc.scheme == GNSS_SCHEME_CNAB2 ? k_update_batch<T, GNSS_SCHEME_CNAB2>
                                                     : k_update_batch<T, GNSS_SCHEME_RK3IF>;
            CK(c, launch_dep(kb, dim3((unsigned)nblk), dim3(256), 0, s, SF, H, R, g, c->kx_keep, c->ky_keep, c->nkz,
                             c->ncp, uc, full_rows, *bt.mc, bt.nmem, bt.ms_sh, bt.ms_scr));
            return GNSS_OK;
        }
        if (stats_dst) {   // statistics of the new state summed by the update itself (one partial row per block)
            nblk = std::min<long long>(nblk, STAT_BLOCKS);
            auto ku = uc.scheme == GNSS_SCHEME_CNAB2 ? k_update<T, GNSS_SCHEME_CNAB2, true>
                                                     : k_update<T, GNSS_SCHEME_RK3IF, true>;
            CK(c, launch_dep(ku, dim3((unsigned)nblk), dim3(256), 0, s, SF, H, R, g, c->kx_keep, c->ky_keep, c->nkz,
                             c->ncp, uc, full_rows, c->stat_part, c->mean64));
            c->launches++;
            CK(c, launch_dep(k_stats_final, dim3(1), dim3(STAT_SUMS * 32), 0, s, (const double *)c->stat_part,
                             (int)nblk, stats_dst));
            return GNSS_OK;
        }
        auto ku = uc.scheme == GNSS_SCHEME_CNAB2 ? k_update<T, GNSS_SCHEME_CNAB2> : k_update<T, GNSS_SCHEME_RK3IF>;
        CK(c, launch_dep(ku, dim3((unsigned)nblk), dim3(256), 0, s, SF, H, R, g, c->kx_keep, c->ky_keep, c->nkz,
                         c->ncp, uc, full_rows, (double *)nullptr, c->mean64));
    }
    return GNSS_OK;
}

static UpdCoef base_coef(const gnss_ctx *c) {
    UpdCoef u{};
    const gnss_config &k = c->cfg;
    u.nf = 3 + k.n_scalars;
    u.scheme = k.scheme;
    u.dt = k.dt;
    // solver.cu:599-611: num = Re for u, v, w; Re*Sc for s; Re*Sc_c for c
    const double num[5] = {k.re, k.re, k.re, k.re * k.sc, k.re * k.sc_c};
    for (int q = 0; q < 5; ++q) {
        u.hnum[q] = k.dt / 2.0 / num[q];
        u.nu[q] = 1.0 / num[q];
    }
    return u;
}

template <typename T>
static gnss_status step_t(gnss_ctx *c, const gnss_fields *state, const gnss_fields *hist, int euler, cudaStream_t s,
                          double *stats_dst = nullptr, double *diag = nullptr) {
    UpdCoef uc = base_coef(c);
    if (c->cfg.scheme == GNSS_SCHEME_CNAB2) {
        uc.euler = euler ? 1 : 0;
        return nonlinear_and_update<T>(c, state, nullptr, hist, uc, s, stats_dst, diag);
    }
    // IF-RK3: the history lives in context scratch after the step's quantities
    gnss_status st = ensure_scratch_step(c);
    if (st) return st;
    void *hb = reinterpret_cast<V2<T> *>(c->scratch) + c->p_elems * (size_t)c->n_xout +
               c->q_elems * (size_t)c->n_raw;
    const double gam[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
    const double zet[4] = {0.0, -17.0 / 60.0, -5.0 / 12.0, 0.0};
    for (int k = 0; k < 3; ++k) {
        uc.substep = k;
        uc.gam = gam[k];
        uc.zet_next = zet[k + 1];
        uc.alph = gam[k] + zet[k];
        st = nonlinear_and_update<T>(c, state, hb, nullptr, uc, s, k == 2 ? stats_dst : nullptr,
                                     k == 0 ? diag : nullptr);   // the state the step starts from
        if (st) return st;
    }
    return GNSS_OK;
}

// ============================================================== statistics
static void stats_of_sums(const gnss_ctx *c, const double *h, double *out);

template <typename T> static gnss_status stats_t(gnss_ctx *c, const gnss_fields *st, double *out, cudaStream_t s) {
    FieldSet<T> F{};
    void *sp[5] = {st->u, st->v, st->w, st->s, st->c};
    for (int q = 0; q < 5; ++q) F.p[q] = reinterpret_cast<V2<T> *>(sp[q]);
    const int has_s = st->s != nullptr, has_c = st->c != nullptr;
    c->launches += 2;
    k_stats_partial<T><<<STAT_BLOCKS, STAT_THREADS, 0, s>>>(F, has_s, has_c, c->g, c->stat_part);
    LAUNCH_CK(c);
    k_stats_final<<<1, STAT_SUMS * 32, 0, s>>>(c->stat_part, STAT_BLOCKS, c->stat_dev);
    LAUNCH_CK(c);
    CK(c, cudaMemcpyAsync(c->stat_host, c->stat_dev, sizeof(double) * STAT_SUMS, cudaMemcpyDeviceToHost, s));
    CK(c, cudaStreamSynchronize(s));
    gnss_status chk = gnss_check(c, s);
    if (chk) return chk;
    stats_of_sums(c, c->stat_host, out);
    return GNSS_OK;
}

// The GNSS_NSTATS statistics from the STAT_SUMS spectral sums (the
// normalisations of calcTurbStats, statistics.cu:1494-1845).
static void stats_of_sums(const gnss_ctx *c, const double *h, double *out) {
    const gnss_config &k = c->cfg;
    const double nn = (double)k.nx * k.ny * k.nz;
    const double n2 = nn * nn;
    out[GNSS_STAT_KE] = (h[0] / n2) / 2.0;
    out[GNSS_STAT_VRMS2] = (h[0] / n2) / 3.0;
    out[GNSS_STAT_EPS] = k.nu_stats * (h[1] / n2);
    out[GNSS_STAT_CHI_S] = 2.0 * (k.nu_stats / k.sc) * (h[2] / n2);
    out[GNSS_STAT_CHI_C] = 2.0 * (k.nu_stats / k.sc_c) * (h[3] / n2);
    out[GNSS_STAT_VAR_S] = h[4] / n2;
    out[GNSS_STAT_VAR_C] = h[5] / n2;
}

// calcTurbStats_mgpu (statistics.cu:2039-2156): spectral sums; the vorticity
// statistics over the grid after three inverse transforms of the vorticity
// (scratch fields 1..3; field 0 is the transforms' own scratch); mean
// profiles from the kx = kz = 0 modes.
static gnss_status ensure_turb_buffers(gnss_ctx *c) {
    const size_t nvals = TURB_SUMS + VORT_SUMS + 5 * (size_t)c->g.ny;
    if (!c->turb_part) {
        if (cudaMalloc(&c->turb_part, sizeof(double) * STAT_BLOCKS * std::max(TURB_SUMS, VORT_SUMS)) != cudaSuccess ||
            cudaMalloc(&c->turb_dev, sizeof(double) * nvals) != cudaSuccess ||
            cudaMallocHost(&c->turb_host, sizeof(double) * nvals) != cudaSuccess) {
            cudaGetLastError();
            return fail(c, GNSS_ERR_NOMEM, "cannot allocate statistics buffers");
        }
        c->owned_bytes += sizeof(double) * (STAT_BLOCKS * std::max(TURB_SUMS, VORT_SUMS) + nvals);
    }
    return GNSS_OK;
}

// spectral sums and mean profiles of a state into turb_dev (no synchronisation)
template <typename T> static gnss_status turb_spectral_t(gnss_ctx *c, const FieldSet<T> &F, bool has_s, cudaStream_t s) {
    const Geom &g = c->g;
    c->launches += 3;
    k_turb_partial<T><<<STAT_BLOCKS, STAT_THREADS, 0, s>>>(F, has_s, g, c->turb_part);
    LAUNCH_CK(c);
    k_sums_final<TURB_SUMS><<<1, TURB_SUMS * 32, 0, s>>>(c->turb_part, STAT_BLOCKS, TURB_SUMS, c->turb_dev);
    LAUNCH_CK(c);
    k_yprof<T><<<5, 256, 0, s>>>(F, g, reinterpret_cast<const V2<T> *>(c->tw[1]),
                                 c->turb_dev + TURB_SUMS + VORT_SUMS);
    LAUNCH_CK(c);
    return GNSS_OK;
}

// vorticity sums over the grid into turb_dev + TURB_SUMS, by three inverse transforms (no synchronisation)
template <typename T> static gnss_status turb_vort_t(gnss_ctx *c, const FieldSet<T> &F, cudaStream_t s) {
    const Geom &g = c->g;
    gnss_status stt = ensure_scratch(c, 4);
    if (stt) return stt;
    V2<T> *o[3];
    for (int q = 0; q < 3; ++q) o[q] = fld<T>(c->scratch, c->nspec, 1 + q);
    c->launches++;
    k_vorticity<T><<<grid_for((long long)c->nspec, 256), 256, 0, s>>>(F.p[0], F.p[1], F.p[2], o[0], o[1], o[2], g);
    LAUNCH_CK(c);
    for (int q = 0; q < 3; ++q) {
        gnss_status e = inverse_t<T>(c, o[q], s);
        if (e) return e;
    }
    c->launches += 2;
    k_vort_partial<T><<<STAT_BLOCKS, STAT_THREADS, 0, s>>>(reinterpret_cast<const T *>(o[0]),
                                                            reinterpret_cast<const T *>(o[1]),
                                                            reinterpret_cast<const T *>(o[2]), g, c->turb_part);
    LAUNCH_CK(c);
    k_sums_final<VORT_SUMS><<<1, VORT_SUMS * 32, 0, s>>>(c->turb_part, STAT_BLOCKS, VORT_SUMS,
                                                         c->turb_dev + TURB_SUMS);
    LAUNCH_CK(c);
    return GNSS_OK;
}

// turb_dev to the host and into gnss_turb (synchronises)
static gnss_status turb_finish(gnss_ctx *c, bool has_s, gnss_turb *out, double *yprof, cudaStream_t s) {
    const Geom &g = c->g;
    const size_t nvals = TURB_SUMS + VORT_SUMS + 5 * (size_t)g.ny;
    CK(c, cudaMemcpyAsync(c->turb_host, c->turb_dev, sizeof(double) * nvals, cudaMemcpyDeviceToHost, s));
    CK(c, cudaStreamSynchronize(s));
    gnss_status chk = gnss_check(c, s);
    if (chk) return chk;
    const gnss_config &k = c->cfg;
    const double nn = (double)k.nx * k.ny * k.nz, n2 = nn * nn, nu = k.nu_stats;
    const double *h = c->turb_host;
    out->ke = (h[0] / n2) / 2.0;
    out->vrms = std::sqrt((h[0] / n2) / 3.0);
    out->epsilon = nu * (h[1] / n2);
    out->eta = std::sqrt(std::sqrt(nu * nu * nu / out->epsilon));
    out->l = 3 * M_PI / 4 * (h[2] / n2) / out->ke;
    out->lambda = std::sqrt(15.0 * nu * out->vrms * out->vrms / out->epsilon);
    out->chi = has_s ? 2.0 * (nu / k.sc) * (h[3] / n2) : 0.0;
    out->omega = h[TURB_SUMS] / nn;
    out->omega_x = std::sqrt(h[TURB_SUMS + 1] / nn);
    out->omega_y = std::sqrt(h[TURB_SUMS + 2] / nn);
    out->omega_z = std::sqrt(h[TURB_SUMS + 3] / nn);
    if (yprof) std::memcpy(yprof, h + TURB_SUMS + VORT_SUMS, sizeof(double) * 5 * (size_t)g.ny);
    return GNSS_OK;
}

template <typename T> static FieldSet<T> fieldset_of(const gnss_fields *st) {
    FieldSet<T> F{};
    void *sp[5] = {st->u, st->v, st->w, st->s, st->c};
    for (int q = 0; q < 5; ++q) F.p[q] = reinterpret_cast<V2<T> *>(sp[q]);
    return F;
}

template <typename T>
static gnss_status turb_stats_t(gnss_ctx *c, const gnss_fields *st, gnss_turb *out, double *yprof, cudaStream_t s) {
    gnss_status r = ensure_turb_buffers(c);
    if (r) return r;
    const FieldSet<T> F = fieldset_of<T>(st);
    if ((r = turb_spectral_t<T>(c, F, st->s != nullptr, s))) return r;
    if ((r = turb_vort_t<T>(c, F, s))) return r;
    return turb_finish(c, st->s != nullptr, out, yprof, s);
}

template <typename T> static bool zdiag_fits(const gnss_ctx *c) {
    GNSS_SIZE_SWITCH_OR(c->g.nz, return (Launch<T, NN_>::zreg_fits(c->n_phys, c->n_raw, c->ncp)), return false);
}

// One step with the calcTurbStats statistics of the state it starts from.  The
// spectral sums and profiles come from that state before the step; the
// vorticity sums from the physical vorticity the step's z kernel forms anyway
// (per-block rows into turb_part, zeroed first, summed after the step), where a
// register z kernel exists; elsewhere from three inverse transforms of the
// vorticity before the step.
template <typename T>
static gnss_status step_turb_t(gnss_ctx *c, const gnss_fields *st, const gnss_fields *hist, int euler, gnss_turb *out,
                               double *yprof, cudaStream_t s) {
    gnss_status r = ensure_turb_buffers(c);
    if (r) return r;
    const FieldSet<T> F = fieldset_of<T>(st);
    if ((r = turb_spectral_t<T>(c, F, st->s != nullptr, s))) return r;
    if (zdiag_fits<T>(c)) {
        CK(c, cudaMemsetAsync(c->turb_part, 0, sizeof(double) * STAT_BLOCKS * VORT_SUMS, s));
        if ((r = step_t<T>(c, st, hist, euler, s, nullptr, c->turb_part))) return r;
        c->launches++;
        k_sums_final<VORT_SUMS><<<1, VORT_SUMS * 32, 0, s>>>(c->turb_part, STAT_BLOCKS, VORT_SUMS,
                                                             c->turb_dev + TURB_SUMS);
        LAUNCH_CK(c);
    } else {
        if ((r = turb_vort_t<T>(c, F, s))) return r;
        if ((r = step_t<T>(c, st, hist, euler, s))) return r;
    }
    return turb_finish(c, st->s != nullptr, out, yprof, s);
}

// ============================================================== C ABI
// (C linkage comes from the declarations in gnss_b200.h)


const char *gnss_status_string(gnss_status st) {
    switch (st) {
        case GNSS_OK: return "ok";
        case GNSS_ERR_INVALID: return "invalid argument";
        case GNSS_ERR_CUDA: return "CUDA error";
        case GNSS_ERR_NOMEM: return "out of memory";
        case GNSS_ERR_UNSUPPORTED: return "unsupported";
        case GNSS_ERR_TIMEOUT: return "device wait timed out";
        default: return "unknown status";
    }
}

const char *gnss_last_error(const gnss_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

long long gnss_launch_count(const gnss_ctx *ctx) { return ctx ? ctx->launches : -1; }

gnss_status gnss_check(gnss_ctx *c, void *stream) {
    if (!c) return GNSS_ERR_INVALID;
    CK(c, cudaSetDevice(c->cfg.device));
    unsigned h = 0;
    CK(c, cudaMemcpyAsync(&h, c->d_err, sizeof h, cudaMemcpyDeviceToHost, S(stream)));
    CK(c, cudaStreamSynchronize(S(stream)));
    if (h) {
        CK(c, cudaMemsetAsync(c->d_err, 0, sizeof h, S(stream)));
        CK(c, cudaStreamSynchronize(S(stream)));
        return fail(c, GNSS_ERR_TIMEOUT, "a bounded device wait timed out (flags 0x%x)", h);
    }
    return GNSS_OK;
}

gnss_status gnss_stage_bytes(const gnss_ctx *c, double *bytes) {
    if (!c || !bytes) return GNSS_ERR_INVALID;
    const double e = (double)c->elem;
    const int nf = 3 + c->cfg.n_scalars;
    const double nkx = c->kx_keep.count(), nky = c->ky_keep.count();
    const double box = nky * nkx * c->nkz;                    // kept modes of one state field
    const double pe = (double)c->p_elems, qe = (double)c->q_elems;
    const double re = nky * nkx * c->ncp;                     // x-forward output
    bytes[0] = e * (c->n_xin * box + c->n_xout * pe);          // x inverse
    bytes[1] = e * (c->n_xout * pe + c->n_raw * qe);           // y inverse
    bytes[2] = e * (c->n_raw * qe + c->nnl * qe);              // z physical
    bytes[3] = e * (c->nnl * qe + c->nnl * pe);                // y forward
    bytes[4] = e * (c->nnl * pe + c->nnl * re);                // x forward
    const double sph = (double)c->n_sphere;
    bytes[5] = e * (c->nnl * sph + 4.0 * nf * sph);            // update (after the first step): nl, state, hist in;
                                                               // state, hist out, inside the sphere
    return GNSS_OK;
}

gnss_status gnss_set_option(gnss_ctx *c, int key, int value) {
    if (!c) return GNSS_ERR_INVALID;
    if (key == GNSS_OPT_TEST_WAIT) {   // poll cap of the z kernel's waits; block 0 withholds its first copy
        if (value < 0) return fail(c, GNSS_ERR_INVALID, "bad poll cap %d", value);
        CK(c, cudaSetDevice(c->cfg.device));
        const unsigned v = (unsigned)value;
        CK(c, cudaMemcpy(c->d_err + 1, &v, sizeof v, cudaMemcpyHostToDevice));
        c->test_wait = value;
        return GNSS_OK;
    }
    if (key != GNSS_OPT_ZVARIANT && key != GNSS_OPT_PVARIANT) return fail(c, GNSS_ERR_INVALID, "unknown option %d", key);
    const int top = key == GNSS_OPT_ZVARIANT ? GNSS_VARIANT_WARPSPEC : GNSS_VARIANT_TENSOR;
    if (value < GNSS_VARIANT_AUTO || value > top || (key == GNSS_OPT_PVARIANT && value == GNSS_VARIANT_WARPSPEC))
        return fail(c, GNSS_ERR_INVALID, "bad variant %d for option %d", value, key);
    (key == GNSS_OPT_ZVARIANT ? c->zvariant : c->pvariant) = value;
    return GNSS_OK;
}

template <typename T> static int zkernel_of(const gnss_ctx *c) {
    GNSS_SIZE_SWITCH_OR(c->g.nz,
                        return (Launch<T, NN_>::zkernel(c->zvariant, c->n_phys, c->n_raw, c->nnl, c->ncp)),
                        return GNSS_VARIANT_STAGED);
}

gnss_status gnss_get_option(const gnss_ctx *c, int key, int *value) {
    if (!c || !value) return GNSS_ERR_INVALID;
    if (key == GNSS_OPT_ZVARIANT) *value = c->zvariant;
    else if (key == GNSS_OPT_PVARIANT) *value = c->pvariant;
    else if (key == GNSS_OPT_TEST_WAIT) *value = c->test_wait;
    else if (key == GNSS_OPT_ZKERNEL)
        *value = c->cfg.precision == GNSS_FP64 ? zkernel_of<double>(c) : zkernel_of<float>(c);
    else return GNSS_ERR_INVALID;
    return GNSS_OK;
}

gnss_status gnss_profile_enable(gnss_ctx *c, int on) {
    if (!c) return GNSS_ERR_INVALID;
    c->profiling = on != 0;
    c->ev_rec.clear();
    return GNSS_OK;
}

gnss_status gnss_profile_read(gnss_ctx *c, double *ms, long long *launches) {
    if (!c || !ms || !launches) return fail(c, GNSS_ERR_INVALID, "null argument");
    for (int k = 0; k < GNSS_NSTAGES; ++k) { ms[k] = 0.0; launches[k] = 0; }
    for (auto &r : c->ev_rec) {
        CK(c, cudaEventSynchronize(c->ev_pool[r.second.second]));
        float t = 0.f;
        CK(c, cudaEventElapsedTime(&t, c->ev_pool[r.second.first], c->ev_pool[r.second.second]));
        ms[r.first] += t;
        launches[r.first] += 1;
    }
    c->ev_rec.clear();
    return GNSS_OK;
}

size_t gnss_field_bytes(const gnss_ctx *ctx) { return ctx ? ctx->nspec * ctx->elem : 0; }

gnss_status gnss_get_config(const gnss_ctx *ctx, gnss_config *out) {
    if (!ctx || !out) return GNSS_ERR_INVALID;
    *out = ctx->cfg;
    return GNSS_OK;
}
size_t gnss_workspace_bytes(const gnss_ctx *ctx) { return ctx ? ctx->owned_bytes : 0; }

// scratch fields any operation of this context can ask for (the step's, or one field for the transforms)
static int scratch_fields_max(const gnss_ctx *c) {
    const size_t need = step_scratch_elems(c);
    const int nf = (int)((need + c->nspec - 1) / c->nspec);
    return nf > 1 ? nf : 1;
}

size_t gnss_scratch_bytes(const gnss_ctx *c) {
    return c ? (size_t)scratch_fields_max(c) * c->nspec * c->elem : 0;
}

gnss_status gnss_attach_scratch(gnss_ctx *c, void *ptr, size_t bytes) {
    if (!c) return GNSS_ERR_INVALID;
    if (!ptr || (reinterpret_cast<uintptr_t>(ptr) % 256) != 0)
        return fail(c, GNSS_ERR_INVALID, "scratch must be a 256-byte aligned device pointer");
    if (bytes < gnss_scratch_bytes(c))
        return fail(c, GNSS_ERR_INVALID, "scratch of %zu bytes, %zu needed", bytes, gnss_scratch_bytes(c));
    CK(c, cudaSetDevice(c->cfg.device));
    if (c->scratch && !c->scratch_ext) {
        cudaFree(c->scratch);
        c->owned_bytes -= (size_t)c->nscratch * c->nspec * c->elem;
    }
    c->scratch = ptr;
    c->scratch_ext = true;
    c->nscratch = (int)(bytes / (c->nspec * c->elem));
    return GNSS_OK;
}

template <typename T> static void *make_twiddles(int n, gnss_ctx *c) {
    std::vector<V2<T>> h(n);
    const long double twopi = 6.283185307179586476925286766559L;
    for (int k = 0; k < n; ++k) {
        long double a = twopi * (long double)k / (long double)n;
        h[k].x = (T)cosl(a);
        h[k].y = (T)(-sinl(a));
    }
    void *d = nullptr;
    if (cudaMalloc(&d, sizeof(V2<T>) * n) != cudaSuccess) return nullptr;
    if (cudaMemcpy(d, h.data(), sizeof(V2<T>) * n, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d);
        return nullptr;
    }
    c->owned_bytes += sizeof(V2<T>) * n;
    return d;
}

// Derivatives are split across the passes: kx factors in the x inverse, ky
// factors in the y inverse, kz factors and the two-field combinations of the
// vorticity (solver.cu:68-114) in the z pass.
//   x inverse (state -> P):  P0 X[u] P1 X[v] P2 X[w] P3 X[s] P4 X[ikx v] P5 X[ikx w]
//                            P6 X[ikx s] [P7 X[c] P8 X[ikx c]] [P9 X[-k^2 s]]
//   y inverse (P -> Q):      Q0 U00 Q1 V00 Q2 W00 Q3 S00 Q4 U01 Q5 W01 Q6 S01
//                            Q7 V10 Q8 W10 Q9 S10 [Q10 C00 Q11 C01 Q12 C10] [Q13 L00]
//   (first index: i kx applied, second: i ky applied)
//   z pass:  u = U00, v = V00, w = W00, w1 = W01 - ikz V00, w2 = ikz U00 - W10,
//            w3 = V10 - U01, sx = S10, sy = S01, sz = ikz S00,
//            [cx = C10, cy = C01, cz = ikz C00], [c = C00, lap s = L00]
static void set_recipes(gnss_ctx *c) {
    const bool two = c->cfg.n_scalars > 1, al = two && c->cfg.alpha != 0.0;
    auto xv = [&](int in, int var, int mul, int out) {
        c->xvar_mul[in][var] = (signed char)mul;
        c->xvar_out[in][var] = (signed char)out;
        if (c->xvar_n[in] < var + 1) c->xvar_n[in] = (signed char)(var + 1);
    };
    for (int i = 0; i < 5; ++i) c->xvar_in[i] = (signed char)i;
    xv(0, 0, V_ONE, 0);
    xv(1, 0, V_ONE, 1); xv(1, 1, V_IK_ROW, 4);
    xv(2, 0, V_ONE, 2); xv(2, 1, V_IK_ROW, 5);
    xv(3, 0, V_ONE, 3); xv(3, 1, V_IK_ROW, 6);
    c->n_xin = 4;
    c->n_xout = 7;
    if (two) {
        xv(4, 0, V_ONE, 7); xv(4, 1, V_IK_ROW, 8);
        c->n_xin = 5;
        c->n_xout = 9;
        if (al) {   // s a second time, for -k^2 s
            c->xvar_in[5] = 3;
            xv(5, 0, V_LAP, 9);
            c->n_xin = 6;
            c->n_xout = 10;
        }
    }
    auto yv = [&](int in, int var, int mul, int out) {
        c->yvar_mul[in][var] = (signed char)mul;
        c->yvar_out[in][var] = (signed char)out;
        if (c->yvar_n[in] < var + 1) c->yvar_n[in] = (signed char)(var + 1);
    };
    yv(0, 0, V_ONE, 0); yv(0, 1, V_IK_ROW, 4);    // X[u]     -> U00, U01
    yv(1, 0, V_ONE, 1);                           // X[v]     -> V00
    yv(2, 0, V_ONE, 2); yv(2, 1, V_IK_ROW, 5);    // X[w]     -> W00, W01
    yv(3, 0, V_ONE, 3); yv(3, 1, V_IK_ROW, 6);    // X[s]     -> S00, S01
    yv(4, 0, V_ONE, 7);                           // X[ikx v] -> V10
    yv(5, 0, V_ONE, 8);                           // X[ikx w] -> W10
    yv(6, 0, V_ONE, 9);                           // X[ikx s] -> S10
    c->n_raw = 10;
    if (two) {
        yv(7, 0, V_ONE, 10); yv(7, 1, V_IK_ROW, 11);   // X[c]     -> C00, C01
        yv(8, 0, V_ONE, 12);                           // X[ikx c] -> C10
        c->n_raw = 13;
        if (al) { yv(9, 0, V_ONE, 13); c->n_raw = 14; }   // X[-k^2 s] -> L00
    }
    auto zq = [&](int q, int r0, int k0, int s0, int r1 = -1, int k1 = 0, int s1 = 1) {
        ZRecipe &z = c->zrec.q[q];
        z.r[0] = (signed char)r0; z.ikz[0] = (signed char)k0; z.sgn[0] = (signed char)s0;
        z.r[1] = (signed char)r1; z.ikz[1] = (signed char)k1; z.sgn[1] = (signed char)s1;
    };
    zq(0, 0, 0, 1);               // u
    zq(1, 1, 0, 1);               // v
    zq(2, 2, 0, 1);               // w
    zq(3, 5, 0, 1, 1, 1, -1);     // w1 = W01 - ikz V00
    zq(4, 0, 1, 1, 8, 0, -1);     // w2 = ikz U00 - W10
    zq(5, 7, 0, 1, 4, 0, -1);     // w3 = V10 - U01
    zq(6, 9, 0, 1);               // sx
    zq(7, 6, 0, 1);               // sy
    zq(8, 3, 1, 1);               // sz
    c->n_phys = 9;
    c->nnl = 4;
    if (two) {
        zq(9, 12, 0, 1);          // cx
        zq(10, 11, 0, 1);         // cy
        zq(11, 10, 1, 1);         // cz
        c->n_phys = 12;
        c->nnl = 5;
        if (al) {
            zq(12, 10, 0, 1);     // c
            zq(13, 13, 0, 1);     // lap s
            c->n_phys = 14;
        }
    }
}

// Kept indices of one axis: i is kept when its wavenumber alone does not
// exceed the truncation radius (the test of solver.cu:36 restricted to one
// axis); with the Nyquist index kept, every index is.
static KeepMap keep_of(int n, double dk, double kmax2) {
    const double kn = dk * ((double)(n / 2) - (double)n);
    if (kn * kn <= kmax2) return KeepMap{n, -1};
    int K = 0;
    while (K + 1 < n / 2 && (dk * (double)(K + 1)) * (dk * (double)(K + 1)) <= kmax2) ++K;
    return KeepMap{n, K};
}

static void set_layout(gnss_ctx *c) {
    const Geom &g = c->g;
    c->kx_keep = keep_of(g.nx, g.dkx, g.kmax2);
    c->ky_keep = keep_of(g.ny, g.dky, g.kmax2);
    const KeepMap kz = keep_of(g.nz, g.dkz, g.kmax2);
    c->nkz = kz.K < 0 ? g.nz2 : kz.K + 1;
    c->herm_row = c->ky_keep.K < 0 && g.ny % 2 == 0;
    c->herm_col = c->kx_keep.K < 0 && g.nx % 2 == 0;
    c->herm_plane = kz.K < 0 && g.nz % 2 == 0;
    c->ncp = (c->nkz + 15) / 16 * 16;
    c->p_elems = (size_t)g.nx * c->ky_keep.count() * c->ncp;
    c->q_elems = (size_t)g.nx * g.ny * c->ncp;
    // modes of the kept box inside the dealiasing sphere (the ones k_update touches after the first step)
    auto wn = [](int i, int n, double dk) { return (i < n / 2) ? dk * (double)i : dk * ((double)i - (double)n); };
    c->n_sphere = 0;
    for (int yc = 0; yc < c->ky_keep.count(); ++yc) {
        const double k2 = wn(c->ky_keep.expand(yc), g.ny, g.dky);
        for (int xc = 0; xc < c->kx_keep.count(); ++xc) {
            const double k1 = wn(c->kx_keep.expand(xc), g.nx, g.dkx);
            const double t = k1 * k1 + k2 * k2;
            for (int z = 0; z < c->nkz; ++z) {
                const double k3 = wn(z, g.nz, g.dkz);
                if (t + k3 * k3 > g.kmax2) break;
                ++c->n_sphere;
            }
        }
    }
}

gnss_status gnss_create(const gnss_config *cfg, gnss_ctx **out) {
    if (!cfg || !out) return GNSS_ERR_INVALID;
    *out = nullptr;
    const gnss_config &k = *cfg;
    if (!size_ok(k.nx) || !size_ok(k.ny) || !size_ok(k.nz)) return GNSS_ERR_INVALID;
    if (k.n_scalars < 1 || k.n_scalars > 2) return GNSS_ERR_INVALID;
    if (k.scheme != GNSS_SCHEME_CNAB2 && k.scheme != GNSS_SCHEME_RK3IF) return GNSS_ERR_INVALID;
    if (k.precision != GNSS_FP64 && k.precision != GNSS_FP32) return GNSS_ERR_INVALID;
    if (!(k.lx > 0 && k.ly > 0 && k.lz > 0 && k.re > 0 && k.sc > 0 && k.sc_c > 0 && k.dt > 0)) return GNSS_ERR_INVALID;
    if (!(k.alias_filter > 0)) return GNSS_ERR_INVALID;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || k.device < 0 || k.device >= ndev) {
        cudaGetLastError();
        return GNSS_ERR_CUDA;
    }
    if (cudaSetDevice(k.device) != cudaSuccess) return GNSS_ERR_CUDA;
    gnss_ctx *c = new gnss_ctx;
    c->cfg = k;
    Geom &g = c->g;
    g.nx = k.nx; g.ny = k.ny; g.nz = k.nz; g.nz2 = k.nz / 2 + 1;
    g.dkx = 2 * M_PI / k.lx;     // (2*PI/l) as in waveNumber_kernel (initialize.cu:686-689)
    g.dky = 2 * M_PI / k.ly;
    g.dkz = 2 * M_PI / k.lz;
    const double kx_max = k.nx * M_PI / k.lx;    // solver.cu:29
    const double k_max = k.alias_filter * kx_max;  // solver.cu:31
    g.kmax2 = k_max * k_max;
    c->nspec = (size_t)k.nx * k.ny * g.nz2;
    c->elem = k.precision == GNSS_FP64 ? sizeof(double2) : sizeof(float2);
    set_recipes(c);
    set_layout(c);
    const int ns[3] = {k.nx, k.ny, k.nz};
    for (int a = 0; a < 3; ++a) {
        c->tw[a] = k.precision == GNSS_FP64 ? make_twiddles<double>(ns[a], c) : make_twiddles<float>(ns[a], c);
        if (!c->tw[a]) { gnss_destroy(c); return GNSS_ERR_NOMEM; }
    }
    if (cudaMalloc(&c->stat_part, sizeof(double) * STAT_BLOCKS * STAT_SUMS) != cudaSuccess ||
        cudaMalloc(&c->stat_dev, sizeof(double) * STAT_SUMS) != cudaSuccess ||
        cudaMallocHost(&c->stat_host, sizeof(double) * STAT_SUMS) != cudaSuccess) {
        cudaGetLastError();
        gnss_destroy(c);
        return GNSS_ERR_NOMEM;
    }
    c->owned_bytes += sizeof(double) * (STAT_BLOCKS * STAT_SUMS + STAT_SUMS);
    if (cudaMalloc(&c->d_err, 2 * sizeof(unsigned)) != cudaSuccess ||
        cudaMemset(c->d_err, 0, 2 * sizeof(unsigned)) != cudaSuccess) {
        cudaGetLastError();
        gnss_destroy(c);
        return GNSS_ERR_NOMEM;
    }
    if (k.precision == GNSS_FP32) {   // the mean-profile line in FP64 (k_update); zero: taken from the fields
        const size_t mb = sizeof(double2) * 10 * (size_t)k.ny;
        if (cudaMalloc(&c->mean64, mb) != cudaSuccess || cudaMemset(c->mean64, 0, mb) != cudaSuccess) {
            cudaGetLastError();
            gnss_destroy(c);
            return GNSS_ERR_NOMEM;
        }
        c->owned_bytes += mb;
    }
    if (cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, k.device) != cudaSuccess) {
        cudaGetLastError();
        gnss_destroy(c);
        return GNSS_ERR_CUDA;
    }
    *out = c;
    return GNSS_OK;
}

gnss_status gnss_destroy(gnss_ctx *c) {
    if (!c) return GNSS_ERR_INVALID;
    cudaSetDevice(c->cfg.device);
    for (int a = 0; a < 3; ++a) if (c->tw[a]) cudaFree(c->tw[a]);
    if (c->scratch && !c->scratch_ext) cudaFree(c->scratch);
    if (c->stat_part) cudaFree(c->stat_part);
    if (c->stat_dev) cudaFree(c->stat_dev);
    if (c->stat_host) cudaFreeHost(c->stat_host);
    if (c->turb_part) cudaFree(c->turb_part);
    if (c->turb_dev) cudaFree(c->turb_dev);
    if (c->turb_host) cudaFreeHost(c->turb_host);
    if (c->d_err) cudaFree(c->d_err);
    if (c->mean64) cudaFree(c->mean64);
    if (c->res) cudaFree(c->res);
    if (c->run_sums) cudaFree(c->run_sums);
    if (c->run_sums_host) cudaFreeHost(c->run_sums_host);
    for (cudaEvent_t e : c->side_ev) if (e) cudaEventDestroy(e);
    if (c->side) cudaStreamDestroy(c->side);
    for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
    delete c;
    return GNSS_OK;
}

#define PREC_CALL(c, fn, ...) ((c)->cfg.precision == GNSS_FP64 ? fn<double>(__VA_ARGS__) : fn<float>(__VA_ARGS__))

gnss_status gnss_turb_stats(gnss_ctx *c, const gnss_fields *state, gnss_turb *out, double *yprof, void *stream) {
    if (!c || !state || !out || !state->u || !state->v || !state->w)
        return fail(c, GNSS_ERR_INVALID, "null argument");
    if (!al_fields(c, state)) return fail(c, GNSS_ERR_INVALID, "misaligned pointer");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, turb_stats_t, c, state, out, yprof, S(stream));
}

gnss_status gnss_forward(gnss_ctx *c, void *f, void *stream) {
    if (!c || !f) return fail(c, GNSS_ERR_INVALID, "null argument");
    if (!al(c, f)) return fail(c, GNSS_ERR_INVALID, "misaligned pointer");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, forward_t, c, f, S(stream));
}

gnss_status gnss_inverse(gnss_ctx *c, void *f, void *stream) {
    if (!c || !f) return fail(c, GNSS_ERR_INVALID, "null argument");
    if (!al(c, f)) return fail(c, GNSS_ERR_INVALID, "misaligned pointer");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, inverse_t, c, f, S(stream));
}

template <typename T> static gnss_status dealias_t(gnss_ctx *c, void *f, cudaStream_t s) {
    c->launches++;
    k_dealias<T><<<grid_for((long long)c->nspec, 256), 256, 0, s>>>(reinterpret_cast<V2<T> *>(f), c->g);
    LAUNCH_CK(c);
    return GNSS_OK;
}
gnss_status gnss_dealias(gnss_ctx *c, void *f, void *stream) {
    if (!c || !f) return fail(c, GNSS_ERR_INVALID, "null argument");
    if (!al(c, f)) return fail(c, GNSS_ERR_INVALID, "misaligned pointer");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, dealias_t, c, f, S(stream));
}

template <typename T>
static gnss_status vort_t(gnss_ctx *c, const void *u, const void *v, const void *w, void *o1, void *o2, void *o3,
                          cudaStream_t s) {
    using V = V2<T>;
    c->launches++;
    k_vorticity<T><<<grid_for((long long)c->nspec, 256), 256, 0, s>>>(
        (const V *)u, (const V *)v, (const V *)w, (V *)o1, (V *)o2, (V *)o3, c->g);
    LAUNCH_CK(c);
    return GNSS_OK;
}
gnss_status gnss_vorticity(gnss_ctx *c, const void *uh, const void *vh, const void *wh, void *o1, void *o2, void *o3,
                           void *stream) {
    if (!c || !uh || !vh || !wh || !o1 || !o2 || !o3) return fail(c, GNSS_ERR_INVALID, "null argument");
    if (!al(c, uh) || !al(c, vh) || !al(c, wh) || !al(c, o1) || !al(c, o2) || !al(c, o3)) return fail(c, GNSS_ERR_INVALID, "misaligned pointer");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, vort_t, c, uh, vh, wh, o1, o2, o3, S(stream));
}

template <typename T>
static gnss_status grad_t(gnss_ctx *c, const void *f, void *x, void *y, void *z, cudaStream_t s) {
    using V = V2<T>;
    c->launches++;
    k_gradient<T><<<grid_for((long long)c->nspec, 256), 256, 0, s>>>((const V *)f, (V *)x, (V *)y, (V *)z, c->g);
    LAUNCH_CK(c);
    return GNSS_OK;
}
gnss_status gnss_gradient(gnss_ctx *c, const void *fh, void *fx, void *fy, void *fz, void *stream) {
    if (!c || !fh || !fx || !fy || !fz) return fail(c, GNSS_ERR_INVALID, "null argument");
    if (!al(c, fh) || !al(c, fx) || !al(c, fy) || !al(c, fz)) return fail(c, GNSS_ERR_INVALID, "misaligned pointer");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, grad_t, c, fh, fx, fy, fz, S(stream));
}

template <typename T>
static gnss_status divg_t(gnss_ctx *c, const void *x, const void *y, const void *z, void *o, cudaStream_t s) {
    using V = V2<T>;
    c->launches++;
    k_divergence<T><<<grid_for((long long)c->nspec, 256), 256, 0, s>>>((const V *)x, (const V *)y, (const V *)z,
                                                                        (V *)o, c->g);
    LAUNCH_CK(c);
    return GNSS_OK;
}
gnss_status gnss_divergence(gnss_ctx *c, const void *fx, const void *fy, const void *fz, void *out, void *stream) {
    if (!c || !fx || !fy || !fz || !out) return fail(c, GNSS_ERR_INVALID, "null argument");
    if (!al(c, fx) || !al(c, fy) || !al(c, fz) || !al(c, out)) return fail(c, GNSS_ERR_INVALID, "misaligned pointer");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, divg_t, c, fx, fy, fz, out, S(stream));
}

template <typename T>
static gnss_status rhs_t(gnss_ctx *c, void *ru, void *rv, void *rw, void *rs, void *rc, cudaStream_t s) {
    using V = V2<T>;
    c->launches++;
    k_make_rhs<T><<<grid_for((long long)c->nspec, 256), 256, 0, s>>>((V *)ru, (V *)rv, (V *)rw, (V *)rs, (V *)rc,
                                                                      c->g);
    LAUNCH_CK(c);
    return GNSS_OK;
}
gnss_status gnss_make_rhs(gnss_ctx *c, void *ru, void *rv, void *rw, void *rs, void *rc, void *stream) {
    if (!c || !ru || !rv || !rw) return fail(c, GNSS_ERR_INVALID, "null argument");
    if (!al(c, ru) || !al(c, rv) || !al(c, rw) || !al(c, rs) || !al(c, rc)) return fail(c, GNSS_ERR_INVALID, "misaligned pointer");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, rhs_t, c, ru, rv, rw, rs, rc, S(stream));
}

template <typename T>
static gnss_status timestep_t(gnss_ctx *c, int euler, const gnss_fields *st, const gnss_fields *r,
                              const gnss_fields *ro, cudaStream_t s) {
    using V = V2<T>;
    UpdCoef u = base_coef(c);
    const gnss_config &k = c->cfg;
    const double num[5] = {k.re, k.re, k.re, k.re * k.sc, k.re * k.sc_c};   // solver.cu:599-611
    void *f[5] = {st->u, st->v, st->w, st->s, st->c};
    void *rr[5] = {r->u, r->v, r->w, r->s, r->c};
    void *oo[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    if (ro) { oo[0] = ro->u; oo[1] = ro->v; oo[2] = ro->w; oo[3] = ro->s; oo[4] = ro->c; }
    for (int q = 0; q < 5; ++q) {
        if (!f[q]) continue;
        if (!rr[q] || (!euler && !oo[q])) return fail(c, GNSS_ERR_INVALID, "missing rhs field %d", q);
        c->launches++;
        k_timestep<T><<<grid_for((long long)c->nspec, 256), 256, 0, s>>>((V *)f[q], (const V *)rr[q],
                                                                          (const V *)oo[q], num[q], u.dt, euler,
                                                                          c->g);
        LAUNCH_CK(c);
    }
    return GNSS_OK;
}
gnss_status gnss_timestep(gnss_ctx *c, int euler, const gnss_fields *state, const gnss_fields *rhs,
                          const gnss_fields *rhs_old, void *stream) {
    if (!c || !state || !rhs || (!euler && !rhs_old)) return fail(c, GNSS_ERR_INVALID, "null argument");
    if (!al_fields(c, state) || !al_fields(c, rhs) || !al_fields(c, rhs_old))
        return fail(c, GNSS_ERR_INVALID, "misaligned pointer");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, timestep_t, c, euler, state, rhs, rhs_old, S(stream));
}

template <typename T>
static gnss_status upd_t(gnss_ctx *c, const gnss_fields *r, const gnss_fields *ro, cudaStream_t s) {
    using V = V2<T>;
    void *rr[5] = {r->u, r->v, r->w, r->s, r->c};
    void *oo[5] = {ro->u, ro->v, ro->w, ro->s, ro->c};
    for (int q = 0; q < 5; ++q) {
        if (!rr[q] && !oo[q]) continue;
        if (!rr[q] || !oo[q]) return fail(c, GNSS_ERR_INVALID, "field %d given on one side only", q);
        c->launches++;
        k_shift_history<T><<<grid_for((long long)c->nspec, 256), 256, 0, s>>>((V *)rr[q], (V *)oo[q],
                                                                               (long long)c->nspec);
        LAUNCH_CK(c);
    }
    return GNSS_OK;
}
gnss_status gnss_update(gnss_ctx *c, const gnss_fields *rhs, const gnss_fields *rhs_old, void *stream) {
    if (!c || !rhs || !rhs_old) return fail(c, GNSS_ERR_INVALID, "null argument");
    if (!al_fields(c, rhs) || !al_fields(c, rhs_old)) return fail(c, GNSS_ERR_INVALID, "misaligned pointer");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, upd_t, c, rhs, rhs_old, S(stream));
}

static long long npoints(const gnss_ctx *c) { return (long long)c->g.nx * c->g.ny * c->g.nz; }

template <typename T>
static gnss_status cross_t(gnss_ctx *c, const void *u, const void *v, const void *w, void *o1, void *o2, void *o3,
                           cudaStream_t s) {
    c->launches++;
    k_cross<T><<<grid_for(npoints(c), 256), 256, 0, s>>>((const T *)u, (const T *)v, (const T *)w, (T *)o1, (T *)o2,
                                                          (T *)o3, c->g);
    LAUNCH_CK(c);
    return GNSS_OK;
}
gnss_status gnss_cross_product(gnss_ctx *c, const void *u, const void *v, const void *w, void *o1, void *o2, void *o3,
                               void *stream) {
    if (!c || !u || !v || !w || !o1 || !o2 || !o3) return fail(c, GNSS_ERR_INVALID, "null argument");
    if (!al(c, u) || !al(c, v) || !al(c, w) || !al(c, o1) || !al(c, o2) || !al(c, o3)) return fail(c, GNSS_ERR_INVALID, "misaligned pointer");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, cross_t, c, u, v, w, o1, o2, o3, S(stream));
}

template <typename T>
static gnss_status dot_t(gnss_ctx *c, const void *a1, const void *a2, const void *a3, const void *b1, const void *b2,
                         const void *b3, void *o, cudaStream_t s) {
    c->launches++;
    k_dot<T><<<grid_for(npoints(c), 256), 256, 0, s>>>((const T *)a1, (const T *)a2, (const T *)a3, (const T *)b1,
                                                        (const T *)b2, (const T *)b3, (T *)o, c->g);
    LAUNCH_CK(c);
    return GNSS_OK;
}
gnss_status gnss_dot_product(gnss_ctx *c, const void *a1, const void *a2, const void *a3, const void *b1,
                             const void *b2, const void *b3, void *out, void *stream) {
    if (!c || !a1 || !a2 || !a3 || !b1 || !b2 || !b3 || !out) return fail(c, GNSS_ERR_INVALID, "null argument");
    if (!al(c, a1) || !al(c, a2) || !al(c, a3) || !al(c, b1) || !al(c, b2) || !al(c, b3) || !al(c, out)) return fail(c, GNSS_ERR_INVALID, "misaligned pointer");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, dot_t, c, a1, a2, a3, b1, b2, b3, out, S(stream));
}

template <typename T>
static gnss_status colloid_t(gnss_ctx *c, const void *u, const void *v, const void *w, const void *cc, const void *cx,
                             const void *cy, const void *cz, const void *sx, const void *sy, const void *sz, void *lap,
                             cudaStream_t s) {
    c->launches++;
    k_colloid<T><<<grid_for(npoints(c), 256), 256, 0, s>>>(
        (const T *)u, (const T *)v, (const T *)w, (const T *)cc, (const T *)cx, (const T *)cy, (const T *)cz,
        (const T *)sx, (const T *)sy, (const T *)sz, (T *)lap, (T)c->cfg.alpha, c->g);
    LAUNCH_CK(c);
    return GNSS_OK;
}
gnss_status gnss_colloid_advection(gnss_ctx *c, const void *u, const void *v, const void *w, const void *cc,
                                   const void *cx, const void *cy, const void *cz, const void *sx, const void *sy,
                                   const void *sz, void *lap_s_inout, void *stream) {
    if (!c || !u || !v || !w || !cc || !cx || !cy || !cz || !sx || !sy || !sz || !lap_s_inout)
        return fail(c, GNSS_ERR_INVALID, "null argument");
    if (!al(c, u) || !al(c, v) || !al(c, w) || !al(c, cc) || !al(c, cx) || !al(c, cy) || !al(c, cz) || !al(c, sx) || !al(c, sy) || !al(c, sz) || !al(c, lap_s_inout)) return fail(c, GNSS_ERR_INVALID, "misaligned pointer");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, colloid_t, c, u, v, w, cc, cx, cy, cz, sx, sy, sz, lap_s_inout, S(stream));
}

static bool state_ok(const gnss_ctx *c, const gnss_fields *st) {
    if (!st || !st->u || !st->v || !st->w || !st->s) return false;
    if (c->cfg.n_scalars > 1 && !st->c) return false;
    return true;
}

// ============================================================== batches (the ensemble's size groups)
static_assert(GNSS_BATCH_MAX <= MAXM, "batch size");

size_t gnss_batch_scratch_bytes(const gnss_ctx *c) { return c ? step_scratch_elems(c) * c->elem : 0; }

template <typename T>
static gnss_status step_batch_t(gnss_ctx *const *cs, int n, const gnss_fields *st0, const gnss_fields *hi0,
                                long long ms_sh, void *scratch, long long ms_scr, int euler, cudaStream_t s) {
    gnss_ctx *c = cs[0];
    UpdCoef uc = base_coef(c);
    uc.euler = euler ? 1 : 0;
    MemberCoef mc{};
    for (int m = 0; m < n; ++m) {
        const UpdCoef u = base_coef(cs[m]);
        mc.dt[m] = u.dt;
        for (int q = 0; q < 5; ++q) {
            mc.hnum[m][q] = u.hnum[q];
            mc.nu[m][q] = u.nu[q];
        }
        mc.mean[m] = cs[m]->mean64;
    }
    Batch bt;
    bt.nmem = n;
    bt.ms_sh = ms_sh;
    bt.ms_scr = ms_scr;
    bt.scratch = scratch;
    bt.mc = &mc;
    return nonlinear_and_update<T>(c, st0, nullptr, hi0, uc, s, nullptr, nullptr, bt);
}

bool gnss_batch_supported(const gnss_ctx *c) {
    if (!c || c->cfg.scheme != GNSS_SCHEME_CNAB2) return false;
    const int zk = c->cfg.precision == GNSS_FP64 ? zkernel_of<double>(c) : zkernel_of<float>(c);
    return zk == GNSS_VARIANT_REGISTER && zr_size(c->g.nx) && zr_size(c->g.ny);
}

gnss_status gnss_step_batch(gnss_ctx *const *cs, int n, const gnss_fields *st0, const gnss_fields *hi0,
                            size_t member_bytes, void *scratch, size_t scratch_bytes, int euler, void *stream) {
    if (!cs || n < 1 || n > GNSS_BATCH_MAX || !cs[0] || !scratch) return GNSS_ERR_INVALID;
    gnss_ctx *c = cs[0];
    const gnss_config &k = c->cfg;
    if (!gnss_batch_supported(c))
        return fail(c, GNSS_ERR_UNSUPPORTED, "batched steps need the CN/AB2 scheme and the register kernels");
    for (int m = 1; m < n; ++m) {
        const gnss_config &o = cs[m] ? cs[m]->cfg : k;
        if (!cs[m] || o.nx != k.nx || o.ny != k.ny || o.nz != k.nz || o.precision != k.precision ||
            o.n_scalars != k.n_scalars || o.scheme != k.scheme || o.alpha != k.alpha || o.device != k.device ||
            o.lx != k.lx || o.ly != k.ly || o.lz != k.lz || o.alias_filter != k.alias_filter)
            return fail(c, GNSS_ERR_INVALID, "member %d of a batch has another geometry", m);
    }
    if (!state_ok(c, st0) || !state_ok(c, hi0)) return fail(c, GNSS_ERR_INVALID, "state or history fields missing");
    if (!al_fields(c, st0) || !al_fields(c, hi0) || member_bytes % c->elem || scratch_bytes % 256 ||
        reinterpret_cast<uintptr_t>(scratch) % 256 || scratch_bytes < gnss_batch_scratch_bytes(c))
        return fail(c, GNSS_ERR_INVALID, "misaligned or short batch buffers");
    CK(c, cudaSetDevice(k.device));
    const long long ms_sh = (long long)(member_bytes / c->elem), ms_scr = (long long)(scratch_bytes / c->elem);
    return PREC_CALL(c, step_batch_t, cs, n, st0, hi0, ms_sh, scratch, ms_scr, euler, S(stream));
}


gnss_status gnss_step(gnss_ctx *c, const gnss_fields *state, const gnss_fields *hist, int euler, void *stream) {
    if (!c) return GNSS_ERR_INVALID;
    if (!state_ok(c, state)) return fail(c, GNSS_ERR_INVALID, "state fields missing");
    if (c->cfg.scheme == GNSS_SCHEME_CNAB2 && !state_ok(c, hist))
        return fail(c, GNSS_ERR_INVALID, "history fields missing");
    if (!al_fields(c, state) || !al_fields(c, hist)) return fail(c, GNSS_ERR_INVALID, "misaligned pointer");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, step_t, c, state, hist, euler, S(stream));
}

gnss_status gnss_step_turb(gnss_ctx *c, const gnss_fields *state, const gnss_fields *hist, int euler, gnss_turb *out,
                           double *yprof, void *stream) {
    if (!c || !out) return fail(c, GNSS_ERR_INVALID, "null argument");
    if (!state_ok(c, state)) return fail(c, GNSS_ERR_INVALID, "state fields missing");
    if (c->cfg.scheme == GNSS_SCHEME_CNAB2 && !state_ok(c, hist))
        return fail(c, GNSS_ERR_INVALID, "history fields missing");
    if (!al_fields(c, state) || !al_fields(c, hist)) return fail(c, GNSS_ERR_INVALID, "misaligned pointer");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, step_turb_t, c, state, hist, euler, out, yprof, S(stream));
}

gnss_status gnss_stats(gnss_ctx *c, const gnss_fields *state, double *out, void *stream) {
    if (!c || !out) return fail(c, GNSS_ERR_INVALID, "null argument");
    if (!state || !state->u || !state->v || !state->w) return fail(c, GNSS_ERR_INVALID, "state fields missing");
    if (!al_fields(c, state)) return fail(c, GNSS_ERR_INVALID, "misaligned pointer");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, stats_t, c, state, out, S(stream));
}

// Strided copy of the sub-box ky in [y0, y0 + ny) x kx in [x0, x0 + nx) x
// kz in [z0, z0 + nz) of one spectral field ([ky][kx][nz2]); nothing when a
// count is zero.  Adds the bytes copied to *bytes.
static cudaError_t copy_sub_box(const gnss_ctx *c, void *dst, const void *src, int y0, int ny, int x0, int nx, int z0,
                                int nz, cudaMemcpyKind kind, cudaStream_t s, size_t *bytes) {
    if (ny <= 0 || nx <= 0 || nz <= 0) return cudaSuccess;
    const size_t pitch = (size_t)c->g.nz2 * c->elem;
    cudaMemcpy3DParms p{};
    p.srcPtr = make_cudaPitchedPtr(const_cast<void *>(src), pitch, pitch, (size_t)c->g.nx);
    p.dstPtr = make_cudaPitchedPtr(dst, pitch, pitch, (size_t)c->g.nx);
    p.srcPos = make_cudaPos((size_t)z0 * c->elem, (size_t)x0, (size_t)y0);
    p.dstPos = p.srcPos;
    p.extent = make_cudaExtent((size_t)nz * c->elem, (size_t)nx, (size_t)ny);
    p.kind = kind;
    *bytes += p.extent.width * p.extent.height * p.extent.depth;
    return cudaMemcpy3DAsync(&p, s);
}

// Index ranges [first, first + count) of the kept indices of one axis, and
// the one range of dropped indices (count 0 when every index is kept).
static int keep_ranges(const KeepMap &m, int first[2], int count[2], int *drop_first, int *drop_count) {
    if (m.K < 0) {
        first[0] = 0;
        count[0] = m.n;
        *drop_first = *drop_count = 0;
        return 1;
    }
    first[0] = 0;
    count[0] = m.K + 1;
    first[1] = m.n - m.K;   // K < n / 2: disjoint from the first range
    count[1] = m.K;
    *drop_first = m.K + 1;
    *drop_count = m.n - 2 * m.K - 1;
    return m.K > 0 ? 2 : 1;
}

// Copies of one spectral field restricted to the kept box (kept ky x kept kx
// x kz < nkz, up to four strided copies; inside = true) or to its complement
// (up to seven; inside = false).  The box holds every mode that the dealias
// mask (solver.cu:36) keeps, and a step never writes outside it, so after a
// dealias the complement is zero for the rest of a run.
static cudaError_t copy_box(const gnss_ctx *c, void *dst, const void *src, bool inside, cudaMemcpyKind kind,
                            cudaStream_t s, size_t *bytes) {
    const Geom &g = c->g;
    int yf[2], yn[2], xf[2], xn[2], yd0, ydn, xd0, xdn;
    const int ny_r = keep_ranges(c->ky_keep, yf, yn, &yd0, &ydn);
    const int nx_r = keep_ranges(c->kx_keep, xf, xn, &xd0, &xdn);
    cudaError_t e = cudaSuccess;
    auto put = [&](cudaError_t r) { if (e == cudaSuccess) e = r; };
    if (!inside) put(copy_sub_box(c, dst, src, yd0, ydn, 0, g.nx, 0, g.nz2, kind, s, bytes));
    for (int a = 0; a < ny_r; ++a) {
        if (!inside) put(copy_sub_box(c, dst, src, yf[a], yn[a], xd0, xdn, 0, g.nz2, kind, s, bytes));
        for (int b = 0; b < nx_r; ++b) {
            if (inside) put(copy_sub_box(c, dst, src, yf[a], yn[a], xf[b], xn[b], 0, c->nkz, kind, s, bytes));
            else put(copy_sub_box(c, dst, src, yf[a], yn[a], xf[b], xn[b], c->nkz, g.nz2 - c->nkz, kind, s, bytes));
        }
    }
    return e;
}

gnss_status gnss_run_host_bytes(gnss_ctx *c, size_t *h2d, size_t *d2h) {
    if (!c || !h2d || !d2h) return GNSS_ERR_INVALID;
    const int nf = 3 + c->cfg.n_scalars;
    int yf[2], yn[2], xf[2], xn[2], d0, dn;
    const int ny_r = keep_ranges(c->ky_keep, yf, yn, &d0, &dn), nx_r = keep_ranges(c->kx_keep, xf, xn, &d0, &dn);
    size_t rows = 0;
    for (int a = 0; a < ny_r; ++a)
        for (int b = 0; b < nx_r; ++b) rows += (size_t)yn[a] * xn[b];
    *h2d = (size_t)nf * rows * (size_t)c->nkz * c->elem;
    *d2h = (size_t)nf * c->nspec * c->elem;
    return GNSS_OK;
}

// gnss_run_host after the upload: the download of the modes outside the
// kept box on the side stream (zero from the dealias to the end of the run,
// so it overlaps the steps; it writes parts of host_out that the upload does
// not read, and host_out may alias host_in), the steps with their statistics
// summed by the update, then the statistics and the kept box downloaded.
static gnss_status run_host_steps(gnss_ctx *c, const gnss_fields *st, const gnss_fields *hi, char *out, int n_steps,
                                  int first_euler, double *stats_out, cudaStream_t s) {
    const int nf = 3 + c->cfg.n_scalars;
    const size_t fb = c->nspec * c->elem;
    void *const sp[5] = {st->u, st->v, st->w, st->s, st->c};
    size_t moved = 0;
    CK(c, cudaEventRecord(c->side_ev[0], s));
    CK(c, cudaStreamWaitEvent(c->side, c->side_ev[0], 0));
    for (int q = 0; q < nf; ++q)
        CK(c, copy_box(c, out + (size_t)q * fb, sp[q], false, cudaMemcpyDeviceToHost, c->side, &moved));
    CK(c, cudaEventRecord(c->side_ev[1], c->side));
    for (int i = 0; i < n_steps; ++i) {
        const int euler = (i == 0 && first_euler) ? 1 : 0;
        double *dst = stats_out ? c->run_sums + (size_t)i * STAT_SUMS : nullptr;
        gnss_status r = PREC_CALL(c, step_t, c, st, hi, euler, s, dst);
        if (r) return r;
    }
    if (stats_out && n_steps > 0)
        CK(c, cudaMemcpyAsync(c->run_sums_host, c->run_sums, sizeof(double) * STAT_SUMS * (size_t)n_steps,
                              cudaMemcpyDeviceToHost, s));
    for (int q = 0; q < nf; ++q)
        CK(c, copy_box(c, out + (size_t)q * fb, sp[q], true, cudaMemcpyDeviceToHost, s, &moved));
    CK(c, cudaStreamWaitEvent(s, c->side_ev[1], 0));
    CK(c, cudaStreamSynchronize(s));
    return GNSS_OK;
}

gnss_status gnss_run_host(gnss_ctx *c, const void *host_in, void *host_out, int n_steps, int first_euler,
                          double *stats_out, void *stream) {
    if (!c || !host_in || !host_out || n_steps < 0) return fail(c, GNSS_ERR_INVALID, "bad argument");
    CK(c, cudaSetDevice(c->cfg.device));
    const int nf = 3 + c->cfg.n_scalars;
    const size_t fb = c->nspec * c->elem;
    if (!c->res) {
        if (cudaMalloc(&c->res, 2 * (size_t)nf * fb) != cudaSuccess) {
            cudaGetLastError();
            c->res = nullptr;
            return fail(c, GNSS_ERR_NOMEM, "cannot allocate resident state");
        }
        c->owned_bytes += 2 * (size_t)nf * fb;
    }
    if (stats_out && n_steps > c->run_sums_cap) {   // per-step sums, read back once after the last step
        if (c->run_sums) cudaFree(c->run_sums);
        if (c->run_sums_host) cudaFreeHost(c->run_sums_host);
        c->run_sums = nullptr;
        c->run_sums_host = nullptr;
        c->run_sums_cap = 0;
        const size_t b = sizeof(double) * STAT_SUMS * (size_t)n_steps;
        if (cudaMalloc(&c->run_sums, b) != cudaSuccess || cudaMallocHost(&c->run_sums_host, b) != cudaSuccess) {
            cudaGetLastError();
            return fail(c, GNSS_ERR_NOMEM, "cannot allocate statistics buffers");
        }
        c->run_sums_cap = n_steps;
    }
    if (!c->side) {
        if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&c->side_ev[0], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&c->side_ev[1], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return fail(c, GNSS_ERR_CUDA, "cannot create the copy stream");
        }
    }
    cudaStream_t s = S(stream);
    char *base = reinterpret_cast<char *>(c->res);
    char *out = static_cast<char *>(host_out);
    const char *in = static_cast<const char *>(host_in);
    gnss_fields st{}, hi{};
    void **sp[5] = {&st.u, &st.v, &st.w, &st.s, &st.c};
    void **hp[5] = {&hi.u, &hi.v, &hi.w, &hi.s, &hi.c};
    for (int q = 0; q < nf; ++q) {
        *sp[q] = base + (size_t)q * fb;
        *hp[q] = base + (size_t)(nf + q) * fb;
    }
    if (!al_fields(c, &st) || !al_fields(c, &hi)) return fail(c, GNSS_ERR_INVALID, "misaligned pointer");
    // The state zeroed, the kept box of each field uploaded and dealiased, as
    // the reference does before its loop (main.cu:156).  The history starts
    // at zero; the Euler step of CN/AB2 writes all of its kept box (the only
    // part ever read) and IF-RK3 keeps its own, so it is cleared only for a
    // CN/AB2 run that starts with AB2.
    const bool clear_hist = c->cfg.scheme == GNSS_SCHEME_CNAB2 && !first_euler;
    CK(c, cudaMemsetAsync(base, 0, (clear_hist ? 2 : 1) * (size_t)nf * fb, s));
    if (c->mean64)   // a new state: its FP64 mean line starts from the uploaded values
        CK(c, cudaMemsetAsync(c->mean64, 0, sizeof(double2) * 10 * (size_t)c->g.ny, s));
    size_t moved = 0;
    for (int q = 0; q < nf; ++q) {
        CK(c, copy_box(c, *sp[q], in + (size_t)q * fb, true, cudaMemcpyHostToDevice, s, &moved));
        gnss_status r = gnss_dealias(c, *sp[q], stream);
        if (r) return r;
    }
    gnss_status r = run_host_steps(c, &st, &hi, out, n_steps, first_euler, stats_out, s);
    cudaStreamSynchronize(c->side);   // no copy into host_out outlives the call, also after an error
    if (r) return r;
    gnss_status chk = gnss_check(c, stream);
    if (chk) return chk;
    if (stats_out)
        for (int i = 0; i < n_steps; ++i)
            stats_of_sums(c, c->run_sums_host + (size_t)i * STAT_SUMS, stats_out + (size_t)i * GNSS_NSTATS);
    return GNSS_OK;
}


// ============================================================== allocation-free forward transform
// For callers that may not allocate device memory at all: code running under
// a memory manager that owns every byte of the device (a framework's caching
// allocator, a fixed per-process budget) and latency-critical loops in which
// a cudaMalloc / cudaFree would synchronise the device.  gnss_forward_noalloc
// computes exactly what gnss_forward computes, but its twiddle tables and its
// one-field scratch live in the file-scope array below instead of in a
// context, and it never calls cudaMalloc, cudaFree or any allocating routine.
//
// Layout of the array: three twiddle tables of GNSS_NOALLOC_TW complex values
// (x, y, z), then GNSS_NOALLOC_MAX_ELEMS complex values of scratch.  Sizes are
// in double2 units, so the same storage serves FP32 (float2) with room to
// spare.  Every GPU that loads the library holds the array until the process
// exits.  All calls share it: it keeps the last call's contents (each call
// rewrites the twiddles it uses and overwrites the scratch it reads), and
// calls that overlap on the GPU, on any stream, race on it.
constexpr size_t GNSS_NOALLOC_TW = 512;
static __device__ __align__(256) double2 g_noalloc_pool[3 * GNSS_NOALLOC_TW + GNSS_NOALLOC_MAX_ELEMS];

// Host-side address of the array on each device, looked up once per device
// (the symbol itself is only a host stand-in, not a device address).
static void *g_noalloc_addr[64];
static bool g_noalloc_ready[64];
static std::mutex g_noalloc_mu;

static gnss_status noalloc_pool_address(int dev, void **out) {
    if (dev < 0 || dev >= 64) return GNSS_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ready[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_pool) != cudaSuccess) {
            cudaGetLastError();
            return GNSS_ERR_CUDA;
        }
        g_noalloc_addr[dev] = p;
        g_noalloc_ready[dev] = true;
    }
    *out = g_noalloc_addr[dev];
    return GNSS_OK;
}

// One twiddle table, passed by value in the launch's parameters (at most
// GNSS_NOALLOC_TW complex values: 8 KB in FP64) and written to its slot of the
// array by a small kernel, so no host buffer is copied and the values are the
// same long-double ones as a context's tables.
template <typename T> struct NoallocTable { V2<T> v[GNSS_NOALLOC_TW]; };
template <typename T> __global__ void k_noalloc_table(V2<T> *dst, int n, const __grid_constant__ NoallocTable<T> t) {
    for (int k = threadIdx.x; k < n; k += blockDim.x) dst[k] = t.v[k];
}

template <typename T> static cudaError_t noalloc_twiddles(V2<T> *dst, int n, cudaStream_t s) {
    NoallocTable<T> h;
    const long double twopi = 6.283185307179586476925286766559L;
    for (int k = 0; k < n; ++k) {
        long double a = twopi * (long double)k / (long double)n;
        h.v[k].x = (T)cosl(a);
        h.v[k].y = (T)(-sinl(a));
    }
    k_noalloc_table<T><<<1, 256, 0, s>>>(dst, n, h);
    return cudaGetLastError();
}

template <typename T> static gnss_status noalloc_forward_t(gnss_ctx *c, void *field, cudaStream_t s) {
    V2<T> *tw = reinterpret_cast<V2<T> *>(c->tw[0]);
    const int ns[3] = {c->cfg.nx, c->cfg.ny, c->cfg.nz};
    for (int a = 0; a < 3; ++a) {
        c->tw[a] = tw + (size_t)a * GNSS_NOALLOC_TW;
        CK(c, noalloc_twiddles<T>(reinterpret_cast<V2<T> *>(c->tw[a]), ns[a], s));
    }
    return forward_t<T>(c, field, s);
}

gnss_status gnss_forward_noalloc(const gnss_config *cfg, void *field, void *stream) {
    if (!cfg || !field) return GNSS_ERR_INVALID;
    const gnss_config &k = *cfg;
    if (!size_ok(k.nx) || !size_ok(k.ny) || !size_ok(k.nz)) return GNSS_ERR_INVALID;
    if (k.precision != GNSS_FP64 && k.precision != GNSS_FP32) return GNSS_ERR_INVALID;
    if (!(k.lx > 0 && k.ly > 0 && k.lz > 0)) return GNSS_ERR_INVALID;
    const size_t nspec = (size_t)k.nx * k.ny * (k.nz / 2 + 1);
    if (nspec > GNSS_NOALLOC_MAX_ELEMS) return GNSS_ERR_INVALID;   // beyond the static scratch
    const size_t elem = k.precision == GNSS_FP64 ? sizeof(double2) : sizeof(float2);
    if (reinterpret_cast<uintptr_t>(field) % elem) return GNSS_ERR_INVALID;
    if (cudaSetDevice(k.device) != cudaSuccess) {
        cudaGetLastError();
        return GNSS_ERR_CUDA;
    }
    void *pool = nullptr;
    gnss_status st = noalloc_pool_address(k.device, &pool);
    if (st) return st;
    // a context on the stack that points into the static array: no device
    // allocation happens below (ensure_scratch finds its one field present)
    gnss_ctx c;
    c.cfg = k;
    c.g.nx = k.nx; c.g.ny = k.ny; c.g.nz = k.nz; c.g.nz2 = k.nz / 2 + 1;
    c.g.dkx = 2 * M_PI / k.lx;
    c.g.dky = 2 * M_PI / k.ly;
    c.g.dkz = 2 * M_PI / k.lz;
    c.nspec = nspec;
    c.elem = elem;
    c.tw[0] = pool;
    c.scratch = reinterpret_cast<double2 *>(pool) + 3 * GNSS_NOALLOC_TW;
    c.nscratch = 1;
    if (cudaDeviceGetAttribute(&c.nsm, cudaDevAttrMultiProcessorCount, k.device) != cudaSuccess) {
        cudaGetLastError();
        std::fprintf(stderr, "gnss_forward_noalloc: cannot read the SM count of device %d\n", k.device);
        return GNSS_ERR_CUDA;
    }
    st = PREC_CALL(&c, noalloc_forward_t, &c, field, S(stream));
    // there is no context to keep the message in: print it
    if (st) std::fprintf(stderr, "gnss_forward_noalloc: %s\n", c.err.c_str());
    return st;
}
