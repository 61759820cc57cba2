// gnss_b200.cu -- host side of the B200 pseudospectral step: context,
// launch orchestration and the C ABI declared in include/gnss_b200.h.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "gnss_b200.h"
#include "kernels.cuh"

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
    double *stat_part = nullptr;                  // STAT_BLOCKS x STAT_SUMS
    double *stat_dev = nullptr;                   // STAT_SUMS
    double *stat_host = nullptr;                  // pinned STAT_SUMS
    void *res = nullptr;                          // resident state + history for gnss_run_host (2 * nf fields)
    size_t owned_bytes = 0;
    int nphys = 0, nnl = 0;                       // quantities in the physical pass, nonlinear outputs
    RecipeSet recipes{};
    std::string err;
    long long launches = 0;                       // kernels launched by this context
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
static inline int grid_for(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    long long cap = 148LL * 16;
    return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

// ============================================================== per-size launchers
template <typename T, int N> struct Launch {
    static cudaError_t strided(int sign, bool recipe, const FieldSet<T> &src, const FieldSet<T> &dst,
                               const Strides &st, int nouter, int nfields, const Geom &g, const RecipeSet &rs,
                               const void *tw, cudaStream_t s) {
        using C = StridedCfg<T, N>;
        dim3 grid((unsigned)(nouter * st.ncolblk), (unsigned)nfields);
        const V2<T> *t = reinterpret_cast<const V2<T> *>(tw);
        if (sign < 0) {
            if (recipe) return go(k_strided<T, N, -1, true>, grid, src, dst, st, g, rs, t, s);
            return go(k_strided<T, N, -1, false>, grid, src, dst, st, g, rs, t, s);
        }
        if (recipe) return go(k_strided<T, N, +1, true>, grid, src, dst, st, g, rs, t, s);
        return go(k_strided<T, N, +1, false>, grid, src, dst, st, g, rs, t, s);
    }
    template <class K>
    static cudaError_t go(K kern, dim3 grid, const FieldSet<T> &src, const FieldSet<T> &dst, const Strides &st,
                          const Geom &g, const RecipeSet &rs, const V2<T> *tw, cudaStream_t s) {
        using C = StridedCfg<T, N>;
        if (C::SMEM > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
            if (e != cudaSuccess) return e;
        }
        kern<<<grid, C::NT, C::SMEM, s>>>(src, dst, st, g, rs, tw);
        return cudaGetLastError();
    }
    static cudaError_t zpass(int dir, const FieldSet<T> &f, int nfields, long long nlines, int nz2, T scale,
                             const void *tw, cudaStream_t s) {
        using C = ZCfg<T, N>;
        long long npairs = (nlines + 1) / 2;
        dim3 grid((unsigned)((npairs + ZWARPS - 1) / ZWARPS), (unsigned)nfields);
        const V2<T> *t = reinterpret_cast<const V2<T> *>(tw);
        auto kern = dir < 0 ? k_zpass<T, N, -1> : k_zpass<T, N, +1>;
        if (C::SMEM > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
            if (e != cudaSuccess) return e;
        }
        kern<<<grid, ZWARPS * 32, C::SMEM, s>>>(f, nlines, nz2, scale, t);
        return cudaGetLastError();
    }
    static cudaError_t zphys(const FieldSet<T> &f, int nin, int nout, long long nlines, int nz2, T scale, T alpha,
                             const void *tw, cudaStream_t s) {
        const int smem = nin * ZPCfg<T, N>::LEN * (int)sizeof(V2<T>);
        auto kern = k_zphys<T, N>;
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (e != cudaSuccess) return e;
        }
        long long npairs = (nlines + 1) / 2;
        kern<<<(unsigned)npairs, nin * 32, smem, s>>>(f, nin, nout, nlines, nz2, scale, alpha,
                                                       reinterpret_cast<const V2<T> *>(tw));
        return cudaGetLastError();
    }
};

#define GNSS_SIZE_SWITCH(n, EXPR)                   \
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
        default: return cudaErrorInvalidValue;      \
    }

template <typename T>
static cudaError_t launch_strided(int n, int sign, bool recipe, const FieldSet<T> &src, const FieldSet<T> &dst,
                                  const Strides &st, int nouter, int nfields, const Geom &g, const RecipeSet &rs,
                                  const void *tw, cudaStream_t s) {
    GNSS_SIZE_SWITCH(n, return (Launch<T, NN_>::strided(sign, recipe, src, dst, st, nouter, nfields, g, rs, tw, s)));
}
template <typename T>
static cudaError_t launch_zpass(int n, int dir, const FieldSet<T> &f, int nfields, long long nlines, int nz2, T scale,
                                const void *tw, cudaStream_t s) {
    GNSS_SIZE_SWITCH(n, return (Launch<T, NN_>::zpass(dir, f, nfields, nlines, nz2, scale, tw, s)));
}
template <typename T>
static cudaError_t launch_zphys(int n, const FieldSet<T> &f, int nin, int nout, long long nlines, int nz2, T scale,
                                T alpha, const void *tw, cudaStream_t s) {
    GNSS_SIZE_SWITCH(n, return (Launch<T, NN_>::zphys(f, nin, nout, nlines, nz2, scale, alpha, tw, s)));
}

template <typename T> static int nb_for(int n) {
    switch (n) {
        case 8: return StridedCfg<T, 8>::NB; case 12: return StridedCfg<T, 12>::NB;
        case 16: return StridedCfg<T, 16>::NB; case 24: return StridedCfg<T, 24>::NB;
        case 32: return StridedCfg<T, 32>::NB; case 48: return StridedCfg<T, 48>::NB;
        case 64: return StridedCfg<T, 64>::NB; case 96: return StridedCfg<T, 96>::NB;
        case 128: return StridedCfg<T, 128>::NB; case 192: return StridedCfg<T, 192>::NB;
        case 256: return StridedCfg<T, 256>::NB; case 384: return StridedCfg<T, 384>::NB;
        default: return StridedCfg<T, 512>::NB;
    }
}

// ============================================================== helpers
template <typename T> static V2<T> *fld(void *base, size_t nspec, int i) {
    return reinterpret_cast<V2<T> *>(base) + nspec * (size_t)i;
}

static gnss_status ensure_scratch(gnss_ctx *c, int nfields) {
    if (c->nscratch >= nfields) return GNSS_OK;
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

// Strides of the x pass from the spectral layout [y][x][kz] to [x][y][kz]
// (inverse) and back (forward), and of the y pass on [x][y][kz].
static Strides x_inv_strides(const gnss_ctx *c, int nb) {
    const Geom &g = c->g;
    Strides s;
    s.s_row = g.nz2; s.s_out = (long long)g.nx * g.nz2;
    s.d_row = (long long)g.ny * g.nz2; s.d_out = g.nz2;
    s.ncols = g.nz2; s.ncolblk = (g.nz2 + nb - 1) / nb;
    return s;
}
static Strides x_fwd_strides(const gnss_ctx *c, int nb) {
    const Geom &g = c->g;
    Strides s;
    s.s_row = (long long)g.ny * g.nz2; s.s_out = g.nz2;
    s.d_row = g.nz2; s.d_out = (long long)g.nx * g.nz2;
    s.ncols = g.nz2; s.ncolblk = (g.nz2 + nb - 1) / nb;
    return s;
}
static Strides y_strides(const gnss_ctx *c, int nb) {
    const Geom &g = c->g;
    Strides s;
    s.s_row = g.nz2; s.s_out = (long long)g.ny * g.nz2;
    s.d_row = g.nz2; s.d_out = (long long)g.ny * g.nz2;
    s.ncols = g.nz2; s.ncolblk = (g.nz2 + nb - 1) / nb;
    return s;
}

// ============================================================== transforms
template <typename T> static gnss_status forward_t(gnss_ctx *c, void *f, cudaStream_t s) {
    gnss_status st = ensure_scratch(c, 1);
    if (st) return st;
    const Geom &g = c->g;
    FieldSet<T> F{}, X{};
    F.p[0] = reinterpret_cast<V2<T> *>(f);
    X.p[0] = fld<T>(c->scratch, c->nspec, 0);
    RecipeSet none{};
    const long long nlines = (long long)g.nx * g.ny;
    c->launches += 3;
    CK(c, launch_zpass<T>(g.nz, -1, F, 1, nlines, g.nz2, T(1), c->tw[2], s));
    CK(c, launch_strided<T>(g.ny, -1, false, F, X, y_strides(c, nb_for<T>(g.ny)), g.nx, 1, g, none, c->tw[1], s));
    CK(c, launch_strided<T>(g.nx, -1, false, X, F, x_fwd_strides(c, nb_for<T>(g.nx)), g.ny, 1, g, none, c->tw[0], s));
    return GNSS_OK;
}

template <typename T> static gnss_status inverse_t(gnss_ctx *c, void *f, cudaStream_t s) {
    gnss_status st = ensure_scratch(c, 1);
    if (st) return st;
    const Geom &g = c->g;
    FieldSet<T> F{}, X{};
    F.p[0] = reinterpret_cast<V2<T> *>(f);
    X.p[0] = fld<T>(c->scratch, c->nspec, 0);
    RecipeSet none{};
    const long long nlines = (long long)g.nx * g.ny;
    const T scale = (T)(1.0 / ((double)g.nx * g.ny * g.nz));
    c->launches += 3;
    CK(c, launch_strided<T>(g.nx, +1, false, F, X, x_inv_strides(c, nb_for<T>(g.nx)), g.ny, 1, g, none, c->tw[0], s));
    CK(c, launch_strided<T>(g.ny, +1, false, X, F, y_strides(c, nb_for<T>(g.ny)), g.nx, 1, g, none, c->tw[1], s));
    CK(c, launch_zpass<T>(g.nz, +1, F, 1, nlines, g.nz2, scale, c->tw[2], s));
    return GNSS_OK;
}

// ============================================================== fused step
// One evaluation of the nonlinear term followed by the spectral update.
//   1 x inverse of the dealiased state, forming u, omega, grad s (, grad c, c, lap s)
//   2 y inverse of those quantities
//   3 z C2R + products + z R2C  (physical space stays on chip)
//   4 y forward of the products
//   5 x forward of the products into spectral layout
//   6 projection, dealias and time update
template <typename T>
static gnss_status nonlinear_and_update(gnss_ctx *c, const gnss_fields *state, void *hist_base, const gnss_fields *hist,
                                        const UpdCoef &uc, cudaStream_t s) {
    const Geom &g = c->g;
    const int nphys = c->nphys, nnl = c->nnl;
    gnss_status st = ensure_scratch(c, nphys);
    if (st) return st;
    FieldSet<T> SF{}, P{}, NLs{}, NLx{}, H{};
    void *sp[5] = {state->u, state->v, state->w, state->s, state->c};
    for (int q = 0; q < 5; ++q) SF.p[q] = reinterpret_cast<V2<T> *>(sp[q]);
    for (int q = 0; q < nphys; ++q) P.p[q] = fld<T>(c->scratch, c->nspec, q);
    for (int q = 0; q < nnl; ++q) {
        NLs.p[q] = P.p[q];
        NLx.p[q] = P.p[nnl + q];
    }
    if (hist) {
        void *hp[5] = {hist->u, hist->v, hist->w, hist->s, hist->c};
        for (int q = 0; q < 5; ++q) H.p[q] = reinterpret_cast<V2<T> *>(hp[q]);
    } else {
        for (int q = 0; q < 5; ++q) H.p[q] = fld<T>(hist_base, c->nspec, q);
    }
    RecipeSet none{};
    const long long nlines = (long long)g.nx * g.ny;
    const T scale = (T)(1.0 / ((double)g.nx * g.ny * g.nz));
    {
        StageTimer t(c, s, 0);
        CK(c, launch_strided<T>(g.nx, +1, true, SF, P, x_inv_strides(c, nb_for<T>(g.nx)), g.ny, nphys, g,
                                c->recipes, c->tw[0], s));
    }
    {
        StageTimer t(c, s, 1);
        CK(c, launch_strided<T>(g.ny, +1, false, P, P, y_strides(c, nb_for<T>(g.ny)), g.nx, nphys, g, none,
                                c->tw[1], s));
    }
    {
        StageTimer t(c, s, 2);
        CK(c, launch_zphys<T>(g.nz, P, nphys, nnl, nlines, g.nz2, scale, (T)c->cfg.alpha, c->tw[2], s));
    }
    {
        StageTimer t(c, s, 3);
        CK(c, launch_strided<T>(g.ny, -1, false, NLs, NLs, y_strides(c, nb_for<T>(g.ny)), g.nx, nnl, g, none,
                                c->tw[1], s));
    }
    {
        StageTimer t(c, s, 4);
        CK(c, launch_strided<T>(g.nx, -1, false, NLs, NLx, x_fwd_strides(c, nb_for<T>(g.nx)), g.ny, nnl, g, none,
                                c->tw[0], s));
    }
    {
        StageTimer t(c, s, 5);
        k_update<T><<<grid_for((long long)c->nspec, 256), 256, 0, s>>>(SF, H, NLx, g, uc);
        LAUNCH_CK(c);
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
        u.num[q] = num[q];
        u.nu[q] = 1.0 / num[q];
    }
    return u;
}

template <typename T>
static gnss_status step_t(gnss_ctx *c, const gnss_fields *state, const gnss_fields *hist, int euler, cudaStream_t s) {
    UpdCoef uc = base_coef(c);
    if (c->cfg.scheme == GNSS_SCHEME_CNAB2) {
        uc.euler = euler ? 1 : 0;
        return nonlinear_and_update<T>(c, state, nullptr, hist, uc, s);
    }
    // IF-RK3: the history lives in context scratch after the step's quantities
    const int nf = 3 + c->cfg.n_scalars;
    gnss_status st = ensure_scratch(c, c->nphys + nf);
    if (st) return st;
    void *hb = fld<T>(c->scratch, c->nspec, c->nphys);
    const double gam[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
    const double zet[4] = {0.0, -17.0 / 60.0, -5.0 / 12.0, 0.0};
    for (int k = 0; k < 3; ++k) {
        uc.substep = k;
        uc.gam = gam[k];
        uc.zet_next = zet[k + 1];
        uc.alph = gam[k] + zet[k];
        st = nonlinear_and_update<T>(c, state, hb, nullptr, uc, s);
        if (st) return st;
    }
    return GNSS_OK;
}

// ============================================================== statistics
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
    const gnss_config &k = c->cfg;
    const double nn = (double)k.nx * k.ny * k.nz;
    const double n2 = nn * nn;
    const double *h = c->stat_host;
    out[GNSS_STAT_KE] = (h[0] / n2) / 2.0;
    out[GNSS_STAT_VRMS2] = (h[0] / n2) / 3.0;
    out[GNSS_STAT_EPS] = k.nu_stats * (h[1] / n2);
    out[GNSS_STAT_CHI_S] = 2.0 * (k.nu_stats / k.sc) * (h[2] / n2);
    out[GNSS_STAT_CHI_C] = 2.0 * (k.nu_stats / k.sc_c) * (h[3] / n2);
    out[GNSS_STAT_VAR_S] = h[4] / n2;
    out[GNSS_STAT_VAR_C] = h[5] / n2;
    return GNSS_OK;
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
        default: return "unknown status";
    }
}

const char *gnss_last_error(const gnss_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

long long gnss_launch_count(const gnss_ctx *ctx) { return ctx ? ctx->launches : -1; }

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
size_t gnss_workspace_bytes(const gnss_ctx *ctx) { return ctx ? ctx->owned_bytes : 0; }

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

static void set_recipes(gnss_ctx *c) {
    // state fields: 0 u, 1 v, 2 w, 3 s, 4 c
    auto R = [](int f0, int m0, int s0, int f1 = -1, int m1 = 0, int s1 = 1) {
        Recipe r{};
        r.f[0] = (signed char)f0; r.m[0] = (signed char)m0; r.s[0] = (signed char)s0;
        r.f[1] = (signed char)f1; r.m[1] = (signed char)m1; r.s[1] = (signed char)s1;
        return r;
    };
    RecipeSet &rs = c->recipes;
    int n = 0;
    rs.r[n++] = R(0, M_ONE, 1);                  // u
    rs.r[n++] = R(1, M_ONE, 1);                  // v
    rs.r[n++] = R(2, M_ONE, 1);                  // w
    rs.r[n++] = R(2, M_IKY, 1, 1, M_IKZ, -1);    // omega_1 = i k2 w - i k3 v   (solver.cu:68-81)
    rs.r[n++] = R(0, M_IKZ, 1, 2, M_IKX, -1);    // omega_2 = i k3 u - i k1 w   (solver.cu:84-97)
    rs.r[n++] = R(1, M_IKX, 1, 0, M_IKY, -1);    // omega_3 = i k1 v - i k2 u   (solver.cu:100-113)
    rs.r[n++] = R(3, M_IKX, 1);                  // ds/dx  (gradientKernel_mgpu, solver.cu:233-256)
    rs.r[n++] = R(3, M_IKY, 1);
    rs.r[n++] = R(3, M_IKZ, 1);
    c->nnl = 4;
    if (c->cfg.n_scalars > 1) {
        rs.r[n++] = R(4, M_IKX, 1);              // grad c (solver.cu:444)
        rs.r[n++] = R(4, M_IKY, 1);
        rs.r[n++] = R(4, M_IKZ, 1);
        c->nnl = 5;
        if (c->cfg.alpha != 0.0) {
            rs.r[n++] = R(4, M_ONE, 1);          // c itself (solver.cu:451)
            rs.r[n++] = R(3, M_LAP, 1);          // lap s = div grad s (solver.cu:425)
        }
    }
    c->nphys = n;
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
    *out = c;
    return GNSS_OK;
}

gnss_status gnss_destroy(gnss_ctx *c) {
    if (!c) return GNSS_ERR_INVALID;
    cudaSetDevice(c->cfg.device);
    for (int a = 0; a < 3; ++a) if (c->tw[a]) cudaFree(c->tw[a]);
    if (c->scratch) cudaFree(c->scratch);
    if (c->stat_part) cudaFree(c->stat_part);
    if (c->stat_dev) cudaFree(c->stat_dev);
    if (c->stat_host) cudaFreeHost(c->stat_host);
    if (c->res) cudaFree(c->res);
    for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
    delete c;
    return GNSS_OK;
}

#define PREC_CALL(c, fn, ...) ((c)->cfg.precision == GNSS_FP64 ? fn<double>(__VA_ARGS__) : fn<float>(__VA_ARGS__))

gnss_status gnss_forward(gnss_ctx *c, void *f, void *stream) {
    if (!c || !f) return fail(c, GNSS_ERR_INVALID, "null argument");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, forward_t, c, f, S(stream));
}

gnss_status gnss_inverse(gnss_ctx *c, void *f, void *stream) {
    if (!c || !f) return fail(c, GNSS_ERR_INVALID, "null argument");
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
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, rhs_t, c, ru, rv, rw, rs, rc, S(stream));
}

template <typename T>
static gnss_status timestep_t(gnss_ctx *c, int euler, const gnss_fields *st, const gnss_fields *r,
                              const gnss_fields *ro, cudaStream_t s) {
    using V = V2<T>;
    UpdCoef u = base_coef(c);
    void *f[5] = {st->u, st->v, st->w, st->s, st->c};
    void *rr[5] = {r->u, r->v, r->w, r->s, r->c};
    void *oo[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    if (ro) { oo[0] = ro->u; oo[1] = ro->v; oo[2] = ro->w; oo[3] = ro->s; oo[4] = ro->c; }
    for (int q = 0; q < 5; ++q) {
        if (!f[q]) continue;
        if (!rr[q] || (!euler && !oo[q])) return fail(c, GNSS_ERR_INVALID, "missing rhs field %d", q);
        c->launches++;
        k_timestep<T><<<grid_for((long long)c->nspec, 256), 256, 0, s>>>((V *)f[q], (const V *)rr[q],
                                                                          (const V *)oo[q], u.num[q], u.dt, euler,
                                                                          c->g);
        LAUNCH_CK(c);
    }
    return GNSS_OK;
}
gnss_status gnss_timestep(gnss_ctx *c, int euler, const gnss_fields *state, const gnss_fields *rhs,
                          const gnss_fields *rhs_old, void *stream) {
    if (!c || !state || !rhs || (!euler && !rhs_old)) return fail(c, GNSS_ERR_INVALID, "null argument");
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
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, colloid_t, c, u, v, w, cc, cx, cy, cz, sx, sy, sz, lap_s_inout, S(stream));
}

static bool state_ok(const gnss_ctx *c, const gnss_fields *st) {
    if (!st || !st->u || !st->v || !st->w || !st->s) return false;
    if (c->cfg.n_scalars > 1 && !st->c) return false;
    return true;
}

gnss_status gnss_step(gnss_ctx *c, const gnss_fields *state, const gnss_fields *hist, int euler, void *stream) {
    if (!c) return GNSS_ERR_INVALID;
    if (!state_ok(c, state)) return fail(c, GNSS_ERR_INVALID, "state fields missing");
    if (c->cfg.scheme == GNSS_SCHEME_CNAB2 && !state_ok(c, hist))
        return fail(c, GNSS_ERR_INVALID, "history fields missing");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, step_t, c, state, hist, euler, S(stream));
}

gnss_status gnss_stats(gnss_ctx *c, const gnss_fields *state, double *out, void *stream) {
    if (!c || !out) return fail(c, GNSS_ERR_INVALID, "null argument");
    if (!state || !state->u || !state->v || !state->w) return fail(c, GNSS_ERR_INVALID, "state fields missing");
    CK(c, cudaSetDevice(c->cfg.device));
    return PREC_CALL(c, stats_t, c, state, out, S(stream));
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
    cudaStream_t s = S(stream);
    char *base = reinterpret_cast<char *>(c->res);
    gnss_fields st{}, hi{};
    void **sp[5] = {&st.u, &st.v, &st.w, &st.s, &st.c};
    void **hp[5] = {&hi.u, &hi.v, &hi.w, &hi.s, &hi.c};
    for (int q = 0; q < nf; ++q) {
        *sp[q] = base + (size_t)q * fb;
        *hp[q] = base + (size_t)(nf + q) * fb;
    }
    CK(c, cudaMemcpyAsync(base, host_in, (size_t)nf * fb, cudaMemcpyHostToDevice, s));
    CK(c, cudaMemsetAsync(base + (size_t)nf * fb, 0, (size_t)nf * fb, s));
    for (int i = 0; i < n_steps; ++i) {
        gnss_status r = gnss_step(c, &st, &hi, (i == 0 && first_euler) ? 1 : 0, stream);
        if (r) return r;
        if (stats_out) {
            r = gnss_stats(c, &st, stats_out + (size_t)i * GNSS_NSTATS, stream);
            if (r) return r;
        }
    }
    CK(c, cudaMemcpyAsync(host_out, base, (size_t)nf * fb, cudaMemcpyDeviceToHost, s));
    CK(c, cudaStreamSynchronize(s));
    return GNSS_OK;
}

