/*
 * oracle.cpp -- CPU FP64 restatement of the reference pseudospectral time step.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h): the checker for the CUDA path and
 * the timed CPU baseline.  Nothing in the product path links or loads it.
 *
 * Every routine cites the reference file:line whose behaviour it restates.
 * The FFT is this project's own mixed-radix Stockham FFT (radix 4, 2, 3) on a
 * [n][batch] interleaved layout, FP64 throughout, with twiddles computed in
 * long double.
 */
#include "oracle.h"

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <map>
#include <mutex>
#include <omp.h>

namespace {

struct cpx { double re, im; };

static inline cpx cmul(cpx a, cpx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

/* ---------------------------------------------------------------- FFT plan */
struct Plan {
    int n;
    std::vector<int> radix;
    std::vector<cpx> wf, wi;   /* exp(-2 pi i k/n), exp(+2 pi i k/n), k < n */
};

static bool factor(int n, std::vector<int> &r) {
    r.clear();
    while (n % 4 == 0) { r.push_back(4); n /= 4; }
    while (n % 2 == 0) { r.push_back(2); n /= 2; }
    while (n % 3 == 0) { r.push_back(3); n /= 3; }
    return n == 1;
}

static std::mutex g_plan_mu;
static std::map<int, Plan *> g_plans;

static const Plan *get_plan(int n) {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    auto it = g_plans.find(n);
    if (it != g_plans.end()) return it->second;
    Plan *p = new Plan;
    p->n = n;
    if (!factor(n, p->radix)) { delete p; return nullptr; }
    p->wf.resize(n); p->wi.resize(n);
    const long double twopi = 6.283185307179586476925286766559L;
    for (int k = 0; k < n; ++k) {
        long double a = twopi * (long double)k / (long double)n;
        double c = (double)cosl(a), s = (double)sinl(a);
        p->wf[k] = {c, -s};
        p->wi[k] = {c, s};
    }
    g_plans[n] = p;
    return p;
}

/* Stockham autosort FFT on x[n][B] (B interleaved independent lines).
 * Stage with radix R and span Ns: butterfly j reads x[j + r*n/R], applies the
 * twiddle w^(r*(j%Ns)*n/(Ns*R)), does a length-R DFT and writes
 * y[(j/Ns)*Ns*R + j%Ns + r*Ns]. sign < 0: forward (exp(-i..)). Result in x. */
static void stockham(const Plan *p, cpx *x, cpx *y, int B, int sign) {
    const int n = p->n;
    const cpx *w = sign < 0 ? p->wf.data() : p->wi.data();
    const double sg = sign < 0 ? -1.0 : 1.0;
    cpx *in = x, *out = y;
    int Ns = 1;
    for (int R : p->radix) {
        const int m = n / R;
        const int tstep = n / (Ns * R);
        for (int j = 0; j < m; ++j) {
            const int k = j % Ns;
            const int idxD = (j / Ns) * Ns * R + k;
            cpx t1 = w[(1 * k * tstep) % n], t2 = w[(2 * k * tstep) % n], t3 = w[(3 * k * tstep) % n];
            const cpx *a0 = in + (size_t)(j) * B;
            const cpx *a1 = in + (size_t)(j + m) * B;
            cpx *o0 = out + (size_t)(idxD) * B;
            cpx *o1 = out + (size_t)(idxD + Ns) * B;
            if (R == 2) {
                for (int b = 0; b < B; ++b) {
                    cpx v0 = a0[b], v1 = cmul(a1[b], t1);
                    o0[b] = {v0.re + v1.re, v0.im + v1.im};
                    o1[b] = {v0.re - v1.re, v0.im - v1.im};
                }
            } else if (R == 4) {
                const cpx *a2 = in + (size_t)(j + 2 * m) * B;
                const cpx *a3 = in + (size_t)(j + 3 * m) * B;
                cpx *o2 = out + (size_t)(idxD + 2 * Ns) * B;
                cpx *o3 = out + (size_t)(idxD + 3 * Ns) * B;
                for (int b = 0; b < B; ++b) {
                    cpx v0 = a0[b], v1 = cmul(a1[b], t1), v2 = cmul(a2[b], t2), v3 = cmul(a3[b], t3);
                    cpx s02 = {v0.re + v2.re, v0.im + v2.im}, d02 = {v0.re - v2.re, v0.im - v2.im};
                    cpx s13 = {v1.re + v3.re, v1.im + v3.im}, d13 = {v1.re - v3.re, v1.im - v3.im};
                    /* d13 * (sg * i) */
                    cpx jd = {-sg * d13.im, sg * d13.re};
                    o0[b] = {s02.re + s13.re, s02.im + s13.im};
                    o2[b] = {s02.re - s13.re, s02.im - s13.im};
                    o1[b] = {d02.re + jd.re, d02.im + jd.im};
                    o3[b] = {d02.re - jd.re, d02.im - jd.im};
                }
            } else { /* R == 3 */
                const cpx *a2 = in + (size_t)(j + 2 * m) * B;
                cpx *o2 = out + (size_t)(idxD + 2 * Ns) * B;
                const double c3 = -0.5, s3 = sg * 0.86602540378443864676;
                for (int b = 0; b < B; ++b) {
                    cpx v0 = a0[b], v1 = cmul(a1[b], t1), v2 = cmul(a2[b], t2);
                    cpx s = {v1.re + v2.re, v1.im + v2.im}, d = {v1.re - v2.re, v1.im - v2.im};
                    cpx m0 = {v0.re + c3 * s.re, v0.im + c3 * s.im};
                    /* i*s3*d */
                    cpx jd = {-s3 * d.im, s3 * d.re};
                    o0[b] = {v0.re + s.re, v0.im + s.im};
                    o1[b] = {m0.re + jd.re, m0.im + jd.im};
                    o2[b] = {m0.re - jd.re, m0.im - jd.im};
                }
            }
        }
        Ns *= R;
        cpx *t = in; in = out; out = t;
    }
    if (in != x) std::memcpy(x, in, sizeof(cpx) * (size_t)n * B);
}

static const int BL = 8; /* lines per batch */

static inline int nthreads_of(const orc_cfg *c) { return c->nthreads > 0 ? c->nthreads : omp_get_max_threads(); }

/* -------------------------------------------------- 3D transform passes */
/* z pass, forward R2C on every (x,y) line of the padded physical layout.
 * Two real lines (a,b) are packed as a+ib, transformed together, and split:
 * A_k = (Z_k + conj Z_{n-k})/2, B_k = (Z_k - conj Z_{n-k})/(2i).            */
static void zpass_r2c(const orc_cfg *c, double *f) {
    const int nx = c->nx, ny = c->ny, nz = c->nz, nz2 = nz / 2 + 1;
    const Plan *p = get_plan(nz);
    const long nlines = (long)nx * ny;
    const long npairs = (nlines + 1) / 2;
#pragma omp parallel num_threads(nthreads_of(c))
    {
        std::vector<cpx> X((size_t)nz * BL), Y((size_t)nz * BL);
#pragma omp for schedule(static)
        for (long pb = 0; pb < (npairs + BL - 1) / BL; ++pb) {
            long p0 = pb * BL;
            int nb = (int)std::min<long>(BL, npairs - p0);
            for (int b = 0; b < BL; ++b) {
                long la = 2 * (p0 + b), lb = la + 1;
                for (int z = 0; z < nz; ++z) {
                    double a = (b < nb && la < nlines) ? f[(size_t)la * 2 * nz2 + z] : 0.0;
                    double bb = (b < nb && lb < nlines) ? f[(size_t)lb * 2 * nz2 + z] : 0.0;
                    X[(size_t)z * BL + b] = {a, bb};
                }
            }
            stockham(p, X.data(), Y.data(), BL, -1);
            for (int b = 0; b < nb; ++b) {
                long la = 2 * (p0 + b), lb = la + 1;
                for (int k = 0; k < nz2; ++k) {
                    cpx zk = X[(size_t)k * BL + b];
                    cpx zm = X[(size_t)((nz - k) % nz) * BL + b];
                    cpx A = {0.5 * (zk.re + zm.re), 0.5 * (zk.im - zm.im)};
                    cpx Bv = {0.5 * (zk.im + zm.im), -0.5 * (zk.re - zm.re)};
                    f[(size_t)la * 2 * nz2 + 2 * k] = A.re;
                    f[(size_t)la * 2 * nz2 + 2 * k + 1] = A.im;
                    if (lb < nlines) {
                        f[(size_t)lb * 2 * nz2 + 2 * k] = Bv.re;
                        f[(size_t)lb * 2 * nz2 + 2 * k + 1] = Bv.im;
                    }
                }
            }
        }
    }
}

/* z pass, inverse C2R.  The imaginary parts of the kz=0 and kz=nz/2 entries are
 * ignored (the standard C2R convention); output scaled by `scale`.            */
static void zpass_c2r(const orc_cfg *c, double *f, double scale) {
    const int nx = c->nx, ny = c->ny, nz = c->nz, nz2 = nz / 2 + 1;
    const Plan *p = get_plan(nz);
    const long nlines = (long)nx * ny;
    const long npairs = (nlines + 1) / 2;
#pragma omp parallel num_threads(nthreads_of(c))
    {
        std::vector<cpx> X((size_t)nz * BL), Y((size_t)nz * BL);
#pragma omp for schedule(static)
        for (long pb = 0; pb < (npairs + BL - 1) / BL; ++pb) {
            long p0 = pb * BL;
            int nb = (int)std::min<long>(BL, npairs - p0);
            for (int b = 0; b < BL; ++b) {
                long la = 2 * (p0 + b), lb = la + 1;
                bool va = b < nb && la < nlines, vb = b < nb && lb < nlines;
                for (int k = 0; k < nz2; ++k) {
                    cpx A = va ? cpx{f[(size_t)la * 2 * nz2 + 2 * k], f[(size_t)la * 2 * nz2 + 2 * k + 1]} : cpx{0, 0};
                    cpx Bv = vb ? cpx{f[(size_t)lb * 2 * nz2 + 2 * k], f[(size_t)lb * 2 * nz2 + 2 * k + 1]} : cpx{0, 0};
                    if (k == 0 || 2 * k == nz) { A.im = 0.0; Bv.im = 0.0; }
                    /* Z_k = A_k + i B_k ; Z_{n-k} = conj(A_k) + i conj(B_k) */
                    X[(size_t)k * BL + b] = {A.re - Bv.im, A.im + Bv.re};
                    if (k > 0 && 2 * k < nz)
                        X[(size_t)(nz - k) * BL + b] = {A.re + Bv.im, -A.im + Bv.re};
                }
            }
            stockham(p, X.data(), Y.data(), BL, +1);
            for (int b = 0; b < nb; ++b) {
                long la = 2 * (p0 + b), lb = la + 1;
                for (int z = 0; z < nz; ++z) {
                    cpx v = X[(size_t)z * BL + b];
                    f[(size_t)la * 2 * nz2 + z] = v.re * scale;
                    if (lb < nlines) f[(size_t)lb * 2 * nz2 + z] = v.im * scale;
                }
                /* the two padding doubles of each line are left as zero */
                f[(size_t)la * 2 * nz2 + nz] = 0.0; f[(size_t)la * 2 * nz2 + nz + 1] = 0.0;
                if (lb < nlines) { f[(size_t)lb * 2 * nz2 + nz] = 0.0; f[(size_t)lb * 2 * nz2 + nz + 1] = 0.0; }
            }
        }
    }
}

/* Strided C2C pass over a complex field viewed as [outer][n][inner]; with
 * `transpose` the result is written as [n][outer][inner] into `dst`.        */
static void strided_pass(const orc_cfg *c, const cpx *src, cpx *dst, int outer, int n, int inner,
                         int sign, bool transpose) {
    const Plan *p = get_plan(n);
    const int nblk = (inner + BL - 1) / BL;
#pragma omp parallel num_threads(nthreads_of(c))
    {
        std::vector<cpx> X((size_t)n * BL), Y((size_t)n * BL);
#pragma omp for schedule(static)
        for (long t = 0; t < (long)outer * nblk; ++t) {
            int o = (int)(t / nblk), k0 = (int)(t % nblk) * BL;
            int nb = std::min(BL, inner - k0);
            for (int l = 0; l < n; ++l)
                for (int b = 0; b < BL; ++b)
                    X[(size_t)l * BL + b] = b < nb ? src[((size_t)o * n + l) * inner + k0 + b] : cpx{0, 0};
            stockham(p, X.data(), Y.data(), BL, sign);
            for (int l = 0; l < n; ++l)
                for (int b = 0; b < nb; ++b) {
                    size_t di = transpose ? ((size_t)l * outer + o) * inner + k0 + b
                                          : ((size_t)o * n + l) * inner + k0 + b;
                    dst[di] = X[(size_t)l * BL + b];
                }
        }
    }
}

/* wavenumbers (initialize.cu:678-691): k_i = 2pi/L * i for i < n/2, else 2pi/L*(i-n) */
static std::vector<double> wavenumbers(int n, double l) {
    std::vector<double> k(n);
    for (int i = 0; i < n; ++i) k[i] = (i < n / 2) ? (2 * M_PI / l) * (double)i : (2 * M_PI / l) * ((double)i - n);
    return k;
}

struct Grid {
    int nx, ny, nz, nz2;
    std::vector<double> kx, ky, kz;
    double kmax2;
    explicit Grid(const orc_cfg *c)
        : nx(c->nx), ny(c->ny), nz(c->nz), nz2(c->nz / 2 + 1),
          kx(wavenumbers(c->nx, c->lx)), ky(wavenumbers(c->ny, c->ly)), kz(wavenumbers(c->nz, c->lz)) {
        double kxm = c->nx * M_PI / c->lx;           /* solver.cu:29 */
        double km = c->alias_filter * kxm;           /* solver.cu:31 */
        kmax2 = km * km;
    }
    size_t nspec() const { return (size_t)nx * ny * nz2; }
};

static int valid(const orc_cfg *c) {
    std::vector<int> r;
    if (!c || c->nx < 2 || c->ny < 2 || c->nz < 2) return 0;
    if ((c->nx | c->ny | c->nz) & 1) return 0;
    return factor(c->nx, r) && factor(c->ny, r) && factor(c->nz, r);
}

} /* namespace */

/* ======================================================================= API */
extern "C" {

int orc_fft_c2c(int n, int batch, double *data, int sign) {
    const Plan *p = get_plan(n);
    if (!p || batch < 1) return 1;
    std::vector<cpx> Y((size_t)n * batch);
    stockham(p, reinterpret_cast<cpx *>(data), Y.data(), batch, sign);
    return 0;
}

int orc_forward(const orc_cfg *c, double *f) {
    if (!valid(c)) return 1;
    const int nx = c->nx, ny = c->ny, nz2 = c->nz / 2 + 1;
    std::vector<cpx> tmp((size_t)nx * ny * nz2);
    zpass_r2c(c, f);
    cpx *F = reinterpret_cast<cpx *>(f);
    /* y pass on [x][y][kz] */
    strided_pass(c, F, F, nx, ny, nz2, -1, false);
    /* x pass: view as [1][x][y*nz2]... the x lines have stride ny*nz2; write transposed [y][x][kz] */
    /* treat [x][ (y,kz) ] as outer=1, n=nx, inner=ny*nz2, then transposed output [y][x][kz]
       needs a per-y split, so run per y below */
#pragma omp parallel for num_threads(nthreads_of(c)) schedule(static)
    for (int y = 0; y < ny; ++y) {
        std::vector<cpx> X((size_t)nx * BL), Y((size_t)nx * BL);
        const Plan *p = get_plan(nx);
        for (int k0 = 0; k0 < nz2; k0 += BL) {
            int nb = std::min(BL, nz2 - k0);
            for (int x = 0; x < nx; ++x)
                for (int b = 0; b < BL; ++b)
                    X[(size_t)x * BL + b] = b < nb ? F[((size_t)x * ny + y) * nz2 + k0 + b] : cpx{0, 0};
            stockham(p, X.data(), Y.data(), BL, -1);
            for (int x = 0; x < nx; ++x)
                for (int b = 0; b < nb; ++b)
                    tmp[((size_t)y * nx + x) * nz2 + k0 + b] = X[(size_t)x * BL + b];
        }
    }
    std::memcpy(F, tmp.data(), sizeof(cpx) * tmp.size());
    return 0;
}

int orc_inverse(const orc_cfg *c, double *f) {
    if (!valid(c)) return 1;
    const int nx = c->nx, ny = c->ny, nz = c->nz, nz2 = nz / 2 + 1;
    std::vector<cpx> tmp((size_t)nx * ny * nz2);
    cpx *F = reinterpret_cast<cpx *>(f);
    /* x pass inverse on [y][x][kz], written transposed as [x][y][kz] (fftfuncs.cu:322-336) */
    strided_pass(c, F, tmp.data(), ny, nx, nz2, +1, true);
    /* y pass inverse on [x][y][kz] */
    strided_pass(c, tmp.data(), F, nx, ny, nz2, +1, false);
    /* z C2R with the 1/N^3 scale (fftfuncs.cu:341-354, cudafuncs.cu:20-31) */
    zpass_c2r(c, f, 1.0 / ((double)nx * ny * nz));
    return 0;
}

/* ------------------------------------------------------ spectral operators */
/* Spectral loops run over the transposed layout idx = kz + nz2*(x + nx*y). */
#define SPEC_LOOP(G)                                                                   \
    _Pragma("omp parallel for num_threads(nthreads_of(c)) schedule(static)")           \
    for (int j = 0; j < (G).ny; ++j)                                                   \
        for (int i = 0; i < (G).nx; ++i)                                               \
            for (int k = 0; k < (G).nz2; ++k)

/* deAliasKernel_mgpu (solver.cu:17-42): zero modes with k^2 > k_max^2 */
int orc_dealias(const orc_cfg *c, double *fh) {
    if (!valid(c)) return 1;
    Grid g(c);
    cpx *F = reinterpret_cast<cpx *>(fh);
    SPEC_LOOP(g) {
        double k2 = g.kx[i] * g.kx[i] + g.ky[j] * g.ky[j] + g.kz[k] * g.kz[k];
        if (k2 > g.kmax2) F[k + (size_t)g.nz2 * (i + (size_t)g.nx * j)] = {0.0, 0.0};
    }
    return 0;
}

/* calcOmega{1,2,3}Kernel_mgpu (solver.cu:68-114): omega_hat = i k x u_hat */
int orc_vorticity(const orc_cfg *c, const double *uh, const double *vh, const double *wh,
                  double *o1, double *o2, double *o3) {
    if (!valid(c)) return 1;
    Grid g(c);
    const cpx *U = (const cpx *)uh, *V = (const cpx *)vh, *W = (const cpx *)wh;
    cpx *O1 = (cpx *)o1, *O2 = (cpx *)o2, *O3 = (cpx *)o3;
    SPEC_LOOP(g) {
        size_t id = k + (size_t)g.nz2 * (i + (size_t)g.nx * j);
        double k1 = g.kx[i], k2 = g.ky[j], k3 = g.kz[k];
        cpx u = U[id], v = V[id], w = W[id];
        O1[id] = {-k2 * w.im + k3 * v.im, k2 * w.re - k3 * v.re};
        O2[id] = {k1 * w.im - k3 * u.im, -k1 * w.re + k3 * u.re};
        O3[id] = {-k1 * v.im + k2 * u.im, k1 * v.re - k2 * u.re};
    }
    return 0;
}

/* gradientKernel_mgpu (solver.cu:233-256): (i kx f, i ky f, i kz f) */
int orc_gradient(const orc_cfg *c, const double *fh, double *fx, double *fy, double *fz) {
    if (!valid(c)) return 1;
    Grid g(c);
    const cpx *F = (const cpx *)fh;
    cpx *X = (cpx *)fx, *Y = (cpx *)fy, *Z = (cpx *)fz;
    SPEC_LOOP(g) {
        size_t id = k + (size_t)g.nz2 * (i + (size_t)g.nx * j);
        cpx f = F[id];
        X[id] = {-g.kx[i] * f.im, g.kx[i] * f.re};
        Y[id] = {-g.ky[j] * f.im, g.ky[j] * f.re};
        Z[id] = {-g.kz[k] * f.im, g.kz[k] * f.re};
    }
    return 0;
}

/* computeRHSKernel_mgpu (solver.cu:461-521): velocity RHS (k k^T/k^2 - I) N,
 * scalars negated, the k = 0 mode zeroed. */
int orc_make_rhs(const orc_cfg *c, double *ru, double *rv, double *rw, double *rs, double *rc) {
    if (!valid(c)) return 1;
    Grid g(c);
    cpx *U = (cpx *)ru, *V = (cpx *)rv, *W = (cpx *)rw, *S = (cpx *)rs, *C = (cpx *)rc;
    SPEC_LOOP(g) {
        size_t id = k + (size_t)g.nz2 * (i + (size_t)g.nx * j);
        double k1 = g.kx[i], k2 = g.ky[j], k3 = g.kz[k];
        double ksq = k1 * k1 + k2 * k2 + k3 * k3;
        if (i == 0 && j == 0 && k == 0) {
            U[id] = V[id] = W[id] = {0.0, 0.0};
            if (S) S[id] = {0.0, 0.0};
            if (C) C[id] = {0.0, 0.0};
            continue;
        }
        cpx t1 = U[id], t2 = V[id], t3 = W[id];
        U[id].re = (k1 * k1 / ksq - 1.0) * t1.re + (k1 * k2 / ksq) * t2.re + (k1 * k3 / ksq) * t3.re;
        U[id].im = (k1 * k1 / ksq - 1.0) * t1.im + (k1 * k2 / ksq) * t2.im + (k1 * k3 / ksq) * t3.im;
        V[id].re = (k2 * k1 / ksq) * t1.re + (k2 * k2 / ksq - 1.0) * t2.re + (k2 * k3 / ksq) * t3.re;
        V[id].im = (k2 * k1 / ksq) * t1.im + (k2 * k2 / ksq - 1.0) * t2.im + (k2 * k3 / ksq) * t3.im;
        W[id].re = (k3 * k1 / ksq) * t1.re + (k3 * k2 / ksq) * t2.re + (k3 * k3 / ksq - 1.0) * t3.re;
        W[id].im = (k3 * k1 / ksq) * t1.im + (k3 * k2 / ksq) * t2.im + (k3 * k3 / ksq - 1.0) * t3.im;
        if (S) S[id] = {-S[id].re, -S[id].im};
        if (C) C[id] = {-C[id].re, -C[id].im};
    }
    return 0;
}

/* ----------------------------------------------------------- the time step */
/* solver_ps (solver.cu:700-765), statement by statement.  Buffers alias like
 * the reference: a field's real view and complex view share storage. */
int orc_step_cnab2(const orc_cfg *c, double **fields, double **rhs_old, int euler) {
    if (!valid(c)) return 1;
    Grid g(c);
    const size_t ns = g.nspec();
    const int nx = g.nx, ny = g.ny, nz = g.nz, nz2 = g.nz2;
    std::vector<double> rbuf(5 * ns * 2, 0.0), tbuf(3 * ns * 2, 0.0);
    double *vel[5], *rhs[5], *tmp[3];
    for (int q = 0; q < 5; ++q) { vel[q] = fields[q]; rhs[q] = rbuf.data() + q * ns * 2; }
    for (int q = 0; q < 3; ++q) tmp[q] = tbuf.data() + q * ns * 2;
    const int nt = nthreads_of(c);
    auto PH = [&](int i, int j, int k) { return (size_t)k + (size_t)2 * nz2 * ((size_t)j + (size_t)ny * i); };

    /* 1. deAlias(vel)  solver.cu:704 */
    for (int q = 0; q < 5; ++q) orc_dealias(c, vel[q]);
    /* 2. inverse u, v, w  solver.cu:707-709 */
    for (int q = 0; q < 3; ++q) orc_inverse(c, vel[q]);
    /* 3. scalarAdvection  solver.cu:407-459 */
    std::memset(rhs[3], 0, ns * 16); std::memset(rhs[4], 0, ns * 16);   /* :414-415 */
    orc_gradient(c, vel[3], rhs[0], rhs[1], rhs[2]);                    /* :423 */
    {   /* divergence(rhs -> rhs.ch) :425, solver.cu:275-290 */
        const cpx *FX = (const cpx *)rhs[0], *FY = (const cpx *)rhs[1], *FZ = (const cpx *)rhs[2];
        cpx *R = (cpx *)rhs[4];
        SPEC_LOOP(g) {
            size_t id = k + (size_t)nz2 * (i + (size_t)nx * j);
            R[id] = {-g.kx[i] * FX[id].im - g.ky[j] * FY[id].im - g.kz[k] * FZ[id].im,
                     g.kx[i] * FX[id].re + g.ky[j] * FY[id].re + g.kz[k] * FZ[id].re};
        }
    }
    for (int q = 0; q < 3; ++q) orc_inverse(c, rhs[q]);                 /* :428-430 */
    /* dotProduct(vel, rhs -> rhs.s) :432, solver.cu:342-356 */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                size_t id = PH(i, j, k);
                rhs[3][id] = vel[0][id] * rhs[0][id] + vel[1][id] * rhs[1][id] + vel[2][id] * rhs[2][id];
            }
    orc_gradient(c, vel[4], tmp[0], tmp[1], tmp[2]);                    /* :444 */
    for (int q = 0; q < 3; ++q) orc_inverse(c, tmp[q]);                 /* :447-449 */
    orc_inverse(c, rhs[4]);                                             /* :450 */
    orc_inverse(c, vel[4]);                                             /* :451 */
    /* colloidAdvection :454, solver.cu:374-388 */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                size_t id = PH(i, j, k);
                rhs[4][id] = c->alpha * (rhs[4][id] * vel[4][id] + tmp[0][id] * rhs[0][id] +
                                         tmp[1][id] * rhs[1][id] + tmp[2][id] * rhs[2][id]) +
                             vel[0][id] * tmp[0][id] + vel[1][id] * tmp[1][id] + vel[2][id] * tmp[2][id];
            }
    /* 4-5. forward u, v, w, c, rhs.s, rhs.c  solver.cu:715-722 */
    orc_forward(c, vel[0]); orc_forward(c, vel[1]); orc_forward(c, vel[2]); orc_forward(c, vel[4]);
    orc_forward(c, rhs[3]); orc_forward(c, rhs[4]);
    /* 6. vorticity(vel -> rhs.uh..wh)  solver.cu:725 */
    orc_vorticity(c, vel[0], vel[1], vel[2], rhs[0], rhs[1], rhs[2]);
    /* 7-8. inverse omega, inverse velocity  solver.cu:728-737 */
    for (int q = 0; q < 3; ++q) orc_inverse(c, rhs[q]);
    for (int q = 0; q < 3; ++q) orc_inverse(c, vel[q]);
    /* 9. crossProduct: omega x u in place over omega  solver.cu:139-164 */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                size_t id = PH(i, j, k);
                double w1 = rhs[0][id], w2 = rhs[1][id], w3 = rhs[2][id];
                rhs[0][id] = w2 * vel[2][id] - w3 * vel[1][id];
                rhs[1][id] = -w1 * vel[2][id] + w3 * vel[0][id];
                rhs[2][id] = w1 * vel[1][id] - w2 * vel[0][id];
            }
    /* 10-11. forward rhs.u..w and vel.u..w  solver.cu:743-750 */
    for (int q = 0; q < 3; ++q) orc_forward(c, rhs[q]);
    for (int q = 0; q < 3; ++q) orc_forward(c, vel[q]);
    /* 12. makeRHS  solver.cu:753 */
    orc_make_rhs(c, rhs[0], rhs[1], rhs[2], rhs[3], rhs[4]);
    /* 13. deAlias(rhs)  solver.cu:756 */
    for (int q = 0; q < 5; ++q) orc_dealias(c, rhs[q]);
    /* 14. timestep  solver.cu:547-616: CN with Euler (first step) or AB2 */
    const double num[5] = {c->re, c->re, c->re, c->re * c->sc, c->re * c->sc_c};
    const double dt = c->dt;
    for (int q = 0; q < 5; ++q) {
        cpx *F = (cpx *)vel[q];
        const cpx *R = (const cpx *)rhs[q], *RO = (const cpx *)rhs_old[q];
        const double nm = num[q];
        SPEC_LOOP(g) {
            size_t id = k + (size_t)nz2 * (i + (size_t)nx * j);
            double ksq = g.kx[i] * g.kx[i] + g.ky[j] * g.ky[j] + g.kz[k] * g.kz[k];
            double a = 1.0 - dt / 2.0 * ksq / nm, b = 1.0 + dt / 2.0 * ksq / nm;
            if (euler) {
                F[id].re = (a * F[id].re + dt * R[id].re) / b;
                F[id].im = (a * F[id].im + dt * R[id].im) / b;
            } else {
                F[id].re = (a * F[id].re + dt * (1.5 * R[id].re - 0.5 * RO[id].re)) / b;
                F[id].im = (a * F[id].im + dt * (1.5 * R[id].im - 0.5 * RO[id].im)) / b;
            }
        }
    }
    /* 15. update: rhs_old <- rhs  solver.cu:618-657 (rhs is scratch here) */
    for (int q = 0; q < 5; ++q) std::memcpy(rhs_old[q], rhs[q], ns * 16);
    return 0;
}

/* ------------------------------------------------------------ RK3 with IF */
/* Wray low-storage RK3 in integrating-factor form.  Per substep s (1..3):
 *   u_s = E(a_s dt) * (u_{s-1} + g_s dt N_{s-1} + Q_{s-1}),
 *   Q_s = z_{s+1} dt E(a_s dt) N_{s-1},     Q_0 = 0,
 * with E(t) = exp(-nu k^2 t), g = (8/15, 5/12, 3/4), z = (0, -17/60, -5/12),
 * a = g + z.  N is the dealiased, projected nonlinear term P(u x omega) for the
 * velocity and -(u . grad phi) for each scalar (the reference's RHS without
 * the viscous term, solver.cu:461-521). */
static int nonlinear_rhs(const orc_cfg *c, const Grid &g, double **st, double **N, int n_scalars) {
    const size_t ns = g.nspec();
    const int nx = g.nx, ny = g.ny, nz = g.nz, nz2 = g.nz2;
    const int nt = nthreads_of(c);
    std::vector<double> buf(12 * ns * 2);
    double *P[12];
    for (int q = 0; q < 12; ++q) P[q] = buf.data() + q * ns * 2;
    /* dealiased copies of u, v, w and spectral omega, grad s (, grad c) */
    std::vector<double> sc((3 + n_scalars) * ns * 2);
    double *S[5];
    for (int q = 0; q < 3 + n_scalars; ++q) {
        S[q] = sc.data() + q * ns * 2;
        std::memcpy(S[q], st[q], ns * 16);
        orc_dealias(c, S[q]);
    }
    for (int q = 0; q < 3; ++q) std::memcpy(P[q], S[q], ns * 16);
    orc_vorticity(c, S[0], S[1], S[2], P[3], P[4], P[5]);
    orc_gradient(c, S[3], P[6], P[7], P[8]);
    if (n_scalars > 1) orc_gradient(c, S[4], P[9], P[10], P[11]);
    const int np = n_scalars > 1 ? 12 : 9;
    for (int q = 0; q < np; ++q) orc_inverse(c, P[q]);
    auto PH = [&](int i, int j, int k) { return (size_t)k + (size_t)2 * nz2 * ((size_t)j + (size_t)ny * i); };
    for (int q = 0; q < 3 + n_scalars; ++q) std::memset(N[q], 0, ns * 16);
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                size_t id = PH(i, j, k);
                double u = P[0][id], v = P[1][id], w = P[2][id];
                double o1 = P[3][id], o2 = P[4][id], o3 = P[5][id];
                N[0][id] = o2 * w - o3 * v;
                N[1][id] = -o1 * w + o3 * u;
                N[2][id] = o1 * v - o2 * u;
                N[3][id] = u * P[6][id] + v * P[7][id] + w * P[8][id];
                if (n_scalars > 1) N[4][id] = u * P[9][id] + v * P[10][id] + w * P[11][id];
            }
    for (int q = 0; q < 3 + n_scalars; ++q) orc_forward(c, N[q]);
    orc_make_rhs(c, N[0], N[1], N[2], N[3], n_scalars > 1 ? N[4] : nullptr);
    for (int q = 0; q < 3 + n_scalars; ++q) orc_dealias(c, N[q]);
    return 0;
}

int orc_step_rk3if(const orc_cfg *c, double **fields, double **hist, int n_scalars) {
    if (!valid(c) || n_scalars < 1 || n_scalars > 2) return 1;
    Grid g(c);
    const size_t ns = g.nspec();
    const int nf = 3 + n_scalars;
    const int nx = g.nx, nz2 = g.nz2;
    std::vector<double> nbuf(nf * ns * 2);
    double *N[5];
    for (int q = 0; q < nf; ++q) N[q] = nbuf.data() + q * ns * 2;
    const double gam[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
    const double zet[4] = {0.0, -17.0 / 60.0, -5.0 / 12.0, 0.0};
    const double nu[5] = {1.0 / c->re, 1.0 / c->re, 1.0 / c->re, 1.0 / (c->re * c->sc), 1.0 / (c->re * c->sc_c)};
    const double dt = c->dt;
    for (int q = 0; q < nf; ++q) std::memset(hist[q], 0, ns * 16);
    for (int s = 0; s < 3; ++s) {
        nonlinear_rhs(c, g, fields, N, n_scalars);
        const double a = gam[s] + zet[s];
        for (int q = 0; q < nf; ++q) {
            cpx *F = (cpx *)fields[q], *Q = (cpx *)hist[q];
            const cpx *NN = (const cpx *)N[q];
            SPEC_LOOP(g) {
                size_t id = k + (size_t)nz2 * (i + (size_t)nx * j);
                double ksq = g.kx[i] * g.kx[i] + g.ky[j] * g.ky[j] + g.kz[k] * g.kz[k];
                double E = std::exp(-nu[q] * ksq * a * dt);
                cpx f = F[id], n = NN[id], h = Q[id];
                if (ksq > g.kmax2) f = {0.0, 0.0};
                F[id] = {E * (f.re + gam[s] * dt * n.re + h.re), E * (f.im + gam[s] * dt * n.im + h.im)};
                Q[id] = {zet[s + 1] * dt * E * n.re, zet[s + 1] * dt * E * n.im};
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------- statistics */
/* calcVrms / calcDissipationRate / calcScalarDissipationRate
 * (statistics.cu:1494-1585, 1587-1669, 1758-1845): sums over the full spectrum
 * via the kz mirror, normalised by NN^2.  Scalar variance (not in the
 * reference) is the same sum of |s_hat|^2 without the k = 0 mode. */
int orc_stats(const orc_cfg *c, double **fields, double *out) {
    if (!valid(c)) return 1;
    Grid g(c);
    const double NN = (double)g.nx * g.ny * g.nz;
    long double su = 0, se = 0, ss = 0, sc = 0, vs = 0, vc = 0;
    const cpx *U = (const cpx *)fields[0], *V = (const cpx *)fields[1], *W = (const cpx *)fields[2];
    const cpx *S = fields[3] ? (const cpx *)fields[3] : nullptr;
    const cpx *C = fields[4] ? (const cpx *)fields[4] : nullptr;
#pragma omp parallel for num_threads(nthreads_of(c)) reduction(+ : su, se, ss, sc, vs, vc) schedule(static)
    for (int j = 0; j < g.ny; ++j)
        for (int i = 0; i < g.nx; ++i)
            for (int k = 0; k < g.nz2; ++k) {
                size_t id = k + (size_t)g.nz2 * (i + (size_t)g.nx * j);
                double wgt = (k == 0 || 2 * k == g.nz) ? 1.0 : 2.0;
                double ksq = g.kx[i] * g.kx[i] + g.ky[j] * g.ky[j] + g.kz[k] * g.kz[k];
                double e = U[id].re * U[id].re + U[id].im * U[id].im + V[id].re * V[id].re + V[id].im * V[id].im +
                           W[id].re * W[id].re + W[id].im * W[id].im;
                su += wgt * e;
                se += wgt * ksq * e;
                bool k0 = (i == 0 && j == 0 && k == 0);
                if (S) {
                    double m = S[id].re * S[id].re + S[id].im * S[id].im;
                    ss += wgt * ksq * m;
                    if (!k0) vs += wgt * m;
                }
                if (C) {
                    double m = C[id].re * C[id].re + C[id].im * C[id].im;
                    sc += wgt * ksq * m;
                    if (!k0) vc += wgt * m;
                }
            }
    const double n2 = NN * NN;
    out[0] = (double)(su / n2) / 2.0;
    out[1] = (double)(su / n2) / 3.0;
    out[2] = c->nu_stats * (double)(se / n2);
    out[3] = 2.0 * (c->nu_stats / c->sc) * (double)(ss / n2);
    out[4] = 2.0 * (c->nu_stats / c->sc_c) * (double)(sc / n2);
    out[5] = (double)(vs / n2);
    out[6] = (double)(vc / n2);
    return 0;
}

/* calcTurbStats_mgpu (statistics.cu:2039-2156), in the reference's own
 * form: spectral sums for Vrms, KE, epsilon, the integral length and chi
 * (calcVrms, calcDissipationRate, calcIntegralLength,
 * calcScalarDissipationRate); vorticity transformed to physical space for
 * the rms of its components and the volume average of its magnitude
 * (statistics.cu:2083-2106); the fields transformed to physical space and
 * averaged over x and z for the mean profiles (calcYprof, :1943-2003);
 * lambda, eta and l from the derived formulas (:2147-2150). */
int orc_turb_stats(const orc_cfg *c, double **fields, double *out, double *yprof) {
    if (!valid(c)) return 1;
    Grid g(c);
    const double NN = (double)g.nx * g.ny * g.nz;
    const size_t nspec = (size_t)g.nx * g.ny * g.nz2;
    double st[7];
    orc_stats(c, fields, st);
    const double ke = st[0];
    const double vrms = std::sqrt(st[1]);                       /* statistics.cu:1582 */
    const double eps = st[2];
    const double chi = st[3];
    long double sl = 0;                                          /* calcIntegralLengthKernel_mgpu */
    const cpx *U = (const cpx *)fields[0], *V = (const cpx *)fields[1], *W = (const cpx *)fields[2];
#pragma omp parallel for num_threads(nthreads_of(c)) reduction(+ : sl) schedule(static)
    for (int j = 0; j < g.ny; ++j)
        for (int i = 0; i < g.nx; ++i)
            for (int k = 0; k < g.nz2; ++k) {
                const size_t id = k + (size_t)g.nz2 * (i + (size_t)g.nx * j);
                const double wgt = (k == 0 || 2 * k == g.nz) ? 1.0 : 2.0;
                const double ksq = g.kx[i] * g.kx[i] + g.ky[j] * g.ky[j] + g.kz[k] * g.kz[k];
                if (ksq > 0) {
                    const double e = (U[id].re * U[id].re + U[id].im * U[id].im) / (NN * NN) +
                                     (V[id].re * V[id].re + V[id].im * V[id].im) / (NN * NN) +
                                     (W[id].re * W[id].re + W[id].im * W[id].im) / (NN * NN);
                    sl += wgt * e / (2.0 * std::sqrt(ksq));
                }
            }
    /* vorticity in physical space (vorticity + inverseTransform, :2079-2092) */
    std::vector<double> om[3];
    for (auto &o : om) o.assign(2 * nspec, 0.0);
    orc_vorticity(c, fields[0], fields[1], fields[2], om[0].data(), om[1].data(), om[2].data());
    for (auto &o : om) orc_inverse(c, o.data());
    long double s2[3] = {0, 0, 0}, smag = 0;
    for (int i = 0; i < g.nx; ++i)
        for (int j = 0; j < g.ny; ++j)
            for (int k = 0; k < g.nz; ++k) {
                const size_t id = k + 2 * (size_t)g.nz2 * (j + (size_t)g.ny * i);
                const double a = om[0][id], b = om[1][id], d = om[2][id];
                s2[0] += a * a / NN;                            /* volumeAverage_kernel type 1 */
                s2[1] += b * b / NN;
                s2[2] += d * d / NN;
                smag += std::sqrt(a * a + b * b + d * d) / NN;   /* VectorMagnitude + type 0 */
            }
    out[0] = vrms;
    out[1] = ke;
    out[2] = eps;
    out[3] = std::sqrt(std::sqrt(c->nu_stats * c->nu_stats * c->nu_stats / eps));   /* eta, :2149 */
    out[4] = 3 * M_PI / 4 * (double)sl / ke;                                        /* l, :2150 */
    out[5] = std::sqrt(15.0 * c->nu_stats * vrms * vrms / eps);                     /* lambda, :2148 */
    out[6] = chi;
    out[7] = (double)smag;
    out[8] = std::sqrt((double)s2[0]);
    out[9] = std::sqrt((double)s2[1]);
    out[10] = std::sqrt((double)s2[2]);
    if (yprof) {   /* calcYprof: sum over x and z of the physical field / (NX NZ) */
        std::vector<double> f(2 * nspec);
        for (int q = 0; q < 5; ++q) {
            double *pr = yprof + (size_t)q * g.ny;
            for (int j = 0; j < g.ny; ++j) pr[j] = 0.0;
            if (!fields[q]) continue;
            std::copy(fields[q], fields[q] + 2 * nspec, f.begin());
            orc_inverse(c, f.data());
            for (int j = 0; j < g.ny; ++j) {
                long double acc = 0;
                for (int i = 0; i < g.nx; ++i)
                    for (int k = 0; k < g.nz; ++k) acc += f[k + 2 * (size_t)g.nz2 * (j + (size_t)g.ny * i)];
                pr[j] = (double)(acc / ((double)g.nx * g.nz));
            }
        }
    }
    return 0;
}

} /* extern "C" */
