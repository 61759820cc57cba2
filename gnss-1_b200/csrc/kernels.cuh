// kernels.cuh -- the B200 kernels of the pseudospectral step.
//
//   k_strided   x / y axis C2C pass over [outer][row][col] tiles, optionally
//               transposed on store, optionally forming ik-derivative
//               combinations of the dealiased state on load (x inverse).
//   k_zpass     z axis R2C / C2R over pairs of contiguous lines (a + ib).
//   k_zphys     fused z C2R of all physical quantities of a line pair, the
//               nonlinear products (omega x u, u.grad s, colloid term) and the
//               z R2C of the products -- the physical fields never touch HBM.
//   k_update    fused spectral sweep: projection, scalar sign, k=0 rule,
//               dealias mask and the CN/AB2 or IF-RK3 update with history.
//   k_stats_*   deterministic compensated statistics reductions.
//   elementwise kernels mirroring the reference's individual operators.
#pragma once
#include "fft.cuh"

namespace gnss {

constexpr int MAXF = 16;

template <typename T> struct FieldSet { V2<T> *p[MAXF]; };

struct Geom {
    int nx, ny, nz, nz2;
    double dkx, dky, dkz;   // 2 pi / L per axis
    double kmax2;           // (alias_filter * nx * pi / lx)^2
};

// initialize.cu:678-691: k_i = (2 pi / L) * i for i < n/2, else (2 pi / L) * (i - n)
__device__ __forceinline__ double wavenum(int i, int n, double dk) {
    return (i < n / 2) ? dk * (double)i : dk * ((double)i - (double)n);
}
// k_sq in the reference's evaluation order (solver.cu:27)
__device__ __forceinline__ double ksq3(double a, double b, double c) {
    return __dadd_rn(__dadd_rn(__dmul_rn(a, a), __dmul_rn(b, b)), __dmul_rn(c, c));
}

// ------------------------------------------------------------ recipes
// A recipe builds one spectral quantity from at most two state fields:
// out = sum_t sign_t * M_t(k) * state[f_t], M in {1, i kx, i ky, i kz, -k^2}.
enum : signed char { M_ONE = 0, M_IKX = 1, M_IKY = 2, M_IKZ = 3, M_LAP = 4 };
struct Recipe { signed char f[2]; signed char m[2]; signed char s[2]; signed char pad[2]; };
struct RecipeSet { Recipe r[MAXF]; };

template <typename V> __device__ __forceinline__ V apply_mult(V a, int m, double kx, double ky, double kz, double k2) {
    using T = decltype(a.x);
    switch (m) {
        case M_IKX: return V{(T)(-kx) * a.y, (T)kx * a.x};
        case M_IKY: return V{(T)(-ky) * a.y, (T)ky * a.x};
        case M_IKZ: return V{(T)(-kz) * a.y, (T)kz * a.x};
        case M_LAP: return V{(T)(-k2) * a.x, (T)(-k2) * a.y};
        default: return a;
    }
}

// ------------------------------------------------------------ strided pass
struct Strides {
    long long s_row, s_out;   // source element strides of the transform index and the outer index
    long long d_row, d_out;   // destination strides (transposed store when they differ)
    int ncols;                // contiguous columns per row (nz2)
    int ncolblk;              // ceil(ncols / NB)
};

template <typename T, int N> struct StridedCfg {
    static constexpr int NB = (sizeof(T) == 8) ? ((N >= 512) ? 8 : 16) : 16;
    static constexpr int NT0 = N * NB / 16;
    static constexpr int NT = NT0 < 32 ? 32 : (NT0 > 512 ? 512 : NT0);
    static constexpr int SMEM = (plan_nstages(N) > 1) ? N * NB * (int)sizeof(V2<T>) : 0;
};

// grid: x = outer * ncolblk + colblk, y = field (or recipe) index.
// LOAD_RECIPE: row = kx index, outer = ky index, col = kz index of the
// spectral state in src.p[0..4]; recipe blockIdx.y selects the combination.
template <typename T, int N, int SIGN, bool RECIPE>
__global__ void __launch_bounds__(StridedCfg<T, N>::NT)
k_strided(FieldSet<T> src, FieldSet<T> dst, Strides st, Geom g, RecipeSet rs, const V2<T> *__restrict__ tw) {
    using V = V2<T>;
    using C = StridedCfg<T, N>;
    constexpr int NB = C::NB, NT = C::NT;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *sm = reinterpret_cast<V *>(smem_raw);
    const int tid = threadIdx.x;
    const int o = blockIdx.x / st.ncolblk;
    const int c0 = (blockIdx.x % st.ncolblk) * NB;
    const int f = blockIdx.y;
    const V *__restrict__ s = src.p[f];
    V *__restrict__ d = dst.p[f];
    const long long sbase = (long long)o * st.s_out + c0;
    const long long dbase = (long long)o * st.d_out + c0;
    const int ncols = st.ncols;

    auto gld = [&](int row, int b) -> V {
        const int col = c0 + b;
        if (col >= ncols) return V{T(0), T(0)};
        const long long idx = sbase + (long long)row * st.s_row + b;
        if constexpr (!RECIPE) {
            return s[idx];
        } else {
            const Recipe rc = rs.r[f];
            const double kx = wavenum(row, g.nx, g.dkx);
            const double ky = wavenum(o, g.ny, g.dky);
            const double kz = wavenum(col, g.nz, g.dkz);
            const double k2 = ksq3(kx, ky, kz);
            V acc = V{T(0), T(0)};
            if (k2 > g.kmax2) return acc;   // dealias mask (solver.cu:36)
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                if (rc.f[t] >= 0) {
                    V a = apply_mult(src.p[rc.f[t]][idx], rc.m[t], kx, ky, kz, k2);
                    acc = rc.s[t] > 0 ? cadd(acc, a) : csub(acc, a);
                }
            }
            return acc;
        }
    };
    auto gst = [&](int row, int b, V v) {
        if (c0 + b < ncols) d[dbase + (long long)row * st.d_row + b] = v;
    };
    auto smacc = [&](int row, int b) -> V & { return sm[row * NB + b]; };
    fft_columns<T, N, SIGN, NB, NT>(tid, tw, gld, smacc, gst, SyncBlock{});
}

// ------------------------------------------------------------ z pass
// One warp per pair of contiguous lines (la, la+1) of one field; 8 warps per
// block.  DIR < 0: real padded lines -> nz2 complex per line (R2C, in place).
// DIR > 0: nz2 complex -> real padded lines scaled by `scale` (C2R, in place);
// the imaginary parts of the kz = 0 and kz = nz/2 entries are ignored and the
// two padding reals of each line are set to zero.
constexpr int ZWARPS = 8;

template <typename T, int N> struct ZCfg {
    static constexpr int LEN = padded_len<T>(N);
    static constexpr int SMEM = ZWARPS * LEN * (int)sizeof(V2<T>);
};

// In-place FFT of one padded line in shared memory by one warp.
template <typename T, int N, int SIGN, int S = 0>
__device__ __forceinline__ void warp_line_fft(int lane, V2<T> *line, const V2<T> *tw) {
    using V = V2<T>;
    if constexpr (S < plan_nstages(N)) {
        fft_stage<T, N, S, SIGN, 1, 32, true>(
            lane, tw, [&](int row, int) -> V { return line[padded<T>(row)]; },
            [&](int row, int, V v) { line[padded<T>(row)] = v; }, SyncWarp{});
        __syncwarp();
        warp_line_fft<T, N, SIGN, S + 1>(lane, line, tw);
    }
}

// Z_k = A_k + i B_k for k <= N/2 and Z_{N-k} = conj(A_k) + i conj(B_k), from
// the half spectra of two real lines (C2R packing); Im of A_0, B_0, A_{N/2},
// B_{N/2} ignored.
template <typename T, int N>
__device__ __forceinline__ void pack_c2r(int lane, V2<T> *line, const V2<T> *__restrict__ A, const V2<T> *__restrict__ B,
                                         bool hasB) {
    using V = V2<T>;
    for (int k = lane; k <= N / 2; k += 32) {
        V a = A[k];
        V b = hasB ? B[k] : V{T(0), T(0)};
        if (k == 0 || 2 * k == N) { a.y = T(0); b.y = T(0); }
        line[padded<T>(k)] = V{a.x - b.y, a.y + b.x};
        if (k > 0 && 2 * k < N) line[padded<T>(N - k)] = V{a.x + b.y, b.x - a.y};
    }
}

// A_k = (Z_k + conj Z_{N-k})/2, B_k = (Z_k - conj Z_{N-k})/(2i), k = 0..N/2.
template <typename T, int N>
__device__ __forceinline__ void unpack_r2c(int lane, const V2<T> *line, V2<T> *__restrict__ A, V2<T> *__restrict__ B,
                                           bool hasB) {
    using V = V2<T>;
    for (int k = lane; k <= N / 2; k += 32) {
        V zk = line[padded<T>(k)];
        V zm = line[padded<T>((N - k) % N)];
        A[k] = V{T(0.5) * (zk.x + zm.x), T(0.5) * (zk.y - zm.y)};
        if (hasB) B[k] = V{T(0.5) * (zk.y + zm.y), T(-0.5) * (zk.x - zm.x)};
    }
}

template <typename T, int N, int DIR>
__global__ void __launch_bounds__(ZWARPS * 32)
k_zpass(FieldSet<T> f, long long nlines, int nz2, T scale, const V2<T> *__restrict__ tw) {
    using V = V2<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    V *line = reinterpret_cast<V *>(smem_raw) + warp * ZCfg<T, N>::LEN;
    const long long pair = (long long)blockIdx.x * ZWARPS + warp;
    const long long la = 2 * pair, lb = la + 1;
    if (la >= nlines) return;
    const bool hasB = lb < nlines;
    V *base = f.p[blockIdx.y];
    if constexpr (DIR < 0) {
        const T *ra = reinterpret_cast<const T *>(base + la * nz2);
        const T *rb = reinterpret_cast<const T *>(base + lb * nz2);
        for (int n = lane; n < N; n += 32) line[padded<T>(n)] = V{ra[n], hasB ? rb[n] : T(0)};
        __syncwarp();
        warp_line_fft<T, N, -1>(lane, line, tw);
        unpack_r2c<T, N>(lane, line, base + la * nz2, base + lb * nz2, hasB);
    } else {
        pack_c2r<T, N>(lane, line, base + la * nz2, base + lb * nz2, hasB);
        __syncwarp();
        warp_line_fft<T, N, +1>(lane, line, tw);
        T *ra = reinterpret_cast<T *>(base + la * nz2);
        T *rb = reinterpret_cast<T *>(base + lb * nz2);
        for (int n = lane; n < 2 * nz2; n += 32) {
            V z = n < N ? line[padded<T>(n)] : V{T(0), T(0)};
            ra[n] = z.x * scale;
            if (hasB) rb[n] = z.y * scale;
        }
    }
}

// ------------------------------------------------------------ fused z + products
// Inputs (in f.p, [x][y][kz] lines after the x and y inverse passes):
//   0 u, 1 v, 2 w, 3 w1, 4 w2, 5 w3, 6 sx, 7 sy, 8 sz,
//   [9 cx, 10 cy, 11 cz]            when two scalars,
//   [12 c, 13 lap s]                when two scalars and alpha != 0.
// Outputs written in place into f.p[0..nout): z R2C of
//   0 (w x u)_x, 1 (w x u)_y, 2 (w x u)_z    (crossProductKernel_mgpu, solver.cu:139-164)
//   3 u . grad s                             (dotKernel_mgpu, solver.cu:342-356)
//   4 alpha (lap s c + grad c . grad s) + u . grad c   (colloidAdvectionKernel_mgpu, solver.cu:374-388)
// One warp per input field; one block per line pair.
template <typename T, int N> struct ZPCfg {
    static constexpr int LEN = padded_len<T>(N);
};

template <typename T, int N>
__global__ void __launch_bounds__(14 * 32)
k_zphys(FieldSet<T> f, int nin, int nout, long long nlines, int nz2, T scale, T alpha, const V2<T> *__restrict__ tw) {
    using V = V2<T>;
    constexpr int LEN = ZPCfg<T, N>::LEN;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V *reg = reinterpret_cast<V *>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long la = 2 * (long long)blockIdx.x, lb = la + 1;
    const bool hasB = lb < nlines;
    // phase 1: every warp brings one quantity to physical space
    if (warp < nin) {
        V *line = reg + warp * LEN;
        const V *src = f.p[warp];
        pack_c2r<T, N>(lane, line, src + la * nz2, src + lb * nz2, hasB);
        __syncwarp();
        warp_line_fft<T, N, +1>(lane, line, tw);
    }
    __syncthreads();
    // phase 2: pointwise products on both lines (real part = line a, imag = line b)
    const bool has_c = nin >= 12, has_al = nin >= 14;
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
        const int pn = padded<T>(n);
        V u = reg[0 * LEN + pn], v = reg[1 * LEN + pn], w = reg[2 * LEN + pn];
        V o1 = reg[3 * LEN + pn], o2 = reg[4 * LEN + pn], o3 = reg[5 * LEN + pn];
        V sx = reg[6 * LEN + pn], sy = reg[7 * LEN + pn], sz = reg[8 * LEN + pn];
        u = cscale(u, scale); v = cscale(v, scale); w = cscale(w, scale);
        o1 = cscale(o1, scale); o2 = cscale(o2, scale); o3 = cscale(o3, scale);
        sx = cscale(sx, scale); sy = cscale(sy, scale); sz = cscale(sz, scale);
        V n1 = V{o2.x * w.x - o3.x * v.x, o2.y * w.y - o3.y * v.y};
        V n2 = V{-o1.x * w.x + o3.x * u.x, -o1.y * w.y + o3.y * u.y};
        V n3 = V{o1.x * v.x - o2.x * u.x, o1.y * v.y - o2.y * u.y};
        V ns = V{u.x * sx.x + v.x * sy.x + w.x * sz.x, u.y * sx.y + v.y * sy.y + w.y * sz.y};
        V nc = V{T(0), T(0)};
        if (has_c) {
            V cx = cscale(reg[9 * LEN + pn], scale), cy = cscale(reg[10 * LEN + pn], scale);
            V cz = cscale(reg[11 * LEN + pn], scale);
            V adv = V{u.x * cx.x + v.x * cy.x + w.x * cz.x, u.y * cx.y + v.y * cy.y + w.y * cz.y};
            if (has_al) {
                V cc = cscale(reg[12 * LEN + pn], scale), ls = cscale(reg[13 * LEN + pn], scale);
                V dr = V{ls.x * cc.x + cx.x * sx.x + cy.x * sy.x + cz.x * sz.x,
                         ls.y * cc.y + cx.y * sx.y + cy.y * sy.y + cz.y * sz.y};
                nc = V{alpha * dr.x + adv.x, alpha * dr.y + adv.y};
            } else {
                nc = adv;
            }
        }
        reg[0 * LEN + pn] = n1;
        reg[1 * LEN + pn] = n2;
        reg[2 * LEN + pn] = n3;
        reg[3 * LEN + pn] = ns;
        if (has_c) reg[4 * LEN + pn] = nc;
    }
    __syncthreads();
    // phase 3: z R2C of the products, written over the input lines
    if (warp < nout) {
        V *line = reg + warp * LEN;
        warp_line_fft<T, N, -1>(lane, line, tw);
        V *dstp = f.p[warp];
        unpack_r2c<T, N>(lane, line, dstp + la * nz2, dstp + lb * nz2, hasB);
    }
}

// ------------------------------------------------------------ spectral update
struct UpdCoef {
    int nf;           // fields updated: 3 + n_scalars
    int scheme;       // GNSS_SCHEME_*
    int euler;        // CN/AB2: first step
    double dt;
    double num[5];    // CN: reference "num" (Re, Re*Sc, Re*Sc_c)
    double nu[5];     // IF: diffusivity per field
    double gam, zet_next, alph;   // IF-RK3 substep coefficients
    int substep;      // IF-RK3: 0, 1, 2 (substep 0 ignores the history input)
};

template <typename T>
__global__ void __launch_bounds__(256)
k_update(FieldSet<T> state, FieldSet<T> hist, FieldSet<T> nl, Geom g, UpdCoef c) {
    using V = V2<T>;
    const long long nspec = (long long)g.nx * g.ny * g.nz2;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < nspec;
         idx += (long long)gridDim.x * blockDim.x) {
        const int kzi = (int)(idx % g.nz2);
        const long long t = idx / g.nz2;
        const int kxi = (int)(t % g.nx);
        const int kyi = (int)(t / g.nx);
        const double k1 = wavenum(kxi, g.nx, g.dkx), k2 = wavenum(kyi, g.ny, g.dky), k3 = wavenum(kzi, g.nz, g.dkz);
        const double ksq = ksq3(k1, k2, k3);
        const bool masked = ksq > g.kmax2;
        double R[5][2];
        // makeRHS (solver.cu:461-521): (k k^T / k^2 - I) N for the velocity,
        // -N for the scalars, zero at k = 0; then deAlias(rhs) (solver.cu:756)
        if ((kxi == 0 && kyi == 0 && kzi == 0) || masked) {
            for (int q = 0; q < 5; ++q) R[q][0] = R[q][1] = 0.0;
        } else {
            V a = nl.p[0][idx], b = nl.p[1][idx], cc = nl.p[2][idx];
            double t1r = a.x, t1c = a.y, t2r = b.x, t2c = b.y, t3r = cc.x, t3c = cc.y;
            R[0][0] = (k1 * k1 / ksq - 1.0) * t1r + (k1 * k2 / ksq) * t2r + (k1 * k3 / ksq) * t3r;
            R[0][1] = (k1 * k1 / ksq - 1.0) * t1c + (k1 * k2 / ksq) * t2c + (k1 * k3 / ksq) * t3c;
            R[1][0] = (k2 * k1 / ksq) * t1r + (k2 * k2 / ksq - 1.0) * t2r + (k2 * k3 / ksq) * t3r;
            R[1][1] = (k2 * k1 / ksq) * t1c + (k2 * k2 / ksq - 1.0) * t2c + (k2 * k3 / ksq) * t3c;
            R[2][0] = (k3 * k1 / ksq) * t1r + (k3 * k2 / ksq) * t2r + (k3 * k3 / ksq - 1.0) * t3r;
            R[2][1] = (k3 * k1 / ksq) * t1c + (k3 * k2 / ksq) * t2c + (k3 * k3 / ksq - 1.0) * t3c;
            for (int q = 3; q < c.nf; ++q) {
                V s = nl.p[q][idx];
                R[q][0] = -(double)s.x;
                R[q][1] = -(double)s.y;
            }
        }
        for (int q = 0; q < c.nf; ++q) {
            V fv = state.p[q][idx];
            double fr = masked ? 0.0 : (double)fv.x, fi = masked ? 0.0 : (double)fv.y;
            if (c.scheme == 0) {
                // eulerKernel_mgpu / adamsBashforthKernel_mgpu (solver.cu:547-585)
                const double a = 1.0 - c.dt / 2.0 * ksq / c.num[q];
                const double bb = 1.0 + c.dt / 2.0 * ksq / c.num[q];
                double nr, ni;
                if (c.euler) {
                    nr = (a * fr + c.dt * R[q][0]) / bb;
                    ni = (a * fi + c.dt * R[q][1]) / bb;
                } else {
                    V ro = hist.p[q][idx];
                    nr = (a * fr + c.dt * (1.5 * R[q][0] - 0.5 * (double)ro.x)) / bb;
                    ni = (a * fi + c.dt * (1.5 * R[q][1] - 0.5 * (double)ro.y)) / bb;
                }
                state.p[q][idx] = V{(T)nr, (T)ni};
                hist.p[q][idx] = V{(T)R[q][0], (T)R[q][1]};   // updateKernel_mgpu (solver.cu:618-637)
            } else {
                const double E = exp(-c.nu[q] * ksq * c.alph * c.dt);
                double hr = 0.0, hi = 0.0;
                if (c.substep > 0) {
                    V h = hist.p[q][idx];
                    hr = (double)h.x;
                    hi = (double)h.y;
                }
                const double nr = E * (fr + c.gam * c.dt * R[q][0] + hr);
                const double ni = E * (fi + c.gam * c.dt * R[q][1] + hi);
                state.p[q][idx] = V{(T)nr, (T)ni};
                hist.p[q][idx] = V{(T)(c.zet_next * c.dt * E * R[q][0]), (T)(c.zet_next * c.dt * E * R[q][1])};
            }
        }
    }
}

// ------------------------------------------------------------ statistics
// Six sums per thread, Kahan-compensated, reduced in a fixed tree order per
// block; the partials are summed in a fixed order by one block.  The result
// is independent of scheduling (unlike atomicAdd in statistics.cu:1555).
constexpr int STAT_SUMS = 6;
constexpr int STAT_BLOCKS = 1184;   // 8 x 148 SMs
constexpr int STAT_THREADS = 256;

struct Kahan {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add(double x) {
        double y = x - c;
        double t = s + y;
        c = (t - s) - y;
        s = t;
    }
};

template <typename T>
__global__ void __launch_bounds__(STAT_THREADS)
k_stats_partial(FieldSet<T> st, int has_s, int has_c, Geom g, double *__restrict__ partial) {
    using V = V2<T>;
    __shared__ double red[STAT_SUMS][STAT_THREADS];
    Kahan acc[STAT_SUMS];
    const long long nspec = (long long)g.nx * g.ny * g.nz2;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < nspec;
         idx += (long long)gridDim.x * blockDim.x) {
        const int kzi = (int)(idx % g.nz2);
        const long long t = idx / g.nz2;
        const int kxi = (int)(t % g.nx), kyi = (int)(t / g.nx);
        const double k1 = wavenum(kxi, g.nx, g.dkx), k2 = wavenum(kyi, g.ny, g.dky), k3 = wavenum(kzi, g.nz, g.dkz);
        const double ksq = ksq3(k1, k2, k3);
        const double wt = (kzi == 0 || 2 * kzi == g.nz) ? 1.0 : 2.0;   // kz mirror (statistics.cu:1505-1532)
        V a = st.p[0][idx], b = st.p[1][idx], c = st.p[2][idx];
        const double e = (double)a.x * a.x + (double)a.y * a.y + (double)b.x * b.x + (double)b.y * b.y +
                         (double)c.x * c.x + (double)c.y * c.y;
        acc[0].add(wt * e);
        acc[1].add(wt * ksq * e);
        const bool k0 = (idx == 0);
        if (has_s) {
            V s = st.p[3][idx];
            const double m = (double)s.x * s.x + (double)s.y * s.y;
            acc[2].add(wt * ksq * m);
            if (!k0) acc[4].add(wt * m);
        }
        if (has_c) {
            V s = st.p[4][idx];
            const double m = (double)s.x * s.x + (double)s.y * s.y;
            acc[3].add(wt * ksq * m);
            if (!k0) acc[5].add(wt * m);
        }
    }
    for (int q = 0; q < STAT_SUMS; ++q) red[q][threadIdx.x] = acc[q].s;
    __syncthreads();
    for (int w = STAT_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int q = 0; q < STAT_SUMS; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < STAT_SUMS; ++q) partial[blockIdx.x * STAT_SUMS + q] = red[q][0];
}

__global__ void __launch_bounds__(STAT_SUMS * 32) k_stats_final(const double *__restrict__ partial, int nblocks,
                                                                 double *__restrict__ out) {
    // warp q sums column q: lanes stride the blocks, then a fixed shuffle tree
    const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Kahan acc;
    for (int b = lane; b < nblocks; b += 32) acc.add(partial[b * STAT_SUMS + q]);
    double v = acc.s;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) out[q] = v;
}

// ------------------------------------------------------------ reference-surface ops
// Spectral index helpers for the transposed layout idx = kz + nz2*(x + nx*y).
struct SpecIdx {
    int kx, ky, kz;
    __device__ __forceinline__ SpecIdx(long long idx, const Geom &g) {
        kz = (int)(idx % g.nz2);
        long long t = idx / g.nz2;
        kx = (int)(t % g.nx);
        ky = (int)(t / g.nx);
    }
};

#define GNSS_GRID_STRIDE(n) \
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < (n); idx += (long long)gridDim.x * blockDim.x)

template <typename T> __global__ void k_dealias(V2<T> *f, Geom g) {
    const long long ns = (long long)g.nx * g.ny * g.nz2;
    GNSS_GRID_STRIDE(ns) {
        SpecIdx s(idx, g);
        const double k1 = wavenum(s.kx, g.nx, g.dkx), k2 = wavenum(s.ky, g.ny, g.dky), k3 = wavenum(s.kz, g.nz, g.dkz);
        if (ksq3(k1, k2, k3) > g.kmax2) f[idx] = V2<T>{T(0), T(0)};
    }
}

template <typename T>
__global__ void k_vorticity(const V2<T> *u, const V2<T> *v, const V2<T> *w, V2<T> *o1, V2<T> *o2, V2<T> *o3, Geom g) {
    using V = V2<T>;
    const long long ns = (long long)g.nx * g.ny * g.nz2;
    GNSS_GRID_STRIDE(ns) {
        SpecIdx s(idx, g);
        const T k1 = (T)wavenum(s.kx, g.nx, g.dkx), k2 = (T)wavenum(s.ky, g.ny, g.dky), k3 = (T)wavenum(s.kz, g.nz, g.dkz);
        V a = u[idx], b = v[idx], c = w[idx];
        o1[idx] = V{-k2 * c.y + k3 * b.y, k2 * c.x - k3 * b.x};
        o2[idx] = V{k1 * c.y - k3 * a.y, -k1 * c.x + k3 * a.x};
        o3[idx] = V{-k1 * b.y + k2 * a.y, k1 * b.x - k2 * a.x};
    }
}

template <typename T> __global__ void k_gradient(const V2<T> *f, V2<T> *fx, V2<T> *fy, V2<T> *fz, Geom g) {
    using V = V2<T>;
    const long long ns = (long long)g.nx * g.ny * g.nz2;
    GNSS_GRID_STRIDE(ns) {
        SpecIdx s(idx, g);
        const T k1 = (T)wavenum(s.kx, g.nx, g.dkx), k2 = (T)wavenum(s.ky, g.ny, g.dky), k3 = (T)wavenum(s.kz, g.nz, g.dkz);
        V a = f[idx];
        fx[idx] = V{-k1 * a.y, k1 * a.x};
        fy[idx] = V{-k2 * a.y, k2 * a.x};
        fz[idx] = V{-k3 * a.y, k3 * a.x};
    }
}

template <typename T>
__global__ void k_divergence(const V2<T> *fx, const V2<T> *fy, const V2<T> *fz, V2<T> *out, Geom g) {
    using V = V2<T>;
    const long long ns = (long long)g.nx * g.ny * g.nz2;
    GNSS_GRID_STRIDE(ns) {
        SpecIdx s(idx, g);
        const T k1 = (T)wavenum(s.kx, g.nx, g.dkx), k2 = (T)wavenum(s.ky, g.ny, g.dky), k3 = (T)wavenum(s.kz, g.nz, g.dkz);
        V a = fx[idx], b = fy[idx], c = fz[idx];
        out[idx] = V{-k1 * a.y - k2 * b.y - k3 * c.y, k1 * a.x + k2 * b.x + k3 * c.x};
    }
}

template <typename T>
__global__ void k_make_rhs(V2<T> *ru, V2<T> *rv, V2<T> *rw, V2<T> *rs, V2<T> *rc, Geom g) {
    using V = V2<T>;
    const long long ns = (long long)g.nx * g.ny * g.nz2;
    GNSS_GRID_STRIDE(ns) {
        SpecIdx s(idx, g);
        const double k1 = wavenum(s.kx, g.nx, g.dkx), k2 = wavenum(s.ky, g.ny, g.dky), k3 = wavenum(s.kz, g.nz, g.dkz);
        const double ksq = ksq3(k1, k2, k3);
        if (s.kx == 0 && s.ky == 0 && s.kz == 0) {
            ru[idx] = rv[idx] = rw[idx] = V{T(0), T(0)};
            if (rs) rs[idx] = V{T(0), T(0)};
            if (rc) rc[idx] = V{T(0), T(0)};
            continue;
        }
        V a = ru[idx], b = rv[idx], c = rw[idx];
        double t1r = a.x, t1c = a.y, t2r = b.x, t2c = b.y, t3r = c.x, t3c = c.y;
        ru[idx] = V{(T)((k1 * k1 / ksq - 1.0) * t1r + (k1 * k2 / ksq) * t2r + (k1 * k3 / ksq) * t3r),
                    (T)((k1 * k1 / ksq - 1.0) * t1c + (k1 * k2 / ksq) * t2c + (k1 * k3 / ksq) * t3c)};
        rv[idx] = V{(T)((k2 * k1 / ksq) * t1r + (k2 * k2 / ksq - 1.0) * t2r + (k2 * k3 / ksq) * t3r),
                    (T)((k2 * k1 / ksq) * t1c + (k2 * k2 / ksq - 1.0) * t2c + (k2 * k3 / ksq) * t3c)};
        rw[idx] = V{(T)((k3 * k1 / ksq) * t1r + (k3 * k2 / ksq) * t2r + (k3 * k3 / ksq - 1.0) * t3r),
                    (T)((k3 * k1 / ksq) * t1c + (k3 * k2 / ksq) * t2c + (k3 * k3 / ksq - 1.0) * t3c)};
        if (rs) { V q = rs[idx]; rs[idx] = V{-q.x, -q.y}; }
        if (rc) { V q = rc[idx]; rc[idx] = V{-q.x, -q.y}; }
    }
}

template <typename T>
__global__ void k_timestep(V2<T> *f, const V2<T> *r, const V2<T> *ro, double num, double dt, int euler, Geom g) {
    using V = V2<T>;
    const long long ns = (long long)g.nx * g.ny * g.nz2;
    GNSS_GRID_STRIDE(ns) {
        SpecIdx s(idx, g);
        const double k1 = wavenum(s.kx, g.nx, g.dkx), k2 = wavenum(s.ky, g.ny, g.dky), k3 = wavenum(s.kz, g.nz, g.dkz);
        const double ksq = ksq3(k1, k2, k3);
        const double a = 1.0 - dt / 2.0 * ksq / num, b = 1.0 + dt / 2.0 * ksq / num;
        V fv = f[idx], rv = r[idx];
        double nr, ni;
        if (euler) {
            nr = (a * fv.x + dt * rv.x) / b;
            ni = (a * fv.y + dt * rv.y) / b;
        } else {
            V o = ro[idx];
            nr = (a * fv.x + dt * (1.5 * rv.x - 0.5 * o.x)) / b;
            ni = (a * fv.y + dt * (1.5 * rv.y - 0.5 * o.y)) / b;
        }
        f[idx] = V{(T)nr, (T)ni};
    }
}

template <typename T> __global__ void k_shift_history(V2<T> *r, V2<T> *ro, long long ns) {
    GNSS_GRID_STRIDE(ns) {
        ro[idx] = r[idx];
        r[idx] = V2<T>{T(0), T(0)};
    }
}

// physical-space point loop over x < nx, y < ny, z < nz of the padded layout
struct PhysIdx {
    long long p;
    __device__ __forceinline__ PhysIdx(long long idx, const Geom &g) {
        const int z = (int)(idx % g.nz);
        const long long t = idx / g.nz;
        const int y = (int)(t % g.ny);
        const int x = (int)(t / g.ny);
        p = (long long)z + 2LL * g.nz2 * ((long long)y + (long long)g.ny * x);
    }
};

template <typename T>
__global__ void k_cross(const T *u, const T *v, const T *w, T *o1, T *o2, T *o3, Geom g) {
    const long long np = (long long)g.nx * g.ny * g.nz;
    GNSS_GRID_STRIDE(np) {
        const long long p = PhysIdx(idx, g).p;
        const T w1 = o1[p], w2 = o2[p], w3 = o3[p];
        o1[p] = w2 * w[p] - w3 * v[p];
        o2[p] = -w1 * w[p] + w3 * u[p];
        o3[p] = w1 * v[p] - w2 * u[p];
    }
}

template <typename T>
__global__ void k_dot(const T *a1, const T *a2, const T *a3, const T *b1, const T *b2, const T *b3, T *out, Geom g) {
    const long long np = (long long)g.nx * g.ny * g.nz;
    GNSS_GRID_STRIDE(np) {
        const long long p = PhysIdx(idx, g).p;
        out[p] = a1[p] * b1[p] + a2[p] * b2[p] + a3[p] * b3[p];
    }
}

template <typename T>
__global__ void k_colloid(const T *u, const T *v, const T *w, const T *c, const T *cx, const T *cy, const T *cz,
                          const T *sx, const T *sy, const T *sz, T *lap, T alpha, Geom g) {
    const long long np = (long long)g.nx * g.ny * g.nz;
    GNSS_GRID_STRIDE(np) {
        const long long p = PhysIdx(idx, g).p;
        lap[p] = alpha * (lap[p] * c[p] + cx[p] * sx[p] + cy[p] * sy[p] + cz[p] * sz[p]) + u[p] * cx[p] +
                 v[p] * cy[p] + w[p] * cz[p];
    }
}

}  // namespace gnss
