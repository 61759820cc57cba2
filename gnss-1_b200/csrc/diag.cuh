// diag.cuh -- turbulence diagnostics of a spectral state (calcTurbStats_mgpu,
// statistics.cu:2039-2156): the spectral sums behind Vrms, KE, epsilon, the
// integral length and chi, the rms of each vorticity component and the volume
// average of |omega| over the grid, and the mean profiles along y.
//
// Spectral sums run over the full spectrum through the kz mirror (weight 1 on
// kz = 0 and kz = nz/2, 2 elsewhere, as calcVrmsKernel_mgpu's kp = NZ - k
// branch, statistics.cu:1505-1532), Kahan-compensated per thread and reduced
// in a fixed order.  The vorticity statistics are taken, as in the
// reference, over the physical vorticity (statistics.cu:2097-2106): a
// spectral (Parseval) sum would differ from the grid average whenever
// Nyquist modes survive the dealiasing (grids thinner than nx along y or z),
// because the inverse transform drops their imaginary parts.  The
// mean profile of a field along y (calcYprof, statistics.cu:1943-2003: the
// average over x and z) is the inverse DFT in y of its kx = kz = 0 modes.
#pragma once
#include "kernels.cuh"

namespace gnss {

constexpr int TURB_SUMS = 4;   // e, k^2 e, e/(2|k|), k^2 |s|^2
constexpr int VORT_SUMS = 4;   // |w|, w_x^2, w_y^2, w_z^2 over the grid

template <typename T>
__global__ void __launch_bounds__(STAT_THREADS)
k_turb_partial(const __grid_constant__ FieldSet<T> st, int has_s, Geom g, double *__restrict__ partial) {
    using V = V2<T>;
    __shared__ double red[TURB_SUMS][STAT_THREADS];
    Kahan acc[TURB_SUMS];
    const long long nspec = (long long)g.nx * g.ny * g.nz2;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < nspec;
         idx += (long long)gridDim.x * blockDim.x) {
        const int kzi = (int)(idx % g.nz2);
        const long long t = idx / g.nz2;
        const int kxi = (int)(t % g.nx), kyi = (int)(t / g.nx);
        const double k1 = wavenum(kxi, g.nx, g.dkx), k2 = wavenum(kyi, g.ny, g.dky), k3 = wavenum(kzi, g.nz, g.dkz);
        const double ksq = ksq3(k1, k2, k3);
        const double wt = (kzi == 0 || 2 * kzi == g.nz) ? 1.0 : 2.0;
        const V a = st.p[0][idx], b = st.p[1][idx], c = st.p[2][idx];
        const double ax = a.x, ay = a.y, bx = b.x, by = b.y, cx = c.x, cy = c.y;
        const double e = ax * ax + ay * ay + bx * bx + by * by + cx * cx + cy * cy;
        acc[0].add(wt * e);                                   // calcVrmsKernel_mgpu
        acc[1].add(wt * ksq * e);                             // calcEpsilonKernel_mgpu
        if (ksq > 0.0) acc[2].add(wt * e / (2.0 * sqrt(ksq)));   // calcIntegralLengthKernel_mgpu (:1693-1700)
        if (has_s) {
            const V s = st.p[3][idx];
            acc[3].add(wt * ksq * ((double)s.x * s.x + (double)s.y * s.y));   // calcScalarDissipationKernel_mgpu
        }
    }
    for (int q = 0; q < TURB_SUMS; ++q) red[q][threadIdx.x] = acc[q].s;
    __syncthreads();
    for (int w = STAT_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int q = 0; q < TURB_SUMS; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < TURB_SUMS; ++q) partial[blockIdx.x * TURB_SUMS + q] = red[q][0];
}

// Sums over the physical points of the three padded real vorticity fields
// [nx][ny][2 nz2]: sqrt(w1^2 + w2^2 + w3^2) (VectorMagnitude + volumeAverage,
// statistics.cu:2005-2040, 1211-1283) and w1^2, w2^2, w3^2
// (volumeAverage_rms, :1285-1305); one row of VORT_SUMS partials per block.
template <typename T>
__global__ void __launch_bounds__(STAT_THREADS)
k_vort_partial(const T *__restrict__ w1, const T *__restrict__ w2, const T *__restrict__ w3, Geom g,
               double *__restrict__ partial) {
    __shared__ double red[VORT_SUMS][STAT_THREADS];
    Kahan acc[VORT_SUMS];
    const long long npts = (long long)g.nx * g.ny * g.nz;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < npts;
         p += (long long)gridDim.x * blockDim.x) {
        const long long line = p / g.nz;
        const long long idx = line * 2 * g.nz2 + (p - line * g.nz);
        const double a = w1[idx], b = w2[idx], c = w3[idx];
        acc[0].add(sqrt(a * a + b * b + c * c));
        acc[1].add(a * a);
        acc[2].add(b * b);
        acc[3].add(c * c);
    }
    for (int q = 0; q < VORT_SUMS; ++q) red[q][threadIdx.x] = acc[q].s;
    __syncthreads();
    for (int w = STAT_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int q = 0; q < VORT_SUMS; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < VORT_SUMS; ++q) partial[blockIdx.x * VORT_SUMS + q] = red[q][0];
}

template <int NS>
__global__ void __launch_bounds__(NS * 32) k_sums_final(const double *__restrict__ partial, int nblocks, int stride,
                                                        double *__restrict__ out) {
    const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Kahan acc;
    for (int b = lane; b < nblocks; b += 32) acc.add(partial[b * stride + q]);
    double v = acc.s;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) out[q] = v;
}

// Mean profile along y of field f (blockIdx.x), from its kx = kz = 0 modes.
// With the reference's inverse scaling (1/NN, cudafuncs.cu:20-31) the x-z
// average of the physical field is
//   prof[j] = (1/NN) sum_ky Re(f(0, ky, 0) exp(+2 pi i ky j / ny));
// tw holds exp(-2 pi i m / ny).
template <typename T>
__global__ void k_yprof(const __grid_constant__ FieldSet<T> st, Geom g, const V2<T> *__restrict__ tw,
                        double *__restrict__ prof) {
    const V2<T> *f = st.p[blockIdx.x];
    double *out = prof + (long long)blockIdx.x * g.ny;
    if (!f) {
        for (int j = threadIdx.x; j < g.ny; j += blockDim.x) out[j] = 0.0;
        return;
    }
    const long long stride = (long long)g.nx * g.nz2;   // ky stride of the (kx = 0, kz = 0) line
    for (int j = threadIdx.x; j < g.ny; j += blockDim.x) {
        Kahan acc;
        for (int ky = 0; ky < g.ny; ++ky) {
            const V2<T> a = f[ky * stride];
            const V2<T> w = tw[(int)(((long long)ky * j) % g.ny)];
            acc.add((double)a.x * (double)w.x + (double)a.y * (double)w.y);   // Re(a conj(w))
        }
        out[j] = acc.s / ((double)g.nx * g.ny * g.nz);
    }
}

}  // namespace gnss
