// diag.cuh -- turbulence diagnostics of a spectral state (calcTurbStats_mgpu,
// statistics.cu:2039-2156): the spectral sums behind Vrms, KE, epsilon, the
// integral length and chi, the rms of each vorticity component, the volume
// average of |omega| and the mean profiles along y.
//
// Spectral sums run over the full spectrum through the kz mirror (weight 1 on
// kz = 0 and kz = nz/2, 2 elsewhere, as calcVrmsKernel_mgpu's kp = NZ - k
// branch, statistics.cu:1505-1532), Kahan-compensated per thread and reduced
// in a fixed order.  The rms of a vorticity component is the spectral sum of
// |i k x u|^2 (Parseval; the reference averages the squares of the physical
// field, statistics.cu:2103-2105).  |omega| itself has no spectral shortcut:
// it is averaged over the physical vorticity (statistics.cu:2097-2106).  The
// mean profile of a field along y (calcYprof, statistics.cu:1943-2003: the
// average over x and z) is the inverse DFT in y of its kx = kz = 0 modes.
#pragma once
#include "kernels.cuh"

namespace gnss {

constexpr int TURB_SUMS = 7;   // e, k^2 e, e/(2|k|), k^2 |s|^2, |w_x|^2, |w_y|^2, |w_z|^2

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
        // i k x u (calcOmega1..3, solver.cu:68-114): magnitudes of k2 w - k3 v, k3 u - k1 w, k1 v - k2 u
        const double o1r = k2 * cx - k3 * bx, o1i = k2 * cy - k3 * by;
        const double o2r = k3 * ax - k1 * cx, o2i = k3 * ay - k1 * cy;
        const double o3r = k1 * bx - k2 * ax, o3i = k1 * by - k2 * ay;
        acc[4].add(wt * (o1r * o1r + o1i * o1i));
        acc[5].add(wt * (o2r * o2r + o2i * o2i));
        acc[6].add(wt * (o3r * o3r + o3i * o3i));
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

// Sum of sqrt(w1^2 + w2^2 + w3^2) over the physical points of three padded
// real fields [nx][ny][2 nz2] (VectorMagnitude + volumeAverage,
// statistics.cu:2005-2040, 1211-1283); one partial per block in column q0 of
// `partial` (stride TURB_SUMS).
template <typename T>
__global__ void __launch_bounds__(STAT_THREADS)
k_absvort_partial(const T *__restrict__ w1, const T *__restrict__ w2, const T *__restrict__ w3, Geom g,
                  double *__restrict__ partial) {
    __shared__ double red[STAT_THREADS];
    Kahan acc;
    const long long npts = (long long)g.nx * g.ny * g.nz;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < npts;
         p += (long long)gridDim.x * blockDim.x) {
        const long long line = p / g.nz;
        const long long idx = line * 2 * g.nz2 + (p - line * g.nz);
        const double a = w1[idx], b = w2[idx], c = w3[idx];
        acc.add(sqrt(a * a + b * b + c * c));
    }
    red[threadIdx.x] = acc.s;
    __syncthreads();
    for (int w = STAT_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x * TURB_SUMS] = red[0];
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
