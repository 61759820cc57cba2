// ic.cu -- the reference's initial temporal jet (initializeJet,
// initialize.cu:615-641), then forward transforms and dealiasing as main.cu
// does (main.cu:149-156).
//
//   noise      generateNoise (initialize.cu:303-612): Gaussian energy spectrum
//              (peak 6 dk, band 20 dk, rms 1) on the modes |k| < kmax, random
//              complex amplitudes from the C library's rand() stream seeded
//              with srand(666*37 + 37*13), the solenoidal cross product ik x A,
//              conjugate symmetry on the kz = 0 plane, scaled by NN; the
//              sequence of random draws is the reference's loop order
//              (x, then y, then kz) and runs on the host, with a private
//              random_r state (the same generator as rand(), so the caller's
//              rand() is left alone).  The spectral noise is moved to the
//              device and inverse-transformed there;
//   jet        u = 0.5 - 0.5 tanh(H/(4 theta)(2|y|/H - 1)) + pert_amp noise_u,
//              v, w = pert_amp noise (initializeVelocityKernel_mgpu,
//              velocitySuperpositionKernel_mgpu, initialize.cu:114-142, 249-264);
//   scalars    s with theta, c with theta_c (initialize.cu:160-194);
//   then       forward transforms and dealiasing, on the device.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "gnss_b200.h"

namespace {

struct Cpx {
    double x, y;
};

// the C library's rand() generator (random_r, 128-byte state) with its own state
struct LibcRand {
    random_data rd;
    alignas(8) char state[128];
    explicit LibcRand(unsigned seed) {
        std::memset(&rd, 0, sizeof rd);
        initstate_r(seed, state, sizeof state, &rd);
    }
    int next() {
        int32_t r = 0;
        random_r(&rd, &r);
        return (int)r;
    }
};

// random_normal (initialize.cu:286-301)
void random_normal(LibcRand &g, double *val, double mu, double sigma) {
    double A, B;
    val[0] = (double)g.next() / RAND_MAX;
    val[1] = (double)g.next() / RAND_MAX;
    A = sigma * std::sqrt(-2.0 * std::log(val[0]));
    B = 2.0 * M_PI * val[1];
    val[0] = A * std::cos(B) + mu;
    val[1] = A * std::sin(B) + mu;
}

// waveNumber_kernel (initialize.cu:678-691)
std::vector<double> wavenumbers(int n, double l) {
    std::vector<double> k(n);
    for (int i = 0; i < n; ++i) k[i] = (i < n / 2) ? (2 * M_PI / l) * (double)i : (2 * M_PI / l) * ((double)i - n);
    return k;
}

// generateNoise (initialize.cu:303-588): the three spectral noise fields,
// transposed layout [ky][kx][kz], scaled by NN.
void generate_noise(const gnss_config &cfg, unsigned seed, std::vector<Cpx> A[3]) {
    const int NX = cfg.nx, NY = cfg.ny, NZ = cfg.nz, NZ2 = NZ / 2 + 1;
    const double NN = (double)NX * NY * NZ;
    const double dkx = 2.0 * M_PI / cfg.lx, dky = 2.0 * M_PI / cfg.ly, dkz = 2.0 * M_PI / cfg.lz;
    const double kxmax = (NX / 2 - 1) * dkx, kymax = (NY / 2 - 1) * dky, kzmax = (NZ / 2 - 1) * dkz;
    double kmax = kxmax;
    if (kymax < kmax) kmax = kymax;
    if (kzmax < kmax) kmax = kzmax;
    double dk = dkx;
    if (dky > dk) dk = dky;
    if (dkz > dk) dk = dkz;
    const int nbins = (int)(kmax / dk + 1);
    const std::vector<double> kx = wavenumbers(NX, cfg.lx), ky = wavenumbers(NY, cfg.ly), kz = wavenumbers(NZ, cfg.lz);
    const double pertpeak = 6.0, pertband = 20.0, pertrms = 1.0;
    std::vector<double> energy(nbins);
    std::vector<int> S(nbins, 0);
    for (int i = 0; i < nbins; ++i) {
        const double kv = i * dk;
        const double num = kv - pertpeak * dk;
        const double den = 2.0 * pertband * dk;
        energy[i] = std::exp(-num * num / (den * den));
    }
    double ke = 0.0;
    for (int i = 0; i < nbins; ++i) ke = ke + energy[i];
    const double rms = std::sqrt(2.0 * ke / 3.0);
    for (int i = 0; i < nbins; ++i) energy[i] = energy[i] * (pertrms * pertrms) / (rms * rms);
    for (int i = 0; i < NX; ++i)
        for (int j = 0; j < NY; ++j)
            for (int k = 0; k < NZ2; ++k) {
                const double ksq = std::sqrt(kx[i] * kx[i] + ky[j] * ky[j] + kz[k] * kz[k]);
                if (ksq < kmax) S[(int)(ksq / dk + 0.5)] += 1;
            }
    const size_t nspec = (size_t)NX * NY * NZ2;
    for (int q = 0; q < 3; ++q) A[q].assign(nspec, Cpx{0.0, 0.0});
    LibcRand g(seed);
    double val[2];
    for (int i = 0; i < NX; i++)
        for (int j = 0; j < NY; j++)
            for (int k = 0; k < NZ2; k++) {
                const size_t idx = k + (size_t)i * NZ2 + (size_t)j * NX * NZ2;
                const double ksq = std::sqrt(kx[i] * kx[i] + ky[j] * ky[j] + kz[k] * kz[k]);
                if (ksq < kmax) {
                    const int bin = (int)(ksq / dk + 0.5);
                    const double sigma = std::sqrt(energy[bin] / (2.0 * S[bin] * ksq * ksq));
                    for (int q = 0; q < 3; ++q) {
                        random_normal(g, val, 0.0, sigma);
                        A[q][idx].x = -val[1];
                        A[q][idx].y = val[0];
                    }
                }
                if (i == 0 && j == 0 && k == 0)
                    for (int q = 0; q < 3; ++q) A[q][idx] = Cpx{0.0, 0.0};
            }
    // solenoidal field: i k x A (initialize.cu:458-479)
    for (int i = 0; i < NX; i++)
        for (int j = 0; j < NY; j++)
            for (int k = 0; k < NZ2; k++) {
                const size_t idx = k + (size_t)i * NZ2 + (size_t)j * NX * NZ2;
                const double a1x = A[0][idx].x, a1y = A[0][idx].y;
                const double a2x = A[1][idx].x, a2y = A[1][idx].y;
                const double a3x = A[2][idx].x, a3y = A[2][idx].y;
                A[0][idx].x = -(ky[j] * a3y - kz[k] * a2y);
                A[0][idx].y = ky[j] * a3x - kz[k] * a2x;
                A[1][idx].x = -(kz[k] * a1y - kx[i] * a3y);
                A[1][idx].y = kz[k] * a1x - kx[i] * a3x;
                A[2][idx].x = -(kx[i] * a2y - ky[j] * a1y);
                A[2][idx].y = kx[i] * a2x - ky[j] * a1x;
            }
    // conjugate symmetry on the kz = 0 plane (initialize.cu:481-541), in the reference's order
    auto mirror = [&](int i, int j, int ip, int jp) {
        const size_t idx = (size_t)i * NZ2 + (size_t)j * NX * NZ2;
        const size_t idxp = (size_t)ip * NZ2 + (size_t)jp * NX * NZ2;
        for (int q = 0; q < 3; ++q) A[q][idx] = Cpx{A[q][idxp].x, -A[q][idxp].y};
    };
    for (int i = NX / 2 + 1; i < NX; i++)
        for (int j = NY / 2 + 1; j < NY; j++) mirror(i, j, NX - i, NY - j);
    for (int i = NX / 2 + 1; i < NX; i++)
        for (int j = 1; j < NY / 2; j++) mirror(i, j, NX - i, NY - j);
    for (int i = NX / 2 + 1; i < NX; i++) mirror(i, 0, NX - i, 0);
    for (int j = NY / 2 + 1; j < NY; j++) mirror(0, j, 0, NY - j);
    // scale by NN to counteract the inverse transform's 1/NN (initialize.cu:575-585)
    for (int q = 0; q < 3; ++q)
        for (Cpx &a : A[q]) a = Cpx{a.x * NN, a.y * NN};
}

template <typename T> struct V2of;
template <> struct V2of<double> { using type = double2; };
template <> struct V2of<float> { using type = float2; };

// jet, scalar and noise superposition on the physical padded layout (the
// reference's kernels: initialize.cu:114-142, 160-194, 249-264)
template <typename T>
__global__ void k_jet_ic(T *u, T *v, T *w, T *s, T *c, int nx, int ny, int nz, double ly, double H, double theta,
                         double theta_c, double scale) {
    const long long npts = (long long)nx * ny * nz;
    const int nz2 = nz / 2 + 1;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < npts;
         p += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(p % nz);
        const long long line = p / nz;
        const int j = (int)(line % ny);
        const long long idx = line * 2 * nz2 + k;
        const double y = -(double)ly / 2 + j * (double)ly / ny;
        const double prof = 0.5 - 0.5 * tanh(H / (4.0 * theta) * (2.0 * fabs(y) / H - 1.0));
        u[idx] = (T)(prof + scale * (double)u[idx]);
        v[idx] = (T)(0.0 + scale * (double)v[idx]);
        w[idx] = (T)(0.0 + scale * (double)w[idx]);
        s[idx] = (T)prof;
        if (c) c[idx] = (T)(0.5 - 0.5 * tanh(H / (4.0 * theta_c) * (2.0 * fabs(y) / H - 1.0)));
        if (k == 0) {   // the two padding reals of the line
            const long long pad = line * 2 * nz2 + nz;
            for (int q = 0; q < 2 * nz2 - nz; ++q) {
                u[pad + q] = v[pad + q] = w[pad + q] = s[pad + q] = T(0);
                if (c) c[pad + q] = T(0);
            }
        }
    }
}

template <typename T>
gnss_status initial_jet_t(gnss_ctx *ctx, const gnss_config &cfg, const gnss_jet_params *p, const gnss_fields *st,
                          cudaStream_t s) {
    using V = typename V2of<T>::type;
    std::vector<Cpx> A[3];
    generate_noise(cfg, p->seed ? p->seed : 666 * 37 + 37 * 13, A);
    const size_t nspec = A[0].size();
    void *f[3] = {st->u, st->v, st->w};
    std::vector<V> h(nspec);
    for (int q = 0; q < 3; ++q) {
        for (size_t i = 0; i < nspec; ++i) h[i] = V{(T)A[q][i].x, (T)A[q][i].y};
        if (cudaMemcpyAsync(f[q], h.data(), nspec * sizeof(V), cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return GNSS_ERR_CUDA;
        gnss_status e = gnss_inverse(ctx, f[q], s);   // physical noise (generateNoise, initialize.cu:605-608)
        if (e) return e;
    }
    const long long npts = (long long)cfg.nx * cfg.ny * cfg.nz;
    const int blocks = (int)std::min<long long>((npts + 255) / 256, 148LL * 16);
    k_jet_ic<T><<<blocks, 256, 0, s>>>((T *)st->u, (T *)st->v, (T *)st->w, (T *)st->s, (T *)st->c, cfg.nx, cfg.ny,
                                       cfg.nz, cfg.ly, p->h, p->theta, p->theta_c, p->pert_amp);
    if (cudaGetLastError() != cudaSuccess) return GNSS_ERR_CUDA;
    void *all[5] = {st->u, st->v, st->w, st->s, st->c};
    for (int q = 0; q < 5; ++q) {
        if (!all[q]) continue;
        gnss_status e = gnss_forward(ctx, all[q], s);   // main.cu:149-153
        if (!e) e = gnss_dealias(ctx, all[q], s);       // main.cu:156
        if (e) return e;
    }
    return cudaStreamSynchronize(s) == cudaSuccess ? GNSS_OK : GNSS_ERR_CUDA;
}

}  // namespace

gnss_status gnss_initial_jet(gnss_ctx *ctx, const gnss_jet_params *p, const gnss_fields *state, void *stream) {
    gnss_config cfg;
    if (!ctx || !p || !state || gnss_get_config(ctx, &cfg)) return GNSS_ERR_INVALID;
    if (!state->u || !state->v || !state->w || !state->s || (cfg.n_scalars == 2 && !state->c)) return GNSS_ERR_INVALID;
    if (!(p->h > 0 && p->theta > 0 && p->theta_c > 0)) return GNSS_ERR_INVALID;
    if (cudaSetDevice(cfg.device) != cudaSuccess) return GNSS_ERR_CUDA;
    gnss_fields f = *state;
    if (cfg.n_scalars == 1) f.c = nullptr;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    return cfg.precision == GNSS_FP64 ? initial_jet_t<double>(ctx, cfg, p, &f, s)
                                      : initial_jet_t<float>(ctx, cfg, p, &f, s);
}
