/*
 * refdriver.cu -- this project's driver around the reference's own CUDA step.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/build_ref.sh compiles it together with the
 * unmodified reference sources (solver.cu, fftfuncs.cu, cudafuncs.cu,
 * allocate.cu, initialize.cu, iofuncs.cu, statistics.cu) and a generated
 * dnsparams.h for one grid configuration.  It replaces the reference's
 * main.cu (main.cu:84-252), which hard-codes its initial condition, file
 * output paths and loop length.
 *
 *   refdrv run  <state_in.bin> <nsteps> <out_dir> [dump_steps,...]
 *       Loads a spectral state (5 fields u,v,w,s,c, complex128 [NY][NX][NZ2]),
 *       dealiases it (main.cu:156) and calls solver_ps nsteps times with
 *       euler = (c == 1) (main.cu:181-189).  Writes out_dir/stats.bin
 *       ((nsteps+1) x 7 doubles) and out_dir/state_<c>.bin, rhsold_<c>.bin.
 *   refdrv time <nsteps> <warmup>
 *       Builds the reference jet profile (initialize.cu:114-212), transforms
 *       and dealiases it (main.cu:149-156), then times nsteps solver_ps calls
 *       with CUDA events on the legacy stream; prints one JSON line.
 *
 * The statistics here are computed by this driver's own reduction (the
 * reference definitions of statistics.cu:1494-1845: KE, u'^2, epsilon, chi,
 * plus scalar variances), so that no reference statistics kernel runs.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <sys/stat.h>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include <cufft.h>

#include "dnsparams.h"
#include "struct_def.h"
#include "declare.h"
#include "allocate.h"
#include "cudafuncs.h"
#include "fftfuncs.h"
#include "solver.h"
#include "initialize.h"

// generateNoise (initialize.cu:388-390) takes its work arrays from malloc and
// assigns only the modes with |k| < kmax; the rest (the Nyquist planes among
// them) is read uninitialized, so its initial condition depends on whatever
// the heap held (NaN in practice when the arrays come from reused heap
// memory).  The driver zero-fills every heap allocation of the program, which
// makes those modes zero, as they are when the arrays come from fresh pages.
extern "C" void *__libc_calloc(size_t, size_t) noexcept;
extern "C" void *malloc(size_t n) noexcept { return __libc_calloc(1, n); }

#define DRV_CHECK(x)                                                                        \
    do {                                                                                    \
        cudaError_t e_ = (x);                                                               \
        if (e_ != cudaSuccess) {                                                            \
            std::fprintf(stderr, "refdrv: CUDA error %s at %s:%d\n", cudaGetErrorString(e_), \
                         __FILE__, __LINE__);                                               \
            std::exit(2);                                                                   \
        }                                                                                   \
    } while (0)

static const size_t NSPEC = (size_t)NX * NY * NZ2;

/* one GPU, the whole grid: what splitData (main.cu:31-82) produces for nGPUs = 1 */
static void drv_split(gpudata *g) {
    g->nGPUs = 1;
    DRV_CHECK(cudaHostAlloc((void **)&g->gpunum, sizeof(int), cudaHostAllocMapped));
    DRV_CHECK(cudaHostAlloc((void **)&g->ny, sizeof(int), cudaHostAllocMapped));
    DRV_CHECK(cudaHostAlloc((void **)&g->nx, sizeof(int), cudaHostAllocMapped));
    DRV_CHECK(cudaHostAlloc((void **)&g->start_y, sizeof(int), cudaHostAllocMapped));
    DRV_CHECK(cudaHostAlloc((void **)&g->start_x, sizeof(int), cudaHostAllocMapped));
    g->gpunum[0] = 0;
    g->nx[0] = NX; g->start_x[0] = 0;
    g->ny[0] = NY; g->start_y[0] = 0;
}

/* per-block partial sums: [0] sum w|u|^2, [1] sum w k^2|u|^2, [2] sum w k^2|s|^2,
 * [3] sum w k^2|c|^2, [4] sum_{k!=0} w|s|^2, [5] sum_{k!=0} w|c|^2 ; w = kz mirror weight */
__global__ void drv_stats_kernel(const double2 *u, const double2 *v, const double2 *w, const double2 *s,
                                 const double2 *c, const double *k1, const double *k2, const double *k3,
                                 double *partial) {
    __shared__ double red[6][256];
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < NSPEC;
         idx += (size_t)gridDim.x * blockDim.x) {
        int k = (int)(idx % NZ2);
        int i = (int)((idx / NZ2) % NX);
        int j = (int)(idx / ((size_t)NZ2 * NX));
        double wt = (k == 0 || 2 * k == NZ) ? 1.0 : 2.0;
        double ksq = k1[i] * k1[i] + k2[j] * k2[j] + k3[k] * k3[k];
        double e = u[idx].x * u[idx].x + u[idx].y * u[idx].y + v[idx].x * v[idx].x + v[idx].y * v[idx].y +
                   w[idx].x * w[idx].x + w[idx].y * w[idx].y;
        double ms = s[idx].x * s[idx].x + s[idx].y * s[idx].y;
        double mc = c[idx].x * c[idx].x + c[idx].y * c[idx].y;
        bool k0 = (idx == 0);
        acc[0] += wt * e;
        acc[1] += wt * ksq * e;
        acc[2] += wt * ksq * ms;
        acc[3] += wt * ksq * mc;
        if (!k0) { acc[4] += wt * ms; acc[5] += wt * mc; }
    }
    for (int q = 0; q < 6; ++q) red[q][threadIdx.x] = acc[q];
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st)
            for (int q = 0; q < 6; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 6; ++q) partial[blockIdx.x * 6 + q] = red[q][0];
}

static void drv_stats(double *out7) {
    const int nb = 592;
    static double *d_part = nullptr;
    if (!d_part) DRV_CHECK(cudaMalloc(&d_part, sizeof(double) * nb * 6));
    drv_stats_kernel<<<nb, 256>>>(vel.uh[0], vel.vh[0], vel.wh[0], vel.sh[0], vel.ch[0], grid.kx[0], grid.ky[0],
                                  grid.kz[0], d_part);
    DRV_CHECK(cudaGetLastError());
    std::vector<double> h(nb * 6);
    DRV_CHECK(cudaMemcpy(h.data(), d_part, sizeof(double) * nb * 6, cudaMemcpyDeviceToHost));
    long double s[6] = {0, 0, 0, 0, 0, 0};
    for (int b = 0; b < nb; ++b)
        for (int q = 0; q < 6; ++q) s[q] += h[b * 6 + q];
    const double n2 = (double)NN * (double)NN;
    out7[0] = (double)(s[0] / n2) / 2.0;                 /* KE    statistics.cu:1549 */
    out7[1] = (double)(s[0] / n2) / 3.0;                 /* u'^2  statistics.cu:1551 */
    out7[2] = nu * (double)(s[1] / n2);                  /* eps   statistics.cu:1637 */
    out7[3] = 2.0 * (nu / Sc) * (double)(s[2] / n2);     /* chi   statistics.cu:1813 */
    out7[4] = 2.0 * (nu / Sc_c) * (double)(s[3] / n2);
    out7[5] = (double)(s[4] / n2);
    out7[6] = (double)(s[5] / n2);
}

static void setup() {
    drv_split(&gpu);
    allocate_memory();                       /* allocate.cu:9-224 */
    plan1dFFT(gpu.nGPUs, fft);               /* fftfuncs.cu:204 */
    plan2dFFT(gpu, fft);                     /* fftfuncs.cu:133 */
    initializeWaveNumbers(gpu, grid);        /* initialize.cu:693 */
    DRV_CHECK(cudaDeviceSynchronize());
}

static cufftDoubleComplex *field_ptr(fielddata f, int q) {
    cufftDoubleComplex **p[5] = {f.uh, f.vh, f.wh, f.sh, f.ch};
    return p[q][0];
}

static void dump(const std::string &path, fielddata f) {
    std::vector<double2> h(NSPEC);
    FILE *fp = std::fopen(path.c_str(), "wb");
    if (!fp) { std::perror(path.c_str()); std::exit(3); }
    for (int q = 0; q < 5; ++q) {
        DRV_CHECK(cudaMemcpy(h.data(), field_ptr(f, q), sizeof(double2) * NSPEC, cudaMemcpyDeviceToHost));
        std::fwrite(h.data(), sizeof(double2), NSPEC, fp);
    }
    std::fclose(fp);
}

static int run(int argc, char **argv) {
    if (argc < 5) { std::fprintf(stderr, "usage: refdrv run <state_in> <nsteps> <out_dir> [dumps]\n"); return 1; }
    const char *in = argv[2];
    int nsteps = std::atoi(argv[3]);
    std::string out = argv[4];
    std::vector<int> dumps;
    if (argc > 5) {
        char *s = argv[5];
        for (char *t = std::strtok(s, ","); t; t = std::strtok(nullptr, ",")) dumps.push_back(std::atoi(t));
    }
    setup();
    {
        FILE *fp = std::fopen(in, "rb");
        if (!fp) { std::perror(in); return 3; }
        std::vector<double2> h(NSPEC);
        for (int q = 0; q < 5; ++q) {
            if (std::fread(h.data(), sizeof(double2), NSPEC, fp) != NSPEC) {
                std::fprintf(stderr, "refdrv: short state file %s\n", in);
                return 3;
            }
            DRV_CHECK(cudaMemcpy(field_ptr(vel, q), h.data(), sizeof(double2) * NSPEC, cudaMemcpyHostToDevice));
        }
        std::fclose(fp);
    }
    deAlias(gpu, grid, vel);                 /* main.cu:156 */
    DRV_CHECK(cudaDeviceSynchronize());
    std::vector<double> st((size_t)(nsteps + 1) * 7);
    drv_stats(&st[0]);
    for (int c = 1; c <= nsteps; ++c) {
        int euler = (c == 1) ? 1 : 0;        /* main.cu:181-186 */
        solver_ps(euler, fft, gpu, grid, vel, rhs, rhs_old, temp);
        DRV_CHECK(cudaDeviceSynchronize());
        drv_stats(&st[(size_t)c * 7]);
        for (int d : dumps)
            if (d == c) {
                dump(out + "/state_" + std::to_string(c) + ".bin", vel);
                dump(out + "/rhsold_" + std::to_string(c) + ".bin", rhs_old);
            }
    }
    FILE *fp = std::fopen((out + "/stats.bin").c_str(), "wb");
    if (!fp) { std::perror("stats.bin"); return 3; }
    std::fwrite(st.data(), sizeof(double), st.size(), fp);
    std::fclose(fp);
    std::printf("{\"n\": %d, \"steps\": %d, \"ke_final\": %.17g}\n", NX, nsteps, st[(size_t)nsteps * 7]);
    return 0;
}

static int timeit(int argc, char **argv) {
    int nsteps = argc > 2 ? std::atoi(argv[2]) : 5;
    int warmup = argc > 3 ? std::atoi(argv[3]) : 2;
    setup();
    initializeVelocity(gpu, vel);            /* initialize.cu:144 */
    initializeScalar(gpu, vel);              /* initialize.cu:196 */
    forwardTransform(fft, gpu, vel.u);       /* main.cu:149-153 */
    forwardTransform(fft, gpu, vel.v);
    forwardTransform(fft, gpu, vel.w);
    forwardTransform(fft, gpu, vel.s);
    forwardTransform(fft, gpu, vel.c);
    deAlias(gpu, grid, vel);                 /* main.cu:156 */
    DRV_CHECK(cudaDeviceSynchronize());
    int c = 1;
    for (int w = 0; w < warmup; ++w, ++c) solver_ps(c == 1, fft, gpu, grid, vel, rhs, rhs_old, temp);
    DRV_CHECK(cudaDeviceSynchronize());
    cudaEvent_t e0, e1;
    DRV_CHECK(cudaEventCreate(&e0));
    DRV_CHECK(cudaEventCreate(&e1));
    std::vector<float> per(nsteps);
    DRV_CHECK(cudaEventRecord(e0, 0));
    for (int s = 0; s < nsteps; ++s, ++c) solver_ps(c == 1, fft, gpu, grid, vel, rhs, rhs_old, temp);
    DRV_CHECK(cudaEventRecord(e1, 0));
    DRV_CHECK(cudaEventSynchronize(e1));
    float ms = 0.f;
    DRV_CHECK(cudaEventElapsedTime(&ms, e0, e1));
    double st[7];
    drv_stats(st);
    std::printf("{\"n\": %d, \"steps\": %d, \"ms_total\": %.6f, \"ms_per_step\": %.6f, \"ke\": %.17g}\n", NX, nsteps,
                (double)ms, (double)ms / nsteps, st[0]);
    return 0;
}

// The reference's file writers (iofuncs.cu:78-260, 329-358), declared here as
// they are defined there (iofuncs.h declares only some of them).
void writeYprofs(const int c, const char *name, double *data);
void writeStats(const int c, const char *name, double in);
void writexyfields(gpudata gpu, const int iter, const char var, double **in, const int zplane);
void writexzfields(gpudata gpu, const int iter, const char var, double **in, const int yplane);
void writeyzfields(gpudata gpu, const int iter, const char var, double **in, const int xplane);
void write3Dfields_mgpu(gpudata gpu, const int iter, const char var, double **in);

// refdrv io: runs the reference's writers on a synthetic physical field, in
// the current directory (rootdir "./", sim_name "refdrv/"): refdrv/u.3,
// refdrv/vis/u_{xy,xz,yz}.3 (planes z = 2, y = 1, x = 4), refdrv/stats/KE
// (three records), refdrv/Yprofs/u_mean.3; the input goes to refdrv/input.bin
// (the padded array [NX][NY][2 NZ2], padding -1) and refdrv/prof.bin.  Host
// code only: no CUDA call is made.
static int io_mode() {
    const size_t n = (size_t)NX * NY * 2 * NZ2;
    std::vector<double> f(n, -1.0);
    for (int i = 0; i < NX; ++i)
        for (int j = 0; j < NY; ++j)
            for (int k = 0; k < NZ; ++k)
                f[k + 2 * NZ2 * (j + NY * (size_t)i)] = i + 0.01 * j + 1e-4 * k + 0.5 * std::sin(0.3 * i + 0.7 * j + 1.1 * k);
    std::vector<double> prof(NY);
    for (int j = 0; j < NY; ++j) prof[j] = 0.25 * j - 1.0 / (j + 1);
    int nx[1] = {NX};
    gpudata g{};
    g.nGPUs = 1;
    g.nx = nx;
    double *in[1] = {f.data()};
    mkdir("refdrv", 0700);
    mkdir("refdrv/vis", 0700);
    mkdir("refdrv/stats", 0700);
    mkdir("refdrv/Yprofs", 0700);
    write3Dfields_mgpu(g, 3, 'u', in);
    writexyfields(g, 3, 'u', in, 2);
    writexzfields(g, 3, 'u', in, 1);
    writeyzfields(g, 3, 'u', in, 4);
    writeStats(0, "KE", 1.5);
    writeStats(1, "KE", 2.5);
    writeStats(2, "KE", -0.125);
    writeYprofs(3, "u_mean", prof.data());
    FILE *fp = std::fopen("refdrv/input.bin", "wb");
    std::fwrite(f.data(), sizeof(double), n, fp);
    std::fclose(fp);
    fp = std::fopen("refdrv/prof.bin", "wb");
    std::fwrite(prof.data(), sizeof(double), NY, fp);
    std::fclose(fp);
    return 0;
}

// refdrv ic <out_dir>: the reference's initial condition as main.cu builds it
// (initializeJet, main.cu:139; forward transforms, :149-153; deAlias, :156),
// dumped as <out_dir>/ic.bin (the 5 spectral fields).
static int ic_mode(int argc, char **argv) {
    if (argc < 3) { std::fprintf(stderr, "usage: refdrv ic <out_dir>\n"); return 1; }
    std::string out = argv[2];
    setup();
    initializeJet(fft, gpu, grid, h_vel, vel, rhs);
    forwardTransform(fft, gpu, vel.u);
    forwardTransform(fft, gpu, vel.v);
    forwardTransform(fft, gpu, vel.w);
    forwardTransform(fft, gpu, vel.s);
    forwardTransform(fft, gpu, vel.c);
    deAlias(gpu, grid, vel);
    DRV_CHECK(cudaDeviceSynchronize());
    dump(out + "/ic.bin", vel);
    return 0;
}

int main(int argc, char **argv) {
    if (argc >= 2 && std::strcmp(argv[1], "run") == 0) return run(argc, argv);
    if (argc >= 2 && std::strcmp(argv[1], "ic") == 0) return ic_mode(argc, argv);
    if (argc >= 2 && std::strcmp(argv[1], "time") == 0) return timeit(argc, argv);
    if (argc >= 2 && std::strcmp(argv[1], "io") == 0) return io_mode();
    std::fprintf(stderr, "usage: refdrv run|time|io|ic ...\n");
    return 1;
}
