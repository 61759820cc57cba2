// refabi.cu -- the reference's own host API, implemented on the B200 library.
//
// A drop-in replacement for the reference's solver.o and fftfuncs.o: it
// exports the same C++ symbols with the same signatures and in-place
// semantics (transposed spectral layout, 1/N^3 on the inverse transform,
// legacy default stream), so the rest of a reference program (main.o,
// statistics.o, initialize.o, iofuncs.o, allocate.o, cudafuncs.o) links
// against it unchanged.  It is compiled inside that program's build, against
// its struct_def.h and dnsparams.h (compile-time sizes and parameters):
//
//   nvcc -std=c++17 -rdc=true -c refabi.cu -I<reference dir> -I<repo>/include
//
// and linked with -lgnss_b200.  One context is created on the first call
// (plan1dFFT/plan2dFFT or any operator) from the dnsparams.h macros; it
// carries both scalars s and c like the reference.  Errors are fatal, as with
// the reference's checkCudaErrors (which exits).  Only nGPUs == 1 is served.
//
// Symbols provided (reference file:line of the function replaced):
//   plan1dFFT fftfuncs.cu:204   plan2dFFT fftfuncs.cu:133   plan3dFFT fftfuncs.cu:233
//   forwardTransform fftfuncs.cu:288   inverseTransform fftfuncs.cu:322
//   deAlias solver.cu:44   vorticity solver.cu:116   gradient solver.cu:258
//   divergence solver.cu:292   crossProduct solver.cu:166   dotProduct solver.cu:358
//   colloidAdvection solver.cu:390   scalarAdvection solver.cu:407   makeRHS solver.cu:523
//   timestep solver.cu:587   update solver.cu:639   solver_ps solver.cu:700
#include <cstdio>
#include <cstdlib>

// the library header first: dnsparams.h defines macros (dt, alpha, ...) that
// collide with field names of gnss_config
#include "gnss_b200.h"

#include <cuda_runtime.h>
#include <cufft.h>

#include "dnsparams.h"
#include "struct_def.h"

static gnss_ctx *g_ctx = nullptr;

static void die(const char *what, gnss_status st) {
    std::fprintf(stderr, "gnss refabi: %s failed: %s (%s)\n", what, gnss_status_string(st),
                 g_ctx ? gnss_last_error(g_ctx) : "");
    std::exit(1);
}

#define REFABI_CALL(what, expr)                 \
    do {                                        \
        gnss_status st_ = (expr);               \
        if (st_ != GNSS_OK) die(what, st_);     \
    } while (0)

static gnss_ctx *ctx() {
    if (g_ctx) return g_ctx;
    int dev = 0;
    cudaGetDevice(&dev);
    // positional: nx, ny, nz, lx, ly, lz, re, sc, sc_c, alpha, dt, alias_filter,
    // nu_stats, n_scalars, scheme, precision, device
    const gnss_config cfg = {NX,  NY,       NZ,         LX,           LY, LZ, (double)Re, (double)Sc, (double)Sc_c,
                             (double)alpha, (double)dt, (double)alias_filter, (double)nu, 2, GNSS_SCHEME_CNAB2,
                             GNSS_FP64,     dev};
    REFABI_CALL("gnss_create", gnss_create(&cfg, &g_ctx));
    return g_ctx;
}

static void one_gpu(const gpudata &gpu) {
    if (gpu.nGPUs != 1) {
        std::fprintf(stderr, "gnss refabi: only nGPUs == 1 is supported (got %d)\n", gpu.nGPUs);
        std::exit(1);
    }
}

static gnss_fields fields_of(const fielddata &f) {
    gnss_fields g = {f.uh[0], f.vh[0], f.wh[0], f.sh[0], f.ch[0]};
    return g;
}

// ------------------------------------------------------------ fftfuncs.cu
void plan1dFFT(int nGPUs, fftdata fft) {
    (void)fft;
    if (nGPUs != 1) {
        std::fprintf(stderr, "gnss refabi: only nGPUs == 1 is supported\n");
        std::exit(1);
    }
    ctx();
}
void plan2dFFT(gpudata gpu, fftdata fft) {
    (void)fft;
    one_gpu(gpu);
    ctx();
}
void plan3dFFT(fftdata fft) {
    (void)fft;
    ctx();
}
void forwardTransform(fftdata fft, gpudata gpu, cufftDoubleReal **f) {
    (void)fft;
    one_gpu(gpu);
    REFABI_CALL("forwardTransform", gnss_forward(ctx(), f[0], nullptr));
}
void inverseTransform(fftdata fft, gpudata gpu, cufftDoubleComplex **f) {
    (void)fft;
    one_gpu(gpu);
    REFABI_CALL("inverseTransform", gnss_inverse(ctx(), f[0], nullptr));
}

// ------------------------------------------------------------ solver.cu
void deAlias(gpudata gpu, griddata grid, fielddata vel) {
    (void)grid;
    one_gpu(gpu);
    cufftDoubleComplex *f[5] = {vel.uh[0], vel.vh[0], vel.wh[0], vel.sh[0], vel.ch[0]};
    for (int q = 0; q < 5; ++q) REFABI_CALL("deAlias", gnss_dealias(ctx(), f[q], nullptr));
}

void vorticity(gpudata gpu, griddata grid, fielddata vel, fielddata rhs) {
    (void)grid;
    one_gpu(gpu);
    REFABI_CALL("vorticity", gnss_vorticity(ctx(), vel.uh[0], vel.vh[0], vel.wh[0], rhs.uh[0], rhs.vh[0],
                                            rhs.wh[0], nullptr));
}

void gradient(gpudata gpu, griddata grid, cufftDoubleComplex **f, fielddata grad) {
    (void)grid;
    one_gpu(gpu);
    REFABI_CALL("gradient", gnss_gradient(ctx(), f[0], grad.uh[0], grad.vh[0], grad.wh[0], nullptr));
}

void divergence(gpudata gpu, griddata grid, fielddata f, cufftDoubleComplex **result) {
    (void)grid;
    one_gpu(gpu);
    REFABI_CALL("divergence", gnss_divergence(ctx(), f.uh[0], f.vh[0], f.wh[0], result[0], nullptr));
}

void crossProduct(gpudata gpu, fielddata vel, fielddata rhs) {
    one_gpu(gpu);
    REFABI_CALL("crossProduct", gnss_cross_product(ctx(), vel.u[0], vel.v[0], vel.w[0], rhs.u[0], rhs.v[0],
                                                   rhs.w[0], nullptr));
    cudaDeviceSynchronize();   // as solver.cu:179
}

void dotProduct(gpudata gpu, fielddata a, fielddata b, cufftDoubleReal **result) {
    one_gpu(gpu);
    REFABI_CALL("dotProduct", gnss_dot_product(ctx(), a.u[0], a.v[0], a.w[0], b.u[0], b.v[0], b.w[0], result[0],
                                               nullptr));
}

void colloidAdvection(gpudata gpu, fielddata vel, fielddata gradC, fielddata Vdp, cufftDoubleReal **divVdp) {
    one_gpu(gpu);
    REFABI_CALL("colloidAdvection",
                gnss_colloid_advection(ctx(), vel.u[0], vel.v[0], vel.w[0], vel.c[0], gradC.u[0], gradC.v[0],
                                       gradC.w[0], Vdp.u[0], Vdp.v[0], Vdp.w[0], divVdp[0], nullptr));
}

// the reference sequence of solver.cu:407-459 on the library's operators
void scalarAdvection(fftdata fft, gpudata gpu, griddata grid, fielddata vel, fielddata rhs, fielddata temp) {
    one_gpu(gpu);
    const size_t bytes = gnss_field_bytes(ctx());
    if (cudaMemset(rhs.s[0], 0, bytes) != cudaSuccess || cudaMemset(rhs.c[0], 0, bytes) != cudaSuccess)
        die("scalarAdvection memset", GNSS_ERR_CUDA);
    gradient(gpu, grid, vel.sh, rhs);
    divergence(gpu, grid, rhs, rhs.ch);
    inverseTransform(fft, gpu, rhs.uh);
    inverseTransform(fft, gpu, rhs.vh);
    inverseTransform(fft, gpu, rhs.wh);
    dotProduct(gpu, vel, rhs, rhs.s);
    gradient(gpu, grid, vel.ch, temp);
    inverseTransform(fft, gpu, temp.uh);
    inverseTransform(fft, gpu, temp.vh);
    inverseTransform(fft, gpu, temp.wh);
    inverseTransform(fft, gpu, rhs.ch);
    inverseTransform(fft, gpu, vel.ch);
    colloidAdvection(gpu, vel, temp, rhs, rhs.c);
}

void makeRHS(gpudata gpu, griddata grid, fielddata rhs) {
    (void)grid;
    one_gpu(gpu);
    REFABI_CALL("makeRHS", gnss_make_rhs(ctx(), rhs.uh[0], rhs.vh[0], rhs.wh[0], rhs.sh[0], rhs.ch[0], nullptr));
}

void timestep(const int flag, gpudata gpu, griddata grid, fielddata vel, fielddata rhs, fielddata rhs_old) {
    (void)grid;
    one_gpu(gpu);
    gnss_fields s = fields_of(vel), r = fields_of(rhs), o = fields_of(rhs_old);
    REFABI_CALL("timestep", gnss_timestep(ctx(), flag, &s, &r, flag ? nullptr : &o, nullptr));
}

void update(gpudata gpu, fielddata rhs, fielddata rhs_old) {
    one_gpu(gpu);
    gnss_fields r = fields_of(rhs), o = fields_of(rhs_old);
    REFABI_CALL("update", gnss_update(ctx(), &r, &o, nullptr));
}

// One time step on the fused B200 path.  Post-conditions as in the reference:
// vel advanced, rhs_old holds this step's right-hand side.  (The reference
// also leaves rhs zeroed and temp holding intermediates; the fused path does
// not touch rhs or temp.)
void solver_ps(const int euler, fftdata fft, gpudata gpu, griddata grid, fielddata vel, fielddata rhs,
               fielddata rhs_old, fielddata temp) {
    (void)fft;
    (void)rhs;
    (void)temp;
    one_gpu(gpu);
    deAlias(gpu, grid, vel);   // solver.cu:704: the reference dealiases the state at every step
    gnss_fields s = fields_of(vel), h = fields_of(rhs_old);
    REFABI_CALL("solver_ps", gnss_step(ctx(), &s, &h, euler, nullptr));
}
