/*
 * oracle.h -- CPU FP64 restatement of the reference pseudospectral step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg (and the
 * CPU reference arm) may load it.  It is never part of the product path.
 *
 * Parity pinning: checked against numpy/pocketfft transforms, analytic
 * known-answer cases (single Fourier modes, Taylor-Green decay, scalar
 * diffusion) and against golden outputs of the reference's own CUDA code
 * (tests/golden/, produced by oracle/refdriver.cu built from the reference
 * sources by oracle/build_ref.sh).
 *
 * Layouts follow the reference exactly:
 *   physical real field  f[x][y][2*nz2]   index z + 2*nz2*(y + ny*x)   (cudafuncs.cu:14-17)
 *   spectral field       F[y][x][nz2]     index kz + nz2*(x + nx*y)    (solver.cu:25, fftfuncs.cu:315)
 * Both occupy nx*ny*nz2 complex doubles; transforms are in place on that buffer.
 */
#ifndef GNSS_ORACLE_H
#define GNSS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_cfg {
    int nx, ny, nz;         /* grid; each size 2^a 3^b, even                         */
    double lx, ly, lz;      /* box lengths                                            */
    double re;              /* velocity diffusivity 1/re  (solver.cu:599-603)        */
    double sc;              /* scalar s diffusivity 1/(re*sc) (solver.cu:604)         */
    double sc_c;            /* scalar c diffusivity 1/(re*sc_c) (solver.cu:605)       */
    double alpha;           /* drift coefficient of c (solver.cu:374-388)            */
    double dt;              /* time step                                              */
    double alias_filter;    /* k_max = alias_filter*nx*pi/lx (solver.cu:29-36)        */
    double nu_stats;        /* nu used by the statistics, H/Re (dnsparams.h:30)       */
    int nthreads;           /* OpenMP threads (0 = default)                           */
} orc_cfg;

/* 3D transforms, in place (fftfuncs.cu:288-359). forward is unnormalised,
 * inverse includes the 1/(nx*ny*nz) scale (cudafuncs.cu:20-31). */
int orc_forward(const orc_cfg *c, double *f);
int orc_inverse(const orc_cfg *c, double *f);

/* spectral operators (solver.cu) on fields of nx*ny*nz2 complex */
int orc_dealias(const orc_cfg *c, double *fh);                                  /* solver.cu:17-42   */
int orc_vorticity(const orc_cfg *c, const double *uh, const double *vh, const double *wh,
                  double *o1, double *o2, double *o3);                             /* solver.cu:68-114  */
int orc_gradient(const orc_cfg *c, const double *fh, double *fx, double *fy, double *fz); /* :233-256 */
int orc_make_rhs(const orc_cfg *c, double *ru, double *rv, double *rw, double *rs, double *rc); /* :461-521 */

/* One reference time step (solver_ps, solver.cu:700-765): fields[5] = uh,vh,wh,sh,ch
 * (spectral, in place), rhs_old[5] the Adams-Bashforth history.  euler=1 on the
 * first step (main.cu:181-186).  Scratch is allocated internally. */
int orc_step_cnab2(const orc_cfg *c, double **fields, double **rhs_old, int euler);

/* One step of the integrating-factor low-storage RK3 scheme (Wray coefficients).
 * fields[nf] spectral state, hist[nf] the RK history; nf = 3 + n_scalars. */
int orc_step_rk3if(const orc_cfg *c, double **fields, double **hist, int n_scalars);

/* Spectral statistics (statistics.cu:1494-1845): out[0]=KE, out[1]=Vrms^2 (sum/3),
 * out[2]=epsilon, out[3]=chi_s, out[4]=chi_c, out[5]=var_s, out[6]=var_c. */
int orc_stats(const orc_cfg *c, double **fields, double *out);

/* Turbulence statistics of calcTurbStats_mgpu (statistics.cu:2039-2156):
 * out[0]=Vrms, [1]=KE, [2]=epsilon, [3]=eta, [4]=l, [5]=lambda, [6]=chi,
 * [7]=omega (mean |vorticity|), [8..10]=rms of the vorticity components;
 * yprof (may be NULL): 5 x ny mean profiles along y of fields[0..4]
 * (zero for a NULL field). */
int orc_turb_stats(const orc_cfg *c, double **fields, double *out, double *yprof);

/* plain batched complex FFT for unit tests: data [n][batch] interleaved complex */
int orc_fft_c2c(int n, int batch, double *data, int sign);

#ifdef __cplusplus
}
#endif
#endif
