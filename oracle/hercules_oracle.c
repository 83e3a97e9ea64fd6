/*
 * hercules_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * FP64 CPU restatement of the HERCULES time step with single-domain semantics
 * (p_row = p_col = 1, i_offset = j_offset = 0, comm_bound = periodic wrap).
 * Every routine names the reference file:line it restates and keeps the
 * reference's operation order, array shapes (ghosted (nx+4,ny+4,nz+4), x fastest,
 * 1-based Fortran indices through the F() macro) and quirks:
 *   - the wall folds of get_u/w/t_eqn_coeff zero the 1-D aa(k)/cc(k) inside the
 *     (i,j) loop, so only the first local mode (kx=ky=0) receives them
 *     (src/module_poisson_solver.f90:257-273, 361-366, 455-469);
 *   - the signed div_max / div_hist_max of screen_div_error (src/module_io.f90:131-145);
 *   - statistics use the interpolants of the last sub-step's start
 *     (src/module_tools.f90:383-385);
 *   - rayleigh_damping leaves ghost cells stale until the next boundary update;
 *   - rayleigh_damping_spec reduces only the real part of the complex plane mean
 *     (src/module_spectral.f90:1372; the imaginary part is taken as 0 here, the
 *     reference leaves it undefined).
 * The FFT is this file's own mixed-radix DFT with the FFTW sign and
 * normalisation conventions of mpi_2d_fft (src/module_tools.f90:518-700):
 * forward e^{-i}, y lines then x lines, each divided by its length, Nyquist
 * zeroed after the forward and before the backward transform. The reference
 * links FFTW 3.3.4 for that arithmetic; results agree to round-off.
 *
 * Parity status: UNPINNED against reference runs (the Fortran/MPI reference
 * cannot be compiled in this image). Pinned by analytic known-answer tests.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "hercules_oracle.h"

typedef double complex cplx;

/* src/module_parameters.f90:32 */
#define PI 3.1415926535897932

/* ------------------------------------------------------------------------ */
/* FFT: recursive mixed-radix decimation in time                            */
/* ------------------------------------------------------------------------ */
typedef struct {
    int n;
    int nf;
    int f[40];
    cplx* tw[2];      /* [0] sign -1 (forward), [1] sign +1 (backward) */
} fftplan;

static void plan_init(fftplan* pl, int n)
{
    pl->n = n;
    pl->nf = 0;
    int m = n;
    int primes[] = {4, 2, 3, 5, 7};
    for (int pi = 0; pi < 5; ++pi) {
        while (m % primes[pi] == 0) { pl->f[pl->nf++] = primes[pi]; m /= primes[pi]; }
    }
    for (int d = 11; m > 1; d += 2) {
        while (m % d == 0) { pl->f[pl->nf++] = d; m /= d; }
    }
    for (int s = 0; s < 2; ++s) {
        pl->tw[s] = (cplx*)malloc(sizeof(cplx) * (size_t)(n > 0 ? n : 1));
        double sg = s == 0 ? -1.0 : 1.0;
        for (int j = 0; j < n; ++j) {
            double a = 2.0 * PI * (double)j / (double)n;
            pl->tw[s][j] = cos(a) + I * (sg * sin(a));
        }
    }
}

static void plan_free(fftplan* pl)
{
    free(pl->tw[0]);
    free(pl->tw[1]);
}

static void fft_rec(const cplx* in, int istride, cplx* out, int n,
                    const cplx* tw, int N0, int twstride, const int* f)
{
    if (n == 1) { out[0] = in[0]; return; }
    int r = f[0];
    int m = n / r;
    for (int q = 0; q < r; ++q)
        fft_rec(in + (size_t)q * istride, istride * r, out + (size_t)q * m, m,
                tw, N0, twstride * r, f + 1);
    cplx t[64];
    int wr = N0 / r;
    for (int k = 0; k < m; ++k) {
        for (int q = 0; q < r; ++q) {
            long e = ((long)q * k * twstride) % N0;
            t[q] = out[(size_t)q * m + k] * tw[e];
        }
        for (int sidx = 0; sidx < r; ++sidx) {
            cplx acc = 0.0;
            for (int q = 0; q < r; ++q) {
                long e = ((long)q * sidx * wr) % N0;
                acc += t[q] * tw[e];
            }
            out[(size_t)k + (size_t)sidx * m] = acc;
        }
    }
}

/* in-place transform of one strided line through two thread-local buffers */
static void fft_line(const fftplan* pl, cplx* base, size_t stride, int sign,
                     cplx* buf_in, cplx* buf_out)
{
    int n = pl->n;
    for (int j = 0; j < n; ++j) buf_in[j] = base[(size_t)j * stride];
    fft_rec(buf_in, 1, buf_out, n, pl->tw[sign < 0 ? 0 : 1], n, 1, pl->f);
    for (int j = 0; j < n; ++j) base[(size_t)j * stride] = buf_out[j];
}

/* ------------------------------------------------------------------------ */
/* state                                                                    */
/* ------------------------------------------------------------------------ */
struct or_state {
    hc_params prm;
    int nx, ny, nz, nia, nja, nka;
    int istr3, iend3, jstr3, jend3, kstr3, kend3;
    double dx, dy, dx2, dy2, dpx_coef;
    cplx wx1, wy1;
    double *dz, *l_t, *l_b, *dz_t, *dz_b;       /* 1-based, length nka+1 */
    double *u, *v, *w, *p, *phi, *t;
    double *ff, *gg, *hh, *ss, *ff0, *gg0, *hh0, *ss0, *qu, *qv, *qw;
    double *uhx, *uhy, *uhz, *vhx, *vhy, *vhz, *whx, *why, *thx, *thy, *thz;
    double *mean[11];
    double *bfx, *bfy, *bfz;                    /* body force (NULL: none), not in the reference */
    double *aa, *cc;                            /* (nx,ny,nka) */
    cplx *bb;
    double *aa_u, *cc_u, *aa_w, *cc_w, *aa_p, *cc_p, *aa_t, *cc_t;
    cplx *bb_u, *bb_w, *bb_p, *bb_t;
    cplx *c_src, *c_var;                        /* (nx,ny,nz) */
    cplx *c_u, *c_v, *c_w, *c_p, *c_phi, *c_t, *c_qu, *c_qv, *c_qw;
    cplx *c_ff, *c_gg, *c_hh, *c_ss;
    double dpx_drive, ubar, time_sim, cfl_max, div_hist_max;
    double rk_a, rk_b, rk_c, got;
    double div_avg_sub[3], div_max_sub[3];
    int nan_flag;
    int stps;
    int initialized;
    fftplan px, py;
};

/* ghosted Fortran array (nia,nja,nka), 1-based */
#define F(a, i, j, k) (a)[(size_t)((i) - 1) + (size_t)s->nia * ((size_t)((j) - 1) + (size_t)s->nja * (size_t)((k) - 1))]
/* (nx,ny,*) array, 1-based */
#define C(a, i, j, k) (a)[(size_t)((i) - 1) + (size_t)s->nx * ((size_t)((j) - 1) + (size_t)s->ny * (size_t)((k) - 1))]

static int g_threads = 0;
void or_set_threads(int n) { g_threads = n; }

static double sq(double x) { return x * x; }   /* Fortran x**2.d0 */

/* ------------------------------------------------------------------------ */
/* mpi_2d_fft  (src/module_tools.f90:518-700), single domain                 */
/* ------------------------------------------------------------------------ */
static void zero_nyquist(int nx, int ny, int nz, cplx* c)
{
    /* l == -nx/2 <=> i = nx/2+1 ; m == -ny/2 <=> j = ny/2+1 (1-based) */
    for (int k = 0; k < nz; ++k) {
        for (int j = 0; j < ny; ++j)
            c[(size_t)(nx / 2) + (size_t)nx * ((size_t)j + (size_t)ny * k)] = 0.0;
        for (int i = 0; i < nx; ++i)
            c[(size_t)i + (size_t)nx * ((size_t)(ny / 2) + (size_t)ny * k)] = 0.0;
    }
}

static void fft2d_planned(const fftplan* px, const fftplan* py, int nx, int ny, int nz,
                          cplx* c, int direction)
{
    if (direction == 1) zero_nyquist(nx, ny, nz, c);
    int sign = direction == -1 ? -1 : 1;
    int nmax = nx > ny ? nx : ny;
    /* y lines, one per (i,k) */
#pragma omp parallel if (g_threads != 1)
    {
        cplx* b1 = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
        cplx* b2 = (cplx*)malloc(sizeof(cplx) * (size_t)nmax);
#pragma omp for collapse(2) schedule(static)
        for (int k = 0; k < nz; ++k)
            for (int i = 0; i < nx; ++i) {
                cplx* base = c + (size_t)i + (size_t)nx * (size_t)ny * k;
                fft_line(py, base, (size_t)nx, sign, b1, b2);
                if (direction == -1)
                    for (int j = 0; j < ny; ++j) base[(size_t)j * nx] = base[(size_t)j * nx] / (double)ny;
            }
#pragma omp for collapse(2) schedule(static)
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j) {
                cplx* base = c + (size_t)nx * ((size_t)j + (size_t)ny * k);
                fft_line(px, base, 1, sign, b1, b2);
                if (direction == -1)
                    for (int i = 0; i < nx; ++i) base[i] = base[i] / (double)nx;
            }
        free(b1);
        free(b2);
    }
    if (direction == -1) zero_nyquist(nx, ny, nz, c);
}

static void mpi_2d_fft(or_state* s, cplx* c, int direction)
{
    fft2d_planned(&s->px, &s->py, s->nx, s->ny, s->nz, c, direction);
}

int or_fft2d(int nx, int ny, int nz, double* c_interleaved, int direction)
{
    if (nx < 2 || ny < 2 || nz < 1 || !c_interleaved) return HC_ERR_ARG;
    fftplan px, py;
    plan_init(&px, nx);
    plan_init(&py, ny);
    fft2d_planned(&px, &py, nx, ny, nz, (cplx*)c_interleaved, direction);
    plan_free(&px);
    plan_free(&py);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* wavenumber index map, used throughout (e.g. src/module_poisson_solver.f90:59-69) */
/* ------------------------------------------------------------------------ */
static int lmap(int i, int n) { return (i <= n / 2) ? i - 1 : i - n - 1; }

/* ------------------------------------------------------------------------ */
/* get_mesh_param (src/module_parameters.f90:432-508)                        */
/* ------------------------------------------------------------------------ */
static void get_mesh_param(or_state* s)
{
    int nz = s->nz, nka = s->nka;
    double zmin = 0.0, zmax = s->prm.lz, zmean, stretch_sysm, coeff_a;
    if (s->prm.ochannel == 0) {
        zmean = 0.5 * (zmin + zmax);
        stretch_sysm = 0.5;
        coeff_a = (2.0 + nz) * stretch_sysm;
    } else {
        zmean = (zmin + zmax);
        stretch_sysm = 1.0;
        coeff_a = (1.0 + nz) * stretch_sysm;
    }
    double* zz = (double*)calloc((size_t)nka + 2, sizeof(double));
    for (int k = 1; k <= nz + 1; ++k)
        zz[k + 2] = zmean + (zmin - zmean) / tanh(2.0 * s->prm.zstretch) *
                    tanh(2.0 * s->prm.zstretch * (k - coeff_a) / (1.0 - coeff_a));
    for (int k = 1; k <= nka; ++k) s->dz[k] = 0.0;
    for (int k = s->kstr3; k <= s->kend3; ++k) s->dz[k] = zz[k + 1] - zz[k];
    s->dz[s->kstr3 - 1] = s->dz[s->kstr3];
    s->dz[s->kend3 + 1] = s->dz[s->kend3];
    s->dz[s->kstr3 - 2] = s->dz[s->kstr3];
    s->dz[s->kend3 + 2] = s->dz[s->kend3];
    for (int k = s->kstr3 - 1; k <= s->kend3 + 1; ++k) {
        s->l_t[k] = s->dz[k] / (s->dz[k] + s->dz[k + 1]);
        s->l_b[k] = s->dz[k] / (s->dz[k] + s->dz[k - 1]);
    }
    for (int k = s->kstr3 - 1; k <= s->kend3 + 1; ++k) {
        s->dz_t[k] = 0.5 * (s->dz[k] + s->dz[k + 1]);
        s->dz_b[k] = 0.5 * (s->dz[k] + s->dz[k - 1]);
    }
    free(zz);
}

/* ------------------------------------------------------------------------ */
/* horizontal modified wavenumbers, as written in the coefficient builders.  */
/* Fortran complex**integer is evaluated by repeated multiplication and      */
/* complex**real through exp(y*log(z)).                                      */
/* ------------------------------------------------------------------------ */
static cplx cpowi(cplx z, int n)
{
    cplx r = 1.0;
    if (n == 0) return r;
    unsigned u;
    cplx x = z;
    if (n < 0) { u = (unsigned)(-n); x = r / x; } else u = (unsigned)n;
    for (;;) {
        if (u & 1u) r *= x;
        u >>= 1;
        if (u) x *= x; else break;
    }
    return r;
}
static cplx cpowr(cplx z, double y) { return y == 0.0 ? 1.0 : cpow(z, y); }

/* cds=1 / cds=2 second-derivative symbols times the caller's scale, and cds=3 */
static cplx kx_helm(or_state* s, int l, double dif, double h2, cplx w1, double L)
{
    double dt = s->prm.dt;
    if (s->prm.cds == 1) return 0.5 * dt * (cpowi(w1, l) + cpowi(w1, -l) - 2.0) * dif / h2;
    if (s->prm.cds == 2)
        return dt * (-cpowr(w1, 2.0 * l) + 16.0 * cpowi(w1, l) - 30.0 + 16.0 * cpowi(w1, -l) -
                     cpowr(w1, -2.0 * l)) / 24.0 * dif / h2;
    return 0.5 * dt * dif * (-sq(2.0 * PI / L * l));
}

static cplx kx_pois(or_state* s, int l, double h2, cplx w1, double L)
{
    if (s->prm.cds == 1) return (cpowi(w1, l) + cpowi(w1, -l) - 2.0) / h2;
    if (s->prm.cds == 2)
        return (cpowr(w1, 3.0 * l) - 54.0 * cpowr(w1, 2.0 * l) + 783.0 * cpowi(w1, l) - 1460.0 +
                783.0 * cpowi(w1, -l) - 54.0 * cpowr(w1, -2.0 * l) + cpowr(w1, -3.0 * l)) /
               576.0 / h2;
    return -sq(2.0 * PI / L * l);
}

/* The builders evaluate kx, ky inside their k,j,i loops; the values depend on
 * the mode only, so they are evaluated once per i and once per j here. */
typedef struct { cplx* x; cplx* y; } symtab;
static symtab sym_tables(or_state* s, int pois, double dif)
{
    symtab t;
    t.x = (cplx*)malloc(sizeof(cplx) * (size_t)(s->nx + 1));
    t.y = (cplx*)malloc(sizeof(cplx) * (size_t)(s->ny + 1));
    for (int i = 1; i <= s->nx; ++i) {
        int l = lmap(i, s->nx);
        t.x[i] = pois ? kx_pois(s, l, s->dx2, s->wx1, s->prm.lx) : kx_helm(s, l, dif, s->dx2, s->wx1, s->prm.lx);
    }
    for (int j = 1; j <= s->ny; ++j) {
        int m = lmap(j, s->ny);
        t.y[j] = pois ? kx_pois(s, m, s->dy2, s->wy1, s->prm.ly) : kx_helm(s, m, dif, s->dy2, s->wy1, s->prm.ly);
    }
    return t;
}
static void sym_free(symtab t) { free(t.x); free(t.y); }

/* get_p_eqn_coeff (src/module_poisson_solver.f90:32-122) */
static void get_p_eqn_coeff(or_state* s, double* aa, cplx* bb, double* cc)
{
    symtab tb = sym_tables(s, 1, 0.0);
    for (int k = 1; k <= s->nka; ++k) { aa[k] = 0.0; cc[k] = 0.0; }
    memset(bb, 0, sizeof(cplx) * (size_t)s->nx * s->ny * s->nka);
    for (int k = s->kstr3; k <= s->kend3; ++k) {
        aa[k] = 1.0 / s->dz[k] / s->dz_b[k];
        cc[k] = 1.0 / s->dz[k] / s->dz_t[k];
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) {
                cplx kx = tb.x[i], ky = tb.y[j];
                C(bb, i, j, k) = kx + ky - aa[k] - cc[k];
                if (k == s->kstr3) { C(bb, i, j, k) = C(bb, i, j, k) + aa[k]; aa[k] = 0.0; }
                if (k == s->kend3) { C(bb, i, j, k) = C(bb, i, j, k) + cc[k]; cc[k] = 0.0; }
            }
    }
    sym_free(tb);
}

/* get_u_eqn_coeff (src/module_poisson_solver.f90:181-282) */
static void get_u_eqn_coeff(or_state* s, double* aa, cplx* bb, double* cc)
{
    double dt = s->prm.dt, nu = s->prm.nu;
    symtab tb = sym_tables(s, 0, nu);
    for (int k = 1; k <= s->nka; ++k) { aa[k] = 0.0; cc[k] = 0.0; }
    memset(bb, 0, sizeof(cplx) * (size_t)s->nx * s->ny * s->nka);
    for (int k = s->kstr3; k <= s->kend3; ++k) {
        aa[k] = -0.5 * dt * nu / s->dz[k] / s->dz_b[k];
        cc[k] = -0.5 * dt * nu / s->dz[k] / s->dz_t[k];
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) {
                cplx kx = tb.x[i], ky = tb.y[j];
                C(bb, i, j, k) = -kx - ky - aa[k] - cc[k];
                if (k == s->kstr3) { C(bb, i, j, k) = C(bb, i, j, k) - aa[k]; aa[k] = 0.0; }
                if (k == s->kend3) {
                    if (s->prm.ochannel == 0) { C(bb, i, j, k) = C(bb, i, j, k) - cc[k]; cc[k] = 0.0; }
                    else { C(bb, i, j, k) = C(bb, i, j, k) + cc[k]; cc[k] = 0.0; }
                }
            }
    }
    sym_free(tb);
}

/* get_w_eqn_coeff (src/module_poisson_solver.f90:287-374) */
static void get_w_eqn_coeff(or_state* s, double* aa, cplx* bb, double* cc)
{
    double dt = s->prm.dt, nu = s->prm.nu;
    symtab tb = sym_tables(s, 0, nu);
    for (int k = 1; k <= s->nka; ++k) { aa[k] = 0.0; cc[k] = 0.0; }
    memset(bb, 0, sizeof(cplx) * (size_t)s->nx * s->ny * s->nka);
    for (int k = s->kstr3; k <= s->kend3 - 1; ++k) {
        aa[k] = -0.5 * dt * nu / s->dz[k] / s->dz_t[k];
        cc[k] = -0.5 * dt * nu / s->dz[k + 1] / s->dz_t[k];
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) {
                cplx kx = tb.x[i], ky = tb.y[j];
                C(bb, i, j, k) = -kx - ky - aa[k] - cc[k];
                if (k == s->kstr3) aa[k] = 0.0;
                if (k == s->kend3 - 1) cc[k] = 0.0;
            }
    }
    sym_free(tb);
}

/* get_t_eqn_coeff (src/module_poisson_solver.f90:379-477) */
static void get_t_eqn_coeff(or_state* s, double* aa, cplx* bb, double* cc)
{
    double dt = s->prm.dt, al = s->prm.alpha;
    symtab tb = sym_tables(s, 0, al);
    for (int k = 1; k <= s->nka; ++k) { aa[k] = 0.0; cc[k] = 0.0; }
    memset(bb, 0, sizeof(cplx) * (size_t)s->nx * s->ny * s->nka);
    for (int k = s->kstr3; k <= s->kend3; ++k) {
        aa[k] = -0.5 * dt * al / s->dz[k] / s->dz_b[k];
        cc[k] = -0.5 * dt * al / s->dz[k] / s->dz_t[k];
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) {
                cplx kx = tb.x[i], ky = tb.y[j];
                C(bb, i, j, k) = -kx - ky - aa[k] - cc[k];
                /* the ghost T(ks-1) folds into the diagonal with -1 (fixed T) or +1
                 * (fixed gradient); aa is cleared inside the loop, so only the first
                 * mode, the mean, receives the fold (as in the reference) */
                if (k == s->kstr3) { C(bb, i, j, k) = C(bb, i, j, k) + (s->prm.tbc_bot ? aa[k] : -aa[k]); aa[k] = 0.0; }
                if (k == s->kend3) { C(bb, i, j, k) = C(bb, i, j, k) - cc[k]; cc[k] = 0.0; }
            }
    }
    sym_free(tb);
}

/* ------------------------------------------------------------------------ */
/* parameters                                                               */
/* ------------------------------------------------------------------------ */
/* update_ri (src/module_parameters.f90:580-590) */
static void update_ri(or_state* s, int stps)
{
    s->got = s->prm.ri_str + (s->prm.ri_end - s->prm.ri_str) * 1.0 / s->prm.imax * stps;
}

/* update_dpx_drive (src/module_parameters.f90:594-613) */
static void update_dpx_drive(or_state* s)
{
    if (s->prm.dp_opt == 1) s->dpx_drive = 1.0;
    else if (s->prm.dp_opt == 2) s->dpx_drive = s->dpx_drive - (s->ubar + s->prm.u_mrf - 1.0) * s->dpx_coef;
}

/* assign_rk_coeff (src/module_parameters.f90:618-641), constants :210-212 */
static const double rkc1[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
static const double rkc2[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};
static const double rkc3[3] = {8.0 / 15.0, 2.0 / 15.0, 1.0 / 3.0};
static void assign_rk_coeff(or_state* s, double a, double b, double c)
{
    if (s->prm.dts == 2) { s->rk_a = a; s->rk_b = b; s->rk_c = c; }
    else { s->rk_a = 1.5; s->rk_b = -0.5; s->rk_c = 1.0; }
}

/* calculate_ubar (src/module_parameters.f90:513-546) */
static void calculate_ubar(or_state* s)
{
    double ub = 0.0;
    for (int k = s->kstr3; k <= s->kend3; ++k)
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i) ub = ub + F(s->u, i, j, k) * s->dz[k];
    ub = ub / s->prm.lz / s->nx / s->ny;
    s->ubar = ub / 1;
}

/* ------------------------------------------------------------------------ */
/* boundary conditions (src/module_boundary.f90)                            */
/* ------------------------------------------------------------------------ */
/* comm_bound :361-487 with p_row = p_col = 1: periodic copy over k in [kstr3-1,kend3+1] */
static void comm_bound(or_state* s, double* var)
{
    for (int k = s->kstr3 - 1; k <= s->kend3 + 1; ++k) {
        for (int j = s->jstr3; j <= s->jend3; ++j) {
            F(var, s->istr3 - 1, j, k) = F(var, s->iend3, j, k);
            F(var, s->istr3 - 2, j, k) = F(var, s->iend3 - 1, j, k);
            F(var, s->iend3 + 1, j, k) = F(var, s->istr3, j, k);
            F(var, s->iend3 + 2, j, k) = F(var, s->istr3 + 1, j, k);
        }
        for (int i = s->istr3 - 2; i <= s->iend3 + 2; ++i) {
            F(var, i, s->jstr3 - 1, k) = F(var, i, s->jend3, k);
            F(var, i, s->jstr3 - 2, k) = F(var, i, s->jend3 - 1, k);
            F(var, i, s->jend3 + 1, k) = F(var, i, s->jstr3, k);
            F(var, i, s->jend3 + 2, k) = F(var, i, s->jstr3 + 1, k);
        }
    }
}

/* update_boundary_uvw :33-128 */
static void update_boundary_uvw(or_state* s, double* u, double* v, double* w)
{
    double um = s->prm.u_mrf;
    int ks = s->kstr3, ke = s->kend3;
    for (int j = s->jstr3; j <= s->jend3; ++j)
        for (int i = s->istr3; i <= s->iend3; ++i) {
            if (s->prm.ochannel == 0) {
                F(u, i, j, ke + 1) = -F(u, i, j, ke) - 2.0 * um;
                F(u, i, j, ks - 1) = -F(u, i, j, ks) - 2.0 * um;
                F(v, i, j, ke + 1) = -F(v, i, j, ke);
                F(v, i, j, ks - 1) = -F(v, i, j, ks);
            } else {
                F(u, i, j, ke + 1) = F(u, i, j, ke);
                F(u, i, j, ks - 1) = -F(u, i, j, ks) - 2.0 * um;
                F(v, i, j, ke + 1) = F(v, i, j, ke);
                F(v, i, j, ks - 1) = -F(v, i, j, ks);
            }
            F(w, i, j, ke) = 0.0;
            F(w, i, j, ke + 1) = -F(w, i, j, ke - 1);
            F(w, i, j, ks - 1) = 0.0;
        }
    if (s->prm.cds != 3) { comm_bound(s, u); comm_bound(s, v); comm_bound(s, w); }
}

/* update_boundary_p :133-162 */
static void update_boundary_p(or_state* s, double* p)
{
    for (int j = s->jstr3; j <= s->jend3; ++j)
        for (int i = s->istr3; i <= s->iend3; ++i) {
            F(p, i, j, s->kend3 + 1) = F(p, i, j, s->kend3);
            F(p, i, j, s->kstr3 - 1) = F(p, i, j, s->kstr3);
        }
    if (s->prm.cds != 3) comm_bound(s, p);
}

/* update_boundary_t :167-196. tbc_bot = 1 (not in the reference): the bottom
 * ghost continues T with the fixed wall gradient tbot, T(ks-1) = T(ks) - tbot dz_b(ks). */
static void update_boundary_t(or_state* s, double* t)
{
    const double gb = s->prm.tbot * s->dz_b[s->kstr3];
    for (int j = s->jstr3; j <= s->jend3; ++j)
        for (int i = s->istr3; i <= s->iend3; ++i) {
            F(t, i, j, s->kend3 + 1) = 2.0 * s->prm.ttop - F(t, i, j, s->kend3);
            F(t, i, j, s->kstr3 - 1) = s->prm.tbc_bot ? F(t, i, j, s->kstr3) - gb
                                                      : 2.0 * s->prm.tbot - F(t, i, j, s->kstr3);
        }
    if (s->prm.cds != 3) comm_bound(s, t);
}

/* update_boundary_uvwhxyz :202-305 */
static void update_boundary_uvwhxyz(or_state* s)
{
    double um = s->prm.u_mrf;
    int ks = s->kstr3, ke = s->kend3;
    for (int j = s->jstr3; j <= s->jend3; ++j)
        for (int i = s->istr3; i <= s->iend3; ++i) {
            if (s->prm.ochannel == 0) {
                F(s->uhx, i, j, ke + 1) = -F(s->uhx, i, j, ke) - 2.0 * um;
                F(s->uhy, i, j, ke + 1) = -F(s->uhy, i, j, ke) - 2.0 * um;
                F(s->uhz, i, j, ke) = -um;
                F(s->uhz, i, j, ke + 1) = -F(s->uhz, i, j, ke - 1) - 2.0 * um;
                F(s->vhx, i, j, ke + 1) = -F(s->vhx, i, j, ke);
                F(s->vhy, i, j, ke + 1) = -F(s->vhy, i, j, ke);
                F(s->vhz, i, j, ke) = 0.0;
                F(s->vhz, i, j, ke + 1) = -F(s->vhz, i, j, ke - 1);
                F(s->whx, i, j, ke) = 0.0;
                F(s->whx, i, j, ke + 1) = -F(s->whx, i, j, ke - 1);
                F(s->why, i, j, ke) = 0.0;
                F(s->why, i, j, ke + 1) = -F(s->why, i, j, ke - 1);
            } else {
                F(s->uhx, i, j, ke + 1) = F(s->uhx, i, j, ke);
                F(s->uhy, i, j, ke + 1) = F(s->uhy, i, j, ke);
                F(s->uhz, i, j, ke) = F(s->u, i, j, ke);
                F(s->uhz, i, j, ke + 1) = F(s->uhz, i, j, ke);
                F(s->vhx, i, j, ke + 1) = F(s->vhx, i, j, ke);
                F(s->vhy, i, j, ke + 1) = F(s->vhy, i, j, ke);
                F(s->vhz, i, j, ke) = F(s->v, i, j, ke);
                F(s->vhz, i, j, ke + 1) = F(s->vhz, i, j, ke);
                F(s->whx, i, j, ke) = 0.0;
                F(s->whx, i, j, ke + 1) = -F(s->whx, i, j, ke - 1);
                F(s->why, i, j, ke) = 0.0;
                F(s->why, i, j, ke + 1) = -F(s->why, i, j, ke - 1);
            }
        }
    for (int j = s->jstr3; j <= s->jend3; ++j)
        for (int i = s->istr3; i <= s->iend3; ++i) {
            F(s->uhx, i, j, ks - 1) = -F(s->uhx, i, j, ks) - 2.0 * um;
            F(s->uhy, i, j, ks - 1) = -F(s->uhy, i, j, ks) - 2.0 * um;
            F(s->uhz, i, j, ks - 1) = -um;
            F(s->vhx, i, j, ks - 1) = -F(s->vhx, i, j, ks);
            F(s->vhy, i, j, ks - 1) = -F(s->vhy, i, j, ks);
            F(s->vhz, i, j, ks - 1) = 0.0;
            F(s->whx, i, j, ks - 1) = 0.0;
            F(s->why, i, j, ks - 1) = 0.0;
        }
    if (s->prm.cds != 3) {
        comm_bound(s, s->uhx); comm_bound(s, s->uhy); comm_bound(s, s->uhz);
        comm_bound(s, s->vhx); comm_bound(s, s->vhy); comm_bound(s, s->vhz);
        comm_bound(s, s->whx); comm_bound(s, s->why);
    }
}

/* update_boundary_thxyz :311-355 */
static void update_boundary_thxyz(or_state* s)
{
    int ks = s->kstr3, ke = s->kend3;
    double tt = s->prm.ttop, tb = s->prm.tbot;
    for (int j = s->jstr3; j <= s->jend3; ++j)
        for (int i = s->istr3; i <= s->iend3; ++i) {
            F(s->thx, i, j, ke + 1) = -F(s->thx, i, j, ke) + 2.0 * tt;
            F(s->thy, i, j, ke + 1) = -F(s->thy, i, j, ke) + 2.0 * tt;
            F(s->thz, i, j, ke) = tt;
            F(s->thz, i, j, ke + 1) = -F(s->thz, i, j, ke - 1) + 2.0 * tt;
        }
    const double gb = tb * s->dz_b[ks];
    for (int j = s->jstr3; j <= s->jend3; ++j)
        for (int i = s->istr3; i <= s->iend3; ++i) {
            if (s->prm.tbc_bot) {   /* fixed gradient: the ghost and the wall value continue T linearly */
                F(s->thx, i, j, ks - 1) = F(s->thx, i, j, ks) - gb;
                F(s->thy, i, j, ks - 1) = F(s->thy, i, j, ks) - gb;
                F(s->thz, i, j, ks - 1) = F(s->t, i, j, ks) - 0.5 * gb;
            } else {
                F(s->thx, i, j, ks - 1) = -F(s->thx, i, j, ks) + 2.0 * tb;
                F(s->thy, i, j, ks - 1) = -F(s->thy, i, j, ks) + 2.0 * tb;
                F(s->thz, i, j, ks - 1) = tb;
            }
        }
    if (s->prm.cds != 3) { comm_bound(s, s->thx); comm_bound(s, s->thy); comm_bound(s, s->thz); }
}

/* ------------------------------------------------------------------------ */
/* interpolation (src/module_tools.f90:410-512)                             */
/* ------------------------------------------------------------------------ */
static void get_interp_fields_uvwhxyz(or_state* s)
{
    double *u = s->u, *v = s->v, *w = s->w;
#pragma omp parallel for collapse(2) schedule(static) if (g_threads != 1)
    for (int k = s->kstr3; k <= s->kend3; ++k)
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i) {
                if (s->prm.cds == 1) {
                    F(s->uhx, i, j, k) = 0.5 * (F(u, i, j, k) + F(u, i - 1, j, k));
                    F(s->uhy, i, j, k) = 0.5 * (F(u, i, j + 1, k) + F(u, i, j, k));
                    F(s->vhx, i, j, k) = 0.5 * (F(v, i + 1, j, k) + F(v, i, j, k));
                    F(s->vhy, i, j, k) = 0.5 * (F(v, i, j, k) + F(v, i, j - 1, k));
                    F(s->whx, i, j, k) = 0.5 * (F(w, i + 1, j, k) + F(w, i, j, k));
                    F(s->why, i, j, k) = 0.5 * (F(w, i, j + 1, k) + F(w, i, j, k));
                } else if (s->prm.cds == 2) {
                    F(s->uhx, i, j, k) = (-F(u, i + 1, j, k) + 9.0 * F(u, i, j, k) + 9.0 * F(u, i - 1, j, k) - F(u, i - 2, j, k)) / 16.0;
                    F(s->uhy, i, j, k) = (-F(u, i, j + 2, k) + 9.0 * F(u, i, j + 1, k) + 9.0 * F(u, i, j, k) - F(u, i, j - 1, k)) / 16.0;
                    F(s->vhx, i, j, k) = (-F(v, i + 2, j, k) + 9.0 * F(v, i + 1, j, k) + 9.0 * F(v, i, j, k) - F(v, i - 1, j, k)) / 16.0;
                    F(s->vhy, i, j, k) = (-F(v, i, j + 1, k) + 9.0 * F(v, i, j, k) + 9.0 * F(v, i, j - 1, k) - F(v, i, j - 2, k)) / 16.0;
                    F(s->whx, i, j, k) = (-F(w, i + 2, j, k) + 9.0 * F(w, i + 1, j, k) + 9.0 * F(w, i, j, k) - F(w, i - 1, j, k)) / 16.0;
                    F(s->why, i, j, k) = (-F(w, i, j + 2, k) + 9.0 * F(w, i, j + 1, k) + 9.0 * F(w, i, j, k) - F(w, i, j - 1, k)) / 16.0;
                }
                F(s->uhz, i, j, k) = F(u, i, j, k + 1) * s->l_t[k] + F(u, i, j, k) * (1.0 - s->l_t[k]);
                F(s->vhz, i, j, k) = F(v, i, j, k + 1) * s->l_t[k] + F(v, i, j, k) * (1.0 - s->l_t[k]);
            }
}

static void get_interp_fields_thxyz(or_state* s)
{
    double* t = s->t;
#pragma omp parallel for collapse(2) schedule(static) if (g_threads != 1)
    for (int k = s->kstr3; k <= s->kend3; ++k)
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i) {
                if (s->prm.cds == 1) {
                    F(s->thx, i, j, k) = 0.5 * (F(t, i + 1, j, k) + F(t, i, j, k));
                    F(s->thy, i, j, k) = 0.5 * (F(t, i, j + 1, k) + F(t, i, j, k));
                } else if (s->prm.cds == 2) {
                    F(s->thx, i, j, k) = (-F(t, i + 2, j, k) + 9.0 * F(t, i + 1, j, k) + 9.0 * F(t, i, j, k) - F(t, i - 1, j, k)) / 16.0;
                    F(s->thy, i, j, k) = (-F(t, i, j + 2, k) + 9.0 * F(t, i, j + 1, k) + 9.0 * F(t, i, j, k) - F(t, i, j - 1, k)) / 16.0;
                }
                F(s->thz, i, j, k) = F(t, i, j, k + 1) * s->l_t[k] + F(t, i, j, k) * (1.0 - s->l_t[k]);
            }
}

/* ------------------------------------------------------------------------ */
/* FD momentum RHS: get_momentum_cnvdiff (src/module_cnvdiff.f90:35-374)    */
/* ------------------------------------------------------------------------ */
static void get_momentum_cnvdiff(or_state* s)
{
    const double dx = s->dx, dy = s->dy, dx2 = s->dx2, dy2 = s->dy2;
    const double dt = s->prm.dt, nu = s->prm.nu, um = s->prm.u_mrf, fc = s->prm.fc;
    const double ug = s->prm.ug, vg = s->prm.vg, got = s->got, t_ref = s->prm.t_ref;
    const double rk_a = s->rk_a, rk_b = s->rk_b, rk_c = s->rk_c;
    const int cds = s->prm.cds, dp_opt = s->prm.dp_opt, isscalar = s->prm.isscalar;
    double *u = s->u, *v = s->v, *w = s->w, *p = s->p, *t = s->t;
    double *uhx = s->uhx, *uhy = s->uhy, *uhz = s->uhz, *vhx = s->vhx, *vhy = s->vhy;
    double *vhz = s->vhz, *whx = s->whx, *why = s->why;
    double *dz = s->dz, *dz_t = s->dz_t, *dz_b = s->dz_b, *l_t = s->l_t;

    update_dpx_drive(s);
    const double dpx_drive = s->dpx_drive;

    /* U equation :55-161 */
#pragma omp parallel for collapse(2) schedule(static) if (g_threads != 1)
    for (int k = s->kstr3; k <= s->kend3; ++k)
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i) {
                double uux = 0, uvy = 0, ux = 0, uxx = 0, uyy = 0, dpdx = 0;
                if (cds == 1) {
                    uux = (sq(F(uhx, i + 1, j, k)) - sq(F(uhx, i, j, k))) / dx;
                    uvy = (F(uhy, i, j, k) * F(vhx, i, j, k) - F(uhy, i, j - 1, k) * F(vhx, i, j - 1, k)) / dy;
                    ux = (F(uhx, i + 1, j, k) - F(uhx, i, j, k)) / dx;
                } else if (cds == 2) {
                    uux = (-sq(F(uhx, i + 2, j, k)) + 27.0 * sq(F(uhx, i + 1, j, k)) - 27.0 * sq(F(uhx, i, j, k)) + sq(F(uhx, i - 1, j, k))) / 24.0 / dx;
                    uvy = (-F(uhy, i, j + 1, k) * F(vhx, i, j + 1, k) + 27.0 * F(uhy, i, j, k) * F(vhx, i, j, k) - 27.0 * F(uhy, i, j - 1, k) * F(vhx, i, j - 1, k) + F(uhy, i, j - 2, k) * F(vhx, i, j - 2, k)) / 24.0 / dy;
                    ux = (-F(uhx, i + 2, j, k) + 27.0 * F(uhx, i + 1, j, k) - 27.0 * F(uhx, i, j, k) + F(uhx, i - 1, j, k)) / 24.0 / dx;
                }
                double uwz = (F(uhz, i, j, k) * F(whx, i, j, k) - F(uhz, i, j, k - 1) * F(whx, i, j, k - 1)) / dz[k];
                if (cds == 1) {
                    uxx = (F(u, i + 1, j, k) - 2.0 * F(u, i, j, k) + F(u, i - 1, j, k)) / dx2;
                    uyy = (F(u, i, j + 1, k) - 2.0 * F(u, i, j, k) + F(u, i, j - 1, k)) / dy2;
                } else if (cds == 2) {
                    uxx = (-F(u, i + 2, j, k) + 16.0 * F(u, i + 1, j, k) - 30.0 * F(u, i, j, k) + 16.0 * F(u, i - 1, j, k) - F(u, i - 2, j, k)) / 12.0 / dx2;
                    uyy = (-F(u, i, j + 2, k) + 16.0 * F(u, i, j + 1, k) - 30.0 * F(u, i, j, k) + 16.0 * F(u, i, j - 1, k) - F(u, i, j - 2, k)) / 12.0 / dy2;
                }
                double uzz = ((F(u, i, j, k + 1) - F(u, i, j, k)) / dz_t[k] - (F(u, i, j, k) - F(u, i, j, k - 1)) / dz_b[k]) / dz[k];
                if (dp_opt == 3)
                    F(s->ff, i, j, k) = -uux - uvy - uwz - um * ux + fc * (0.5 * (F(vhx, i, j, k) + F(vhx, i, j - 1, k)) - vg);
                else
                    F(s->ff, i, j, k) = -uux - uvy - uwz + dpx_drive - um * ux;
                if (s->bfx) F(s->ff, i, j, k) += F(s->bfx, i, j, k);
                if (cds == 1) dpdx = (F(p, i + 1, j, k) - F(p, i, j, k)) / dx;
                else if (cds == 2) dpdx = (-F(p, i + 2, j, k) + 27.0 * F(p, i + 1, j, k) - 27.0 * F(p, i, j, k) + F(p, i - 1, j, k)) / 24.0 / dx;
                F(s->qu, i, j, k) = F(u, i, j, k) + dt * (rk_a * F(s->ff, i, j, k) + rk_b * F(s->ff0, i, j, k)) +
                                    rk_c * 0.5 * dt * nu * (uxx + uyy + uzz) - rk_c * dt * dpdx;
            }

    /* V equation :166-270 */
#pragma omp parallel for collapse(2) schedule(static) if (g_threads != 1)
    for (int k = s->kstr3; k <= s->kend3; ++k)
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i) {
                double vux = 0, vvy = 0, vx = 0, vxx = 0, vyy = 0, dpdy = 0;
                if (cds == 1) {
                    vux = (F(vhx, i, j, k) * F(uhy, i, j, k) - F(vhx, i - 1, j, k) * F(uhy, i - 1, j, k)) / dx;
                    vvy = (sq(F(vhy, i, j + 1, k)) - sq(F(vhy, i, j, k))) / dy;
                    vx = (F(vhx, i, j, k) - F(vhx, i - 1, j, k)) / dx;
                } else if (cds == 2) {
                    vux = (-F(vhx, i + 1, j, k) * F(uhy, i + 1, j, k) + 27.0 * F(vhx, i, j, k) * F(uhy, i, j, k) - 27.0 * F(vhx, i - 1, j, k) * F(uhy, i - 1, j, k) + F(vhx, i - 2, j, k) * F(uhy, i - 2, j, k)) / 24.0 / dx;
                    vvy = (-sq(F(vhy, i, j + 2, k)) + 27.0 * sq(F(vhy, i, j + 1, k)) - 27.0 * sq(F(vhy, i, j, k)) + sq(F(vhy, i, j - 1, k))) / 24.0 / dy;
                    vx = (-F(vhx, i + 1, j, k) + 27.0 * F(vhx, i, j, k) - 27.0 * F(vhx, i - 1, j, k) + F(vhx, i - 2, j, k)) / 24.0 / dx;
                }
                double vwz = (F(vhz, i, j, k) * F(why, i, j, k) - F(vhz, i, j, k - 1) * F(why, i, j, k - 1)) / dz[k];
                if (cds == 1) {
                    vxx = (F(v, i + 1, j, k) - 2.0 * F(v, i, j, k) + F(v, i - 1, j, k)) / dx2;
                    vyy = (F(v, i, j + 1, k) - 2.0 * F(v, i, j, k) + F(v, i, j - 1, k)) / dy2;
                } else if (cds == 2) {
                    vxx = (-F(v, i + 2, j, k) + 16.0 * F(v, i + 1, j, k) - 30.0 * F(v, i, j, k) + 16.0 * F(v, i - 1, j, k) - F(v, i - 2, j, k)) / 12.0 / dx2;
                    vyy = (-F(v, i, j + 2, k) + 16.0 * F(v, i, j + 1, k) - 30.0 * F(v, i, j, k) + 16.0 * F(v, i, j - 1, k) - F(v, i, j - 2, k)) / 12.0 / dy2;
                }
                double vzz = ((F(v, i, j, k + 1) - F(v, i, j, k)) / dz_t[k] - (F(v, i, j, k) - F(v, i, j, k - 1)) / dz_b[k]) / dz[k];
                if (dp_opt == 3)
                    F(s->gg, i, j, k) = -vux - vvy - vwz - um * vx + fc * (ug - 0.5 * (F(uhy, i, j, k) + F(uhy, i - 1, j, k)) - um);
                else
                    F(s->gg, i, j, k) = -vux - vvy - vwz - um * vx;
                if (s->bfx) F(s->gg, i, j, k) += F(s->bfy, i, j, k);
                if (cds == 1) dpdy = (F(p, i, j + 1, k) - F(p, i, j, k)) / dy;
                else if (cds == 2) dpdy = (-F(p, i, j + 2, k) + 27.0 * F(p, i, j + 1, k) - 27.0 * F(p, i, j, k) + F(p, i, j - 1, k)) / 24.0 / dy;
                F(s->qv, i, j, k) = F(v, i, j, k) + dt * (rk_a * F(s->gg, i, j, k) + rk_b * F(s->gg0, i, j, k)) +
                                    rk_c * 0.5 * dt * nu * (vxx + vyy + vzz) - rk_c * dt * dpdy;
            }

    /* W equation :274-370 */
#pragma omp parallel for collapse(2) schedule(static) if (g_threads != 1)
    for (int k = s->kstr3; k <= s->kend3 - 1; ++k)
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i) {
                double wux = 0, wvy = 0, wx = 0, wxx = 0, wyy = 0;
                if (cds == 1) {
                    wux = (F(whx, i, j, k) * F(uhz, i, j, k) - F(whx, i - 1, j, k) * F(uhz, i - 1, j, k)) / dx;
                    wvy = (F(why, i, j, k) * F(vhz, i, j, k) - F(why, i, j - 1, k) * F(vhz, i, j - 1, k)) / dy;
                    wx = (F(whx, i, j, k) - F(whx, i - 1, j, k)) / dx;
                } else if (cds == 2) {
                    wux = (-F(whx, i + 1, j, k) * F(uhz, i + 1, j, k) + 27.0 * F(whx, i, j, k) * F(uhz, i, j, k) - 27.0 * F(whx, i - 1, j, k) * F(uhz, i - 1, j, k) + F(whx, i - 2, j, k) * F(uhz, i - 2, j, k)) / 24.0 / dx;
                    wvy = (-F(why, i, j + 1, k) * F(vhz, i, j + 1, k) + 27.0 * F(why, i, j, k) * F(vhz, i, j, k) - 27.0 * F(why, i, j - 1, k) * F(vhz, i, j - 1, k) + F(why, i, j - 2, k) * F(vhz, i, j - 2, k)) / 24.0 / dy;
                    wx = (-F(whx, i + 1, j, k) + 27.0 * F(whx, i, j, k) - 27.0 * F(whx, i - 1, j, k) + F(whx, i - 2, j, k)) / 24.0 / dx;
                }
                double a1 = sq(0.5 * (F(w, i, j, k) + F(w, i, j, k + 1)));
                double a2 = sq(0.5 * (F(w, i, j, k) + F(w, i, j, k - 1)));
                double wwz = (a1 - a2) / dz_t[k];
                if (cds == 1) {
                    wxx = (F(w, i + 1, j, k) - 2.0 * F(w, i, j, k) + F(w, i - 1, j, k)) / dx2;
                    wyy = (F(w, i, j + 1, k) - 2.0 * F(w, i, j, k) + F(w, i, j - 1, k)) / dy2;
                } else if (cds == 2) {
                    wxx = (-F(w, i + 2, j, k) + 16.0 * F(w, i + 1, j, k) - 30.0 * F(w, i, j, k) + 16.0 * F(w, i - 1, j, k) - F(w, i - 2, j, k)) / 12.0 / dx2;
                    wyy = (-F(w, i, j + 2, k) + 16.0 * F(w, i, j + 1, k) - 30.0 * F(w, i, j, k) + 16.0 * F(w, i, j - 1, k) - F(w, i, j - 2, k)) / 12.0 / dy2;
                }
                double wzz = ((F(w, i, j, k + 1) - F(w, i, j, k)) / dz[k + 1] - (F(w, i, j, k) - F(w, i, j, k - 1)) / dz[k]) / dz_t[k];
                if (isscalar == 1)
                    F(s->hh, i, j, k) = -wux - wvy - wwz - um * wx + got * ((1.0 - l_t[k]) * F(t, i, j, k) + l_t[k] * F(t, i, j, k + 1) - t_ref);
                else
                    F(s->hh, i, j, k) = -wux - wvy - wwz - um * wx;
                if (s->bfx) F(s->hh, i, j, k) += F(s->bfz, i, j, k);
                double dpdz = (F(p, i, j, k + 1) - F(p, i, j, k)) / dz_t[k];
                F(s->qw, i, j, k) = F(w, i, j, k) + dt * (rk_a * F(s->hh, i, j, k) + rk_b * F(s->hh0, i, j, k)) +
                                    rk_c * 0.5 * dt * nu * (wxx + wyy + wzz) - rk_c * dt * dpdz;
            }
}

/* get_temperature_cnvdiff (src/module_cnvdiff.f90:381-473) */
static void get_temperature_cnvdiff(or_state* s, double* qt)
{
    const double dx = s->dx, dy = s->dy, dx2 = s->dx2, dy2 = s->dy2;
    const double dt = s->prm.dt, al = s->prm.alpha, um = s->prm.u_mrf;
    const double rk_a = s->rk_a, rk_b = s->rk_b, rk_c = s->rk_c;
    const int cds = s->prm.cds;
    double *u = s->u, *v = s->v, *w = s->w, *t = s->t;
    double *thx = s->thx, *thy = s->thy, *thz = s->thz;
    double *dz = s->dz, *dz_t = s->dz_t, *dz_b = s->dz_b;
#pragma omp parallel for collapse(2) schedule(static) if (g_threads != 1)
    for (int k = s->kstr3; k <= s->kend3; ++k)
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i) {
                double tux = 0, tvy = 0, tx = 0, txx = 0, tyy = 0;
                if (cds == 1) {
                    tux = (F(thx, i, j, k) * F(u, i, j, k) - F(thx, i - 1, j, k) * F(u, i - 1, j, k)) / dx;
                    tvy = (F(thy, i, j, k) * F(v, i, j, k) - F(thy, i, j - 1, k) * F(v, i, j - 1, k)) / dy;
                    tx = (F(thx, i, j, k) - F(thx, i - 1, j, k)) / dx;
                } else if (cds == 2) {
                    tux = (-F(thx, i + 1, j, k) * F(u, i + 1, j, k) + 27.0 * F(thx, i, j, k) * F(u, i, j, k) - 27.0 * F(thx, i - 1, j, k) * F(u, i - 1, j, k) + F(thx, i - 2, j, k) * F(u, i - 2, j, k)) / 24.0 / dx;
                    tvy = (-F(thy, i, j + 1, k) * F(v, i, j + 1, k) + 27.0 * F(thy, i, j, k) * F(v, i, j, k) - 27.0 * F(thy, i, j - 1, k) * F(v, i, j - 1, k) + F(thy, i, j - 2, k) * F(v, i, j - 2, k)) / 24.0 / dy;
                    tx = (-F(thx, i + 1, j, k) + 27.0 * F(thx, i, j, k) - 27.0 * F(thx, i - 1, j, k) + F(thx, i - 2, j, k)) / 24.0 / dx;
                }
                double twz = (F(thz, i, j, k) * F(w, i, j, k) - F(thz, i, j, k - 1) * F(w, i, j, k - 1)) / dz[k];
                if (cds == 1) {
                    txx = (F(t, i + 1, j, k) - 2.0 * F(t, i, j, k) + F(t, i - 1, j, k)) / dx2;
                    tyy = (F(t, i, j + 1, k) - 2.0 * F(t, i, j, k) + F(t, i, j - 1, k)) / dy2;
                } else if (cds == 2) {
                    txx = (-F(t, i + 2, j, k) + 16.0 * F(t, i + 1, j, k) - 30.0 * F(t, i, j, k) + 16.0 * F(t, i - 1, j, k) - F(t, i - 2, j, k)) / 12.0 / dx2;
                    tyy = (-F(t, i, j + 2, k) + 16.0 * F(t, i, j + 1, k) - 30.0 * F(t, i, j, k) + 16.0 * F(t, i, j - 1, k) - F(t, i, j - 2, k)) / 12.0 / dy2;
                }
                double tzz = ((F(t, i, j, k + 1) - F(t, i, j, k)) / dz_t[k] - (F(t, i, j, k) - F(t, i, j, k - 1)) / dz_b[k]) / dz[k];
                F(s->ss, i, j, k) = -tux - tvy - twz - um * tx;
                F(qt, i, j, k) = F(t, i, j, k) + dt * (rk_a * F(s->ss, i, j, k) + rk_b * F(s->ss0, i, j, k)) +
                                 rk_c * 0.5 * dt * al * (txx + tyy + tzz);
            }
}

/* get_p_eqn_src (src/module_poisson_solver.f90:127-176) */
static void get_p_eqn_src(or_state* s, double* qp)
{
    double *u = s->u, *v = s->v, *w = s->w;
    for (int k = s->kstr3; k <= s->kend3; ++k)
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i) {
                double dudx = 0, dvdy = 0;
                if (s->prm.cds == 1) {
                    dudx = (F(u, i, j, k) - F(u, i - 1, j, k)) / s->dx;
                    dvdy = (F(v, i, j, k) - F(v, i, j - 1, k)) / s->dy;
                } else if (s->prm.cds == 2) {
                    dudx = (-F(u, i + 1, j, k) + 27.0 * F(u, i, j, k) - 27.0 * F(u, i - 1, j, k) + F(u, i - 2, j, k)) / 24.0 / s->dx;
                    dvdy = (-F(v, i, j + 1, k) + 27.0 * F(v, i, j, k) - 27.0 * F(v, i, j - 1, k) + F(v, i, j - 2, k)) / 24.0 / s->dy;
                }
                double dwdz = (F(w, i, j, k) - F(w, i, j, k - 1)) / s->dz[k];
                F(qp, i, j, k) = (dudx + dvdy + dwdz) / s->prm.dt;
            }
}

/* assign_abc / assign_abc_p (src/module_navier_stokes.f90:523-619) */
static void assign_abc(or_state* s, const double* aa_in, const cplx* bb_in, const double* cc_in, int is_p)
{
    size_t nxy = (size_t)s->nx * s->ny;
    for (int k = 1; k <= s->nka; ++k)
        for (size_t ij = 0; ij < nxy; ++ij) {
            size_t idx = ij + nxy * (size_t)(k - 1);
            if (s->prm.dts == 2) {
                s->aa[idx] = s->rk_c * aa_in[k];
                s->cc[idx] = s->rk_c * cc_in[k];
                s->bb[idx] = is_p ? s->rk_c * bb_in[idx] : 1.0 + s->rk_c * bb_in[idx];
            } else {
                s->aa[idx] = aa_in[k];
                s->cc[idx] = cc_in[k];
                s->bb[idx] = is_p ? bb_in[idx] : 1.0 + bb_in[idx];
            }
        }
}

/* Thomas sweep + flags shared by poisson_solver_fft (src/module_poisson_solver.f90:545-640)
 * and poisson_solver_fft_spec (src/module_spectral.f90:646-741). c_src holds the
 * transformed source (nx,ny,nz); the solution goes to c_out (zeroed first). */
static void thomas_with_flags(or_state* s, cplx* c_src, cplx* c_out, int zstagger, int delnull, int tbnd, int ubnd)
{
    int kmax3 = zstagger == 1 ? s->kend3 - 1 : s->kend3;
    int nx = s->nx, ny = s->ny, nz = s->nz;
    double* aa = s->aa; double* cc = s->cc; cplx* bb = s->bb;
    const int g = 2;
    if (delnull == 1) {
        C(aa, 1, 1, s->kstr3) = 0.0;
        C(cc, 1, 1, s->kstr3) = 0.0;
        C(c_src, 1, 1, 1) = 0.0;
    }
    if (tbnd == 1) {
        double aa_t_zstr = -0.5 * s->rk_c * s->prm.dt * s->prm.alpha / s->dz[s->kstr3] / s->dz_b[s->kstr3];
        if (s->prm.tbc_bot)   /* T(ks-1) = T(ks) - tbot dz_b(ks): the constant part moves to the source */
            C(c_src, 1, 1, 1) = C(c_src, 1, 1, 1) + aa_t_zstr * s->prm.tbot * s->dz_b[s->kstr3];
        else
            C(c_src, 1, 1, 1) = C(c_src, 1, 1, 1) - 2.0 * aa_t_zstr * s->prm.tbot;
        double cc_t_zend = -0.5 * s->rk_c * s->prm.dt * s->prm.alpha / s->dz[s->kend3] / s->dz_t[s->kend3];
        C(c_src, 1, 1, nz) = C(c_src, 1, 1, nz) - 2.0 * cc_t_zend * s->prm.ttop;
    }
    if (ubnd == 1) {
        double aa_u_zstr = -0.5 * s->rk_c * s->prm.dt * s->prm.nu / s->dz[s->kstr3] / s->dz_b[s->kstr3];
        C(c_src, 1, 1, 1) = C(c_src, 1, 1, 1) + 2.0 * aa_u_zstr * s->prm.u_mrf;
        if (s->prm.ochannel == 0) {
            double cc_u_zend = -0.5 * s->rk_c * s->prm.dt * s->prm.nu / s->dz[s->kend3] / s->dz_t[s->kend3];
            C(c_src, 1, 1, nz) = C(c_src, 1, 1, nz) + 2.0 * cc_u_zend * s->prm.u_mrf;
        }
    }
    memset(c_out, 0, sizeof(cplx) * (size_t)nx * ny * nz);
    for (int k = s->kstr3 + 1; k <= kmax3; ++k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                cplx tmp = C(aa, i, j, k) / C(bb, i, j, k - 1);
                C(bb, i, j, k) = C(bb, i, j, k) - C(cc, i, j, k - 1) * tmp;
                C(c_src, i, j, k - g) = C(c_src, i, j, k - g) - C(c_src, i, j, k - g - 1) * tmp;
            }
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) C(c_out, i, j, kmax3 - g) = C(c_src, i, j, kmax3 - g) / C(bb, i, j, kmax3);
    for (int k = kmax3 - 1; k >= s->kstr3; --k)
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i)
                C(c_out, i, j, k - g) = (C(c_src, i, j, k - g) - C(cc, i, j, k) * C(c_out, i, j, k - g + 1)) / C(bb, i, j, k);
}

/* poisson_solver_fft (src/module_poisson_solver.f90:483-658) */
static void poisson_solver_fft(or_state* s, const double* r_src, double* r_var, int zstagger, int delnull, int tbnd, int ubnd)
{
    size_t nf = (size_t)s->nia * s->nja * s->nka;
    for (size_t q = 0; q < nf; ++q) r_var[q] = 0.0;
    for (int k = 1; k <= s->nz; ++k)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) C(s->c_src, i, j, k) = F(r_src, i + 2, j + 2, k + 2);
    mpi_2d_fft(s, s->c_src, -1);
    thomas_with_flags(s, s->c_src, s->c_var, zstagger, delnull, tbnd, ubnd);
    mpi_2d_fft(s, s->c_var, 1);
    int kmax3 = zstagger == 1 ? s->kend3 - 1 : s->kend3;
    for (int k = s->kstr3; k <= kmax3; ++k)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) F(r_var, i + 2, j + 2, k) = creal(C(s->c_var, i, j, k - 2));
}

/* calculate_uvw (src/module_navier_stokes.f90:659-734) */
static void calculate_uvw(or_state* s)
{
    double *u = s->u, *v = s->v, *w = s->w, *phi = s->phi;
    double c = s->rk_c * s->prm.dt;
    for (int k = s->kstr3; k <= s->kend3; ++k)
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i) {
                if (s->prm.cds == 1) F(u, i, j, k) = F(u, i, j, k) - c * (F(phi, i + 1, j, k) - F(phi, i, j, k)) / s->dx;
                else if (s->prm.cds == 2) F(u, i, j, k) = F(u, i, j, k) - c * (-F(phi, i + 2, j, k) + 27.0 * F(phi, i + 1, j, k) - 27.0 * F(phi, i, j, k) + F(phi, i - 1, j, k)) / 24.0 / s->dx;
            }
    for (int k = s->kstr3; k <= s->kend3; ++k)
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i) {
                if (s->prm.cds == 1) F(v, i, j, k) = F(v, i, j, k) - c * (F(phi, i, j + 1, k) - F(phi, i, j, k)) / s->dy;
                else if (s->prm.cds == 2) F(v, i, j, k) = F(v, i, j, k) - c * (-F(phi, i, j + 2, k) + 27.0 * F(phi, i, j + 1, k) - 27.0 * F(phi, i, j, k) + F(phi, i, j - 1, k)) / 24.0 / s->dy;
            }
    for (int k = s->kstr3; k <= s->kend3 - 1; ++k)
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i)
                F(w, i, j, k) = F(w, i, j, k) - c * (F(phi, i, j, k + 1) - F(phi, i, j, k)) / s->dz_t[k];
}

/* calculate_new_p (src/module_navier_stokes.f90:739-808) */
static void calculate_new_p(or_state* s)
{
    double *phi = s->phi, *p = s->p;
    for (int k = s->kstr3; k <= s->kend3; ++k)
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i) {
                double phixx = 0, phiyy = 0;
                if (s->prm.cds == 1) {
                    phixx = (F(phi, i + 1, j, k) - 2.0 * F(phi, i, j, k) + F(phi, i - 1, j, k)) / s->dx2;
                    phiyy = (F(phi, i, j + 1, k) - 2.0 * F(phi, i, j, k) + F(phi, i, j - 1, k)) / s->dy2;
                } else if (s->prm.cds == 2) {
                    phixx = (-F(phi, i + 2, j, k) + 16.0 * F(phi, i + 1, j, k) - 30.0 * F(phi, i, j, k) + 16.0 * F(phi, i - 1, j, k) - F(phi, i - 2, j, k)) / 12.0 / s->dx2;
                    phiyy = (-F(phi, i, j + 2, k) + 16.0 * F(phi, i, j + 1, k) - 30.0 * F(phi, i, j, k) + 16.0 * F(phi, i, j - 1, k) - F(phi, i, j - 2, k)) / 12.0 / s->dy2;
                }
                double phizz = ((F(phi, i, j, k + 1) - F(phi, i, j, k)) / s->dz_t[k] - (F(phi, i, j, k) - F(phi, i, j, k - 1)) / s->dz_b[k]) / s->dz[k];
                F(p, i, j, k) = F(p, i, j, k) + F(phi, i, j, k) - s->rk_c * 0.5 * s->prm.dt * s->prm.nu * (phixx + phiyy + phizz);
            }
}

/* rayleigh_damping (src/module_tools.f90:705-749) */
static void rayleigh_damping(or_state* s, double* var)
{
    int nzd = s->prm.nzdamp;
    for (int k = s->kend3 - nzd; k <= s->kend3; ++k) {
        double ml = 0.0;
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i) ml = ml + F(var, i, j, k);
        ml = ml / s->nx / s->ny;
        double mall = ml / 1;
        double zd = (k - s->kend3 + nzd) * 1.0 / nzd;
        double sigz = s->prm.cdamp * 0.5 * (1.0 - cos(PI * zd));
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i) F(var, i, j, k) = F(var, i, j, k) - sigz * (F(var, i, j, k) - mall);
    }
}

/* calculate_mean_fields (src/module_tools.f90:362-404) and _spec (src/module_spectral.f90:1012-1052) */
static void calculate_mean_fields(or_state* s, int spec)
{
    double um = s->prm.u_mrf;
    double *u = s->u, *v = s->v, *w = s->w, *t = s->t;
    double **m = s->mean;
    for (int k = s->kstr3; k <= s->kend3; ++k)
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i) {
                double wc = 0.5 * (F(w, i, j, k) + F(w, i, j, k - 1));
                F(m[4], i, j, k) = F(m[4], i, j, k) + sq(F(u, i, j, k) + um);
                F(m[5], i, j, k) = F(m[5], i, j, k) + sq(F(v, i, j, k));
                F(m[6], i, j, k) = F(m[6], i, j, k) + sq(F(w, i, j, k));
                if (spec) {
                    F(m[7], i, j, k) = F(m[7], i, j, k) + wc * (F(u, i, j, k) + um);
                    F(m[8], i, j, k) = F(m[8], i, j, k) + wc * F(v, i, j, k);
                } else {
                    F(m[7], i, j, k) = F(m[7], i, j, k) + wc * (F(s->uhx, i, j, k) + um);
                    F(m[8], i, j, k) = F(m[8], i, j, k) + wc * F(s->vhy, i, j, k);
                }
                F(m[9], i, j, k) = F(m[9], i, j, k) + sq(F(t, i, j, k));
                F(m[10], i, j, k) = F(m[10], i, j, k) + F(t, i, j, k) * 0.5 * (F(w, i, j, k) + F(w, i, j, k - 1));
                F(m[0], i, j, k) = F(m[0], i, j, k) + F(u, i, j, k) + um;
                F(m[1], i, j, k) = F(m[1], i, j, k) + F(v, i, j, k);
                F(m[2], i, j, k) = F(m[2], i, j, k) + F(w, i, j, k);
                F(m[3], i, j, k) = F(m[3], i, j, k) + F(t, i, j, k);
            }
}

/* screen_cpu_time CFL part (src/module_io.f90:43-68) */
static void screen_cpu_time(or_state* s)
{
    double cfl = 0.0, dt = s->prm.dt;
    for (int k = s->kstr3; k <= s->kend3; ++k)
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i) {
                double c = dt * fabs(F(s->u, i, j, k)) / s->dx + dt * fabs(F(s->v, i, j, k)) / s->dy +
                           dt * fabs(F(s->w, i, j, k)) / s->dz[k];
                if (c > cfl) cfl = c;
            }
    s->cfl_max = cfl;
    s->time_sim = s->time_sim + dt;
}

static int has_nan3(or_state* s, int i, int j, int k)
{
    return F(s->u, i, j, k) != F(s->u, i, j, k) || F(s->v, i, j, k) != F(s->v, i, j, k) || F(s->w, i, j, k) != F(s->w, i, j, k);
}

/* screen_div_error (src/module_io.f90:85-206); returns 1 on NaN (the reference stops) */
static int screen_div_error(or_state* s, int isfinal, int sub)
{
    double div_avg = 0.0, div_max = 0.0;
    double *u = s->u, *v = s->v, *w = s->w;
    for (int k = s->kstr3; k <= s->kend3; ++k)
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i) {
                double dudx = 0, dvdy = 0;
                if (s->prm.cds == 1) {
                    dudx = (F(u, i, j, k) - F(u, i - 1, j, k)) / s->dx;
                    dvdy = (F(v, i, j, k) - F(v, i, j - 1, k)) / s->dy;
                } else if (s->prm.cds == 2) {
                    dudx = (-F(u, i + 1, j, k) + 27.0 * F(u, i, j, k) - 27.0 * F(u, i - 1, j, k) + F(u, i - 2, j, k)) / 24.0 / s->dx;
                    dvdy = (-F(v, i, j + 1, k) + 27.0 * F(v, i, j, k) - 27.0 * F(v, i, j - 1, k) + F(v, i, j - 2, k)) / 24.0 / s->dy;
                }
                double dwdz = (F(w, i, j, k) - F(w, i, j, k - 1)) / s->dz[k];
                double d = dudx + dvdy + dwdz;
                div_avg = div_avg + fabs(d);
                if (fabs(d) > div_max) div_max = d;
                if (has_nan3(s, i, j, k)) { s->nan_flag = 1; return 1; }
                if (isfinal == 1 && fabs(d) > s->div_hist_max) s->div_hist_max = d;
            }
    div_avg = div_avg / s->nx / s->ny / s->nz;
    s->div_avg_sub[sub] = div_avg;
    s->div_max_sub[sub] = div_max;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* time_advancement_fd (src/module_navier_stokes.f90:223-365)               */
/* ------------------------------------------------------------------------ */
static int time_advancement_fd(or_state* s)
{
    int t_its_max = s->prm.dts == 2 ? 3 : 1;
    size_t nf = (size_t)s->nia * s->nja * s->nka;
    for (int t_its = 1; t_its <= t_its_max; ++t_its) {
        if (s->prm.isdamp == 1) {
            rayleigh_damping(s, s->u); rayleigh_damping(s, s->v); rayleigh_damping(s, s->w);
            rayleigh_damping(s, s->p); rayleigh_damping(s, s->t);
        }
        memcpy(s->ff0, s->ff, nf * sizeof(double));
        memcpy(s->gg0, s->gg, nf * sizeof(double));
        memcpy(s->hh0, s->hh, nf * sizeof(double));
        get_interp_fields_uvwhxyz(s);
        update_boundary_uvwhxyz(s);
        assign_rk_coeff(s, rkc1[t_its - 1], rkc2[t_its - 1], rkc3[t_its - 1]);
        get_momentum_cnvdiff(s);
        assign_abc(s, s->aa_u, s->bb_u, s->cc_u, 0);
        poisson_solver_fft(s, s->qu, s->u, 0, 0, 0, 1);
        assign_abc(s, s->aa_u, s->bb_u, s->cc_u, 0);
        poisson_solver_fft(s, s->qv, s->v, 0, 0, 0, 0);
        assign_abc(s, s->aa_w, s->bb_w, s->cc_w, 0);
        poisson_solver_fft(s, s->qw, s->w, 1, 0, 0, 0);
        update_boundary_uvw(s, s->u, s->v, s->w);
        get_p_eqn_src(s, s->qu);
        assign_abc(s, s->aa_p, s->bb_p, s->cc_p, 1);
        poisson_solver_fft(s, s->qu, s->phi, 0, 1, 0, 0);
        update_boundary_p(s, s->phi);
        calculate_uvw(s);
        update_boundary_uvw(s, s->u, s->v, s->w);
        if (s->prm.isscalar == 1) {
            memcpy(s->ss0, s->ss, nf * sizeof(double));
            get_interp_fields_thxyz(s);
            update_boundary_thxyz(s);
            get_temperature_cnvdiff(s, s->qu);
            assign_abc(s, s->aa_t, s->bb_t, s->cc_t, 0);
            poisson_solver_fft(s, s->qu, s->t, 0, 0, 1, 0);
            update_boundary_t(s, s->t);
        }
        if (screen_div_error(s, 1, t_its - 1)) return 1;
        calculate_new_p(s);
        update_boundary_p(s, s->p);
    }
    calculate_mean_fields(s, 0);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* spectral helpers (src/module_spectral.f90)                               */
/* ------------------------------------------------------------------------ */
/* dev_fft_linear_cmplx :1274-1340 */
static void dev_fft_linear_cmplx(or_state* s, const cplx* in, cplx* out, int ord, int dir)
{
    for (int k = 1; k <= s->nz; ++k)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) {
                int l = lmap(i, s->nx), m = lmap(j, s->ny);
                cplx c = C(in, i, j, k);
                if (ord == 1 && dir == 1) c = c * I * 2.0 * PI / s->prm.lx * l;
                else if (ord == 1 && dir == 2) c = c * I * 2.0 * PI / s->prm.ly * m;
                else if (ord == 2 && dir == 1) c = -c * sq(2.0 * PI / s->prm.lx * l);
                else c = -c * sq(2.0 * PI / s->prm.ly * m);
                if (l == -s->nx / 2 || m == -s->ny / 2) c = 0.0;
                C(out, i, j, k) = c;
            }
}

/* dev_fft_nonlinear_cmplx :1061-1150 */
static void dev_fft_nonlinear_cmplx(or_state* s, const double* r1, const double* r2, cplx* out, int dir, int weqn)
{
    for (int k = 1; k <= s->nz; ++k)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) {
                if (weqn == 1) {
                    double tmp1 = F(r1, i + 2, j + 2, k + 1 + 2) * s->l_t[k + 2] + F(r1, i + 2, j + 2, k + 2) * (1.0 - s->l_t[k + 2]);
                    C(out, i, j, k) = tmp1 * F(r2, i + 2, j + 2, k + 2);
                } else {
                    C(out, i, j, k) = F(r1, i + 2, j + 2, k + 2) * F(r2, i + 2, j + 2, k + 2);
                }
            }
    mpi_2d_fft(s, out, -1);
    for (int k = 1; k <= s->nz; ++k)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) {
                int l = lmap(i, s->nx), m = lmap(j, s->ny);
                if (dir == 1) C(out, i, j, k) = C(out, i, j, k) * I * 2.0 * PI / s->prm.lx * l;
                else C(out, i, j, k) = C(out, i, j, k) * I * 2.0 * PI / s->prm.ly * m;
                if (l == -s->nx / 2 || m == -s->ny / 2) C(out, i, j, k) = 0.0;
            }
}

/* real_2_cmplx :1157-1182 */
static void real_2_cmplx(or_state* s, const double* r, cplx* c)
{
    for (int k = 1; k <= s->nz; ++k)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) C(c, i, j, k) = F(r, i + 2, j + 2, k + 2);
    mpi_2d_fft(s, c, -1);
}

/* cmplx_2_real :1188-1217 */
static void cmplx_2_real(or_state* s, const cplx* c, double* r)
{
    size_t n = (size_t)s->nx * s->ny * s->nz;
    memcpy(s->c_var, c, n * sizeof(cplx));
    mpi_2d_fft(s, s->c_var, 1);
    for (int k = 1; k <= s->nz; ++k)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) F(r, i + 2, j + 2, k + 2) = creal(C(s->c_var, i, j, k));
}

/* spectral_truncation :1222-1268 (2/3 rule) */
static void spectral_truncation(or_state* s, cplx* c)
{
    int lx3 = (int)(s->nx / 3.0), ly3 = (int)(s->ny / 3.0);
    for (int k = 1; k <= s->nz; ++k)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) {
                int l = lmap(i, s->nx), m = lmap(j, s->ny);
                if (l >= lx3 || l <= -lx3) C(c, i, j, k) = 0.0;
                if (m >= ly3 || m <= -ly3) C(c, i, j, k) = 0.0;
            }
}

/* rayleigh_damping_spec :1345-1391 */
static void rayleigh_damping_spec(or_state* s, cplx* c)
{
    int nzd = s->prm.nzdamp;
    for (int k = s->kend3 - nzd; k <= s->kend3; ++k) {
        cplx ml = 0.0;
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i) ml = ml + C(c, i - 2, j - 2, k - 2);
        ml = ml / (double)s->nx / (double)s->ny;
        double mall_re = creal(ml) / 1;      /* MPI_ALLREDUCE of count 1, real_type: real part only */
        cplx mall = mall_re;
        double zd = (k - s->kend3 + nzd) * 1.0 / nzd;
        double sigz = s->prm.cdamp * 0.5 * (1.0 - cos(PI * zd));
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i)
                C(c, i - 2, j - 2, k - 2) = C(c, i - 2, j - 2, k - 2) - sigz * (C(c, i - 2, j - 2, k - 2) - mall);
    }
}

static void cadd(or_state* s, cplx* a, const cplx* b, double f)
{
    size_t n = (size_t)s->nx * s->ny * s->nz;
    for (size_t q = 0; q < n; ++q) a[q] = a[q] + f * b[q];
}

#define PHYS_LOOP for (int k = s->kstr3; k <= s->kend3; ++k) for (int j = s->jstr3; j <= s->jend3; ++j) for (int i = s->istr3; i <= s->iend3; ++i)

/* get_momentum_cnvdiff_spec :35-504 */
static void get_momentum_cnvdiff_spec(or_state* s)
{
    double coe_sk = s->prm.issk == 1 ? 0.5 : 1.0;
    double dt = s->prm.dt, nu = s->prm.nu, um = s->prm.u_mrf, fc = s->prm.fc;
    double rk_a = s->rk_a, rk_b = s->rk_b, rk_c = s->rk_c;
    size_t n = (size_t)s->nx * s->ny * s->nz;
    double *u = s->u, *v = s->v, *w = s->w, *p = s->p, *t = s->t;
    double *dz = s->dz, *dz_t = s->dz_t, *dz_b = s->dz_b, *l_t = s->l_t, *l_b = s->l_b;
    cplx *cv = s->c_var, *cs = s->c_src;
    update_dpx_drive(s);

    /* ---- U ---- */
    memcpy(s->c_qu, s->c_u, n * sizeof(cplx));
    dev_fft_linear_cmplx(s, s->c_u, cv, 2, 1); cadd(s, s->c_qu, cv, rk_c * 0.5 * dt * nu);
    dev_fft_linear_cmplx(s, s->c_u, cv, 2, 2); cadd(s, s->c_qu, cv, rk_c * 0.5 * dt * nu);
    PHYS_LOOP {
        double tmp1 = ((F(u, i, j, k + 1) - F(u, i, j, k)) / dz_t[k] - (F(u, i, j, k) - F(u, i, j, k - 1)) / dz_b[k]) / dz[k];
        C(cv, i - 2, j - 2, k - 2) = tmp1;
    }
    mpi_2d_fft(s, cv, -1); cadd(s, s->c_qu, cv, rk_c * 0.5 * dt * nu);
    dev_fft_linear_cmplx(s, s->c_p, cv, 1, 1); cadd(s, s->c_qu, cv, -rk_c * dt);
    cadd(s, s->c_qu, s->c_ff, rk_b * dt);
    memset(s->c_ff, 0, n * sizeof(cplx));
    dev_fft_linear_cmplx(s, s->c_u, cv, 1, 1); cadd(s, s->c_ff, cv, -um);
    dev_fft_nonlinear_cmplx(s, u, u, cv, 1, 0); cadd(s, s->c_ff, cv, -coe_sk);
    dev_fft_nonlinear_cmplx(s, u, v, cv, 2, 0); cadd(s, s->c_ff, cv, -coe_sk);
    PHYS_LOOP {
        double a1 = F(u, i, j, k + 1) * l_t[k] + F(u, i, j, k) * (1.0 - l_t[k]);
        double a2 = F(u, i, j, k - 1) * l_b[k] + F(u, i, j, k) * (1.0 - l_b[k]);
        double tmp1 = (a1 * F(w, i, j, k) - a2 * F(w, i, j, k - 1)) / dz[k];
        double tmp2 = s->prm.dp_opt == 3 ? fc * (F(v, i, j, k) - s->prm.vg) : s->dpx_drive;
        C(cv, i - 2, j - 2, k - 2) = 1.0 / coe_sk * tmp2 - tmp1;
    }
    mpi_2d_fft(s, cv, -1); cadd(s, s->c_ff, cv, coe_sk);
    if (s->prm.issk == 1) {
        dev_fft_linear_cmplx(s, s->c_u, cs, 1, 1); mpi_2d_fft(s, cs, 1);
        PHYS_LOOP { C(cv, i - 2, j - 2, k - 2) = F(u, i, j, k) * creal(C(cs, i - 2, j - 2, k - 2)); }
        mpi_2d_fft(s, cv, -1); cadd(s, s->c_ff, cv, -coe_sk);
        dev_fft_linear_cmplx(s, s->c_u, cs, 1, 2); mpi_2d_fft(s, cs, 1);
        PHYS_LOOP { C(cv, i - 2, j - 2, k - 2) = F(v, i, j, k) * creal(C(cs, i - 2, j - 2, k - 2)); }
        mpi_2d_fft(s, cv, -1); cadd(s, s->c_ff, cv, -coe_sk);
        PHYS_LOOP {
            double a1 = F(u, i, j, k + 1) * l_t[k] + F(u, i, j, k) * (1.0 - l_t[k]);
            double a2 = F(u, i, j, k - 1) * l_b[k] + F(u, i, j, k) * (1.0 - l_b[k]);
            double tmp1 = (a1 - a2) / dz[k];
            double tmp2 = 0.5 * (F(w, i, j, k) + F(w, i, j, k - 1));
            C(cv, i - 2, j - 2, k - 2) = tmp1 * tmp2;
        }
        mpi_2d_fft(s, cv, -1); cadd(s, s->c_ff, cv, -coe_sk);
    }
    if (s->bfx) { real_2_cmplx(s, s->bfx, cv); cadd(s, s->c_ff, cv, 1.0); }
    cadd(s, s->c_qu, s->c_ff, rk_a * dt);

    /* ---- V ---- */
    memcpy(s->c_qv, s->c_v, n * sizeof(cplx));
    dev_fft_linear_cmplx(s, s->c_v, cv, 2, 1); cadd(s, s->c_qv, cv, rk_c * 0.5 * dt * nu);
    dev_fft_linear_cmplx(s, s->c_v, cv, 2, 2); cadd(s, s->c_qv, cv, rk_c * 0.5 * dt * nu);
    PHYS_LOOP {
        double tmp1 = ((F(v, i, j, k + 1) - F(v, i, j, k)) / dz_t[k] - (F(v, i, j, k) - F(v, i, j, k - 1)) / dz_b[k]) / dz[k];
        C(cv, i - 2, j - 2, k - 2) = tmp1;
    }
    mpi_2d_fft(s, cv, -1); cadd(s, s->c_qv, cv, rk_c * 0.5 * dt * nu);
    dev_fft_linear_cmplx(s, s->c_p, cv, 1, 2); cadd(s, s->c_qv, cv, -rk_c * dt);
    cadd(s, s->c_qv, s->c_gg, rk_b * dt);
    memset(s->c_gg, 0, n * sizeof(cplx));
    dev_fft_linear_cmplx(s, s->c_v, cv, 1, 1); cadd(s, s->c_gg, cv, -um);
    dev_fft_nonlinear_cmplx(s, u, v, cv, 1, 0); cadd(s, s->c_gg, cv, -coe_sk);
    dev_fft_nonlinear_cmplx(s, v, v, cv, 2, 0); cadd(s, s->c_gg, cv, -coe_sk);
    PHYS_LOOP {
        double a1 = F(v, i, j, k + 1) * l_t[k] + F(v, i, j, k) * (1.0 - l_t[k]);
        double a2 = F(v, i, j, k - 1) * l_b[k] + F(v, i, j, k) * (1.0 - l_b[k]);
        double tmp1 = (a1 * F(w, i, j, k) - a2 * F(w, i, j, k - 1)) / dz[k];
        double tmp2 = s->prm.dp_opt == 3 ? fc * (s->prm.ug - F(u, i, j, k) - um) : 0.0;
        C(cv, i - 2, j - 2, k - 2) = 1.0 / coe_sk * tmp2 - tmp1;
    }
    mpi_2d_fft(s, cv, -1); cadd(s, s->c_gg, cv, coe_sk);
    if (s->prm.issk == 1) {
        dev_fft_linear_cmplx(s, s->c_v, cs, 1, 1); mpi_2d_fft(s, cs, 1);
        PHYS_LOOP { C(cv, i - 2, j - 2, k - 2) = F(u, i, j, k) * creal(C(cs, i - 2, j - 2, k - 2)); }
        mpi_2d_fft(s, cv, -1); cadd(s, s->c_gg, cv, -coe_sk);
        dev_fft_linear_cmplx(s, s->c_v, cs, 1, 2); mpi_2d_fft(s, cs, 1);
        PHYS_LOOP { C(cv, i - 2, j - 2, k - 2) = F(v, i, j, k) * creal(C(cs, i - 2, j - 2, k - 2)); }
        mpi_2d_fft(s, cv, -1); cadd(s, s->c_gg, cv, -coe_sk);
        PHYS_LOOP {
            double a1 = F(v, i, j, k + 1) * l_t[k] + F(v, i, j, k) * (1.0 - l_t[k]);
            double a2 = F(v, i, j, k - 1) * l_b[k] + F(v, i, j, k) * (1.0 - l_b[k]);
            double tmp1 = (a1 - a2) / dz[k];
            double tmp2 = 0.5 * (F(w, i, j, k) + F(w, i, j, k - 1));
            C(cv, i - 2, j - 2, k - 2) = tmp1 * tmp2;
        }
        mpi_2d_fft(s, cv, -1); cadd(s, s->c_gg, cv, -coe_sk);
    }
    if (s->bfx) { real_2_cmplx(s, s->bfy, cv); cadd(s, s->c_gg, cv, 1.0); }
    cadd(s, s->c_qv, s->c_gg, rk_a * dt);

    /* ---- W ---- */
    memcpy(s->c_qw, s->c_w, n * sizeof(cplx));
    dev_fft_linear_cmplx(s, s->c_w, cv, 2, 1); cadd(s, s->c_qw, cv, rk_c * 0.5 * dt * nu);
    dev_fft_linear_cmplx(s, s->c_w, cv, 2, 2); cadd(s, s->c_qw, cv, rk_c * 0.5 * dt * nu);
    PHYS_LOOP {
        double tmp1 = ((F(w, i, j, k + 1) - F(w, i, j, k)) / dz[k + 1] - (F(w, i, j, k) - F(w, i, j, k - 1)) / dz[k]) / dz_t[k];
        C(cv, i - 2, j - 2, k - 2) = tmp1;
    }
    mpi_2d_fft(s, cv, -1); cadd(s, s->c_qw, cv, rk_c * 0.5 * dt * nu);
    PHYS_LOOP { C(cv, i - 2, j - 2, k - 2) = (F(p, i, j, k + 1) - F(p, i, j, k)) / dz_t[k]; }
    mpi_2d_fft(s, cv, -1); cadd(s, s->c_qw, cv, -rk_c * dt);
    cadd(s, s->c_qw, s->c_hh, rk_b * dt);
    memset(s->c_hh, 0, n * sizeof(cplx));
    dev_fft_linear_cmplx(s, s->c_w, cv, 1, 1); cadd(s, s->c_hh, cv, -um);
    dev_fft_nonlinear_cmplx(s, u, w, cv, 1, 1); cadd(s, s->c_hh, cv, -coe_sk);
    dev_fft_nonlinear_cmplx(s, v, w, cv, 2, 1); cadd(s, s->c_hh, cv, -coe_sk);
    PHYS_LOOP {
        double a1 = sq(0.5 * (F(w, i, j, k) + F(w, i, j, k + 1)));
        double a2 = sq(0.5 * (F(w, i, j, k) + F(w, i, j, k - 1)));
        double tmp1 = (a1 - a2) / dz_t[k];
        if (s->prm.isscalar == 1) {
            double tmp2 = s->got * ((1.0 - l_t[k]) * F(t, i, j, k) + l_t[k] * F(t, i, j, k + 1) - s->prm.t_ref);
            C(cv, i - 2, j - 2, k - 2) = 1.0 / coe_sk * tmp2 - tmp1;
        } else {
            C(cv, i - 2, j - 2, k - 2) = -tmp1;
        }
    }
    mpi_2d_fft(s, cv, -1); cadd(s, s->c_hh, cv, coe_sk);
    if (s->prm.issk == 1) {
        dev_fft_linear_cmplx(s, s->c_w, cs, 1, 1); mpi_2d_fft(s, cs, 1);
        PHYS_LOOP {
            double tmp1 = l_t[k] * F(u, i, j, k + 1) + (1.0 - l_t[k]) * F(u, i, j, k);
            C(cv, i - 2, j - 2, k - 2) = tmp1 * creal(C(cs, i - 2, j - 2, k - 2));
        }
        mpi_2d_fft(s, cv, -1); cadd(s, s->c_hh, cv, -coe_sk);
        dev_fft_linear_cmplx(s, s->c_w, cs, 1, 2); mpi_2d_fft(s, cs, 1);
        PHYS_LOOP {
            double tmp1 = l_t[k] * F(v, i, j, k + 1) + (1.0 - l_t[k]) * F(v, i, j, k);
            C(cv, i - 2, j - 2, k - 2) = tmp1 * creal(C(cs, i - 2, j - 2, k - 2));
        }
        mpi_2d_fft(s, cv, -1); cadd(s, s->c_hh, cv, -coe_sk);
        PHYS_LOOP {
            double a1 = 0.5 * (F(w, i, j, k) + F(w, i, j, k + 1));
            double a2 = 0.5 * (F(w, i, j, k) + F(w, i, j, k - 1));
            double tmp1 = (a1 - a2) / dz_t[k];
            C(cv, i - 2, j - 2, k - 2) = F(w, i, j, k) * tmp1;
        }
        mpi_2d_fft(s, cv, -1); cadd(s, s->c_hh, cv, -coe_sk);
    }
    if (s->bfx) { real_2_cmplx(s, s->bfz, cv); cadd(s, s->c_hh, cv, 1.0); }
    cadd(s, s->c_qw, s->c_hh, rk_a * dt);
}

/* get_temperature_cnvdiff_spec :509-595 */
static void get_temperature_cnvdiff_spec(or_state* s)
{
    double dt = s->prm.dt, al = s->prm.alpha, um = s->prm.u_mrf;
    double rk_a = s->rk_a, rk_b = s->rk_b, rk_c = s->rk_c;
    size_t n = (size_t)s->nx * s->ny * s->nz;
    double *u = s->u, *v = s->v, *w = s->w, *t = s->t;
    double *dz = s->dz, *dz_t = s->dz_t, *dz_b = s->dz_b, *l_t = s->l_t, *l_b = s->l_b;
    cplx* cv = s->c_var;
    cplx* cq = s->c_qu;
    memcpy(cq, s->c_t, n * sizeof(cplx));
    dev_fft_linear_cmplx(s, s->c_t, cv, 2, 1); cadd(s, cq, cv, rk_c * 0.5 * dt * al);
    dev_fft_linear_cmplx(s, s->c_t, cv, 2, 2); cadd(s, cq, cv, rk_c * 0.5 * dt * al);
    PHYS_LOOP {
        double tmp1 = ((F(t, i, j, k + 1) - F(t, i, j, k)) / dz_t[k] - (F(t, i, j, k) - F(t, i, j, k - 1)) / dz_b[k]) / dz[k];
        C(cv, i - 2, j - 2, k - 2) = tmp1;
    }
    mpi_2d_fft(s, cv, -1); cadd(s, cq, cv, rk_c * 0.5 * dt * al);
    cadd(s, cq, s->c_ss, rk_b * dt);
    memset(s->c_ss, 0, n * sizeof(cplx));
    dev_fft_linear_cmplx(s, s->c_t, cv, 1, 1); cadd(s, s->c_ss, cv, -um);
    dev_fft_nonlinear_cmplx(s, u, t, cv, 1, 0); cadd(s, s->c_ss, cv, -1.0);
    dev_fft_nonlinear_cmplx(s, t, v, cv, 2, 0); cadd(s, s->c_ss, cv, -1.0);
    PHYS_LOOP {
        double a1 = F(t, i, j, k + 1) * l_t[k] + F(t, i, j, k) * (1.0 - l_t[k]);
        double a2 = F(t, i, j, k - 1) * l_b[k] + F(t, i, j, k) * (1.0 - l_b[k]);
        C(cv, i - 2, j - 2, k - 2) = (a1 * F(w, i, j, k) - a2 * F(w, i, j, k - 1)) / dz[k];
    }
    mpi_2d_fft(s, cv, -1); cadd(s, s->c_ss, cv, -1.0);
    cadd(s, cq, s->c_ss, rk_a * dt);
}

/* poisson_solver_fft_spec :602-746 */
static void poisson_solver_fft_spec(or_state* s, const cplx* src_in, cplx* out, int zstagger, int delnull, int tbnd, int ubnd)
{
    size_t n = (size_t)s->nx * s->ny * s->nz;
    memcpy(s->c_src, src_in, n * sizeof(cplx));
    thomas_with_flags(s, s->c_src, out, zstagger, delnull, tbnd, ubnd);
}

/* get_div_spec :752-795 */
static void get_div_spec(or_state* s, const cplx* cu, const cplx* cvv, cplx* cdiv)
{
    cplx* cv = s->c_var;
    dev_fft_linear_cmplx(s, cu, cv, 1, 1);
    size_t n = (size_t)s->nx * s->ny * s->nz;
    memcpy(cdiv, cv, n * sizeof(cplx));
    dev_fft_linear_cmplx(s, cvv, cv, 1, 2);
    cadd(s, cdiv, cv, 1.0);
    PHYS_LOOP { C(cv, i - 2, j - 2, k - 2) = (F(s->w, i, j, k) - F(s->w, i, j, k - 1)) / s->dz[k]; }
    mpi_2d_fft(s, cv, -1);
    cadd(s, cdiv, cv, 1.0);
}

/* calculate_uvw_spec :801-849 */
static void calculate_uvw_spec(or_state* s)
{
    cplx* cv = s->c_var;
    double c = s->rk_c * s->prm.dt;
    dev_fft_linear_cmplx(s, s->c_phi, cv, 1, 1); cadd(s, s->c_u, cv, -c);
    dev_fft_linear_cmplx(s, s->c_phi, cv, 1, 2); cadd(s, s->c_v, cv, -c);
    for (int k = s->kstr3; k <= s->kend3 - 1; ++k)
        for (int j = s->jstr3; j <= s->jend3; ++j)
            for (int i = s->istr3; i <= s->iend3; ++i)
                C(cv, i - 2, j - 2, k - 2) = (F(s->phi, i, j, k + 1) - F(s->phi, i, j, k)) / s->dz_t[k];
    mpi_2d_fft(s, cv, -1);
    for (int k = 1; k <= s->nz - 1; ++k)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) C(s->c_w, i, j, k) = C(s->c_w, i, j, k) - c * C(cv, i, j, k);
}

/* calculate_new_p_spec :854-894 */
static void calculate_new_p_spec(or_state* s)
{
    cplx* cv = s->c_var;
    double c = s->rk_c * 0.5 * s->prm.dt * s->prm.nu;
    cadd(s, s->c_p, s->c_phi, 1.0);
    dev_fft_linear_cmplx(s, s->c_phi, cv, 2, 1); cadd(s, s->c_p, cv, -c);
    dev_fft_linear_cmplx(s, s->c_phi, cv, 2, 2); cadd(s, s->c_p, cv, -c);
    PHYS_LOOP {
        double d2 = ((F(s->phi, i, j, k + 1) - F(s->phi, i, j, k)) / s->dz_t[k] - (F(s->phi, i, j, k) - F(s->phi, i, j, k - 1)) / s->dz_b[k]) / s->dz[k];
        C(cv, i - 2, j - 2, k - 2) = d2;
    }
    mpi_2d_fft(s, cv, -1); cadd(s, s->c_p, cv, -c);
}

/* screen_div_error_spec :899-1007 */
static int screen_div_error_spec(or_state* s, int isfinal, int sub)
{
    get_div_spec(s, s->c_u, s->c_v, s->c_src);
    mpi_2d_fft(s, s->c_src, 1);
    double div_avg = 0.0, div_max = 0.0;
    PHYS_LOOP {
        double tmp1 = creal(C(s->c_src, i - 2, j - 2, k - 2));
        div_avg = div_avg + fabs(tmp1);
        if (fabs(tmp1) > div_max) div_max = fabs(tmp1);
        if (has_nan3(s, i, j, k)) { s->nan_flag = 1; return 1; }
        if (isfinal == 1 && fabs(tmp1) > s->div_hist_max) s->div_hist_max = fabs(tmp1);
    }
    div_avg = div_avg / s->nx / s->ny / s->nz;
    s->div_avg_sub[sub] = div_avg;
    s->div_max_sub[sub] = div_max;
    return 0;
}

/* time_advancement_sp (src/module_navier_stokes.f90:371-517) */
static int time_advancement_sp(or_state* s)
{
    int t_its_max = s->prm.dts == 2 ? 3 : 1;
    size_t n = (size_t)s->nx * s->ny * s->nz;
    for (int t_its = 1; t_its <= t_its_max; ++t_its) {
        if (s->prm.isdamp == 1) {
            rayleigh_damping_spec(s, s->c_u); rayleigh_damping_spec(s, s->c_v); rayleigh_damping_spec(s, s->c_w);
            rayleigh_damping_spec(s, s->c_p); rayleigh_damping_spec(s, s->c_t);
        }
        assign_rk_coeff(s, rkc1[t_its - 1], rkc2[t_its - 1], rkc3[t_its - 1]);
        get_momentum_cnvdiff_spec(s);
        assign_abc(s, s->aa_u, s->bb_u, s->cc_u, 0);
        poisson_solver_fft_spec(s, s->c_qu, s->c_u, 0, 0, 0, 1);
        assign_abc(s, s->aa_u, s->bb_u, s->cc_u, 0);
        poisson_solver_fft_spec(s, s->c_qv, s->c_v, 0, 0, 0, 0);
        assign_abc(s, s->aa_w, s->bb_w, s->cc_w, 0);
        poisson_solver_fft_spec(s, s->c_qw, s->c_w, 1, 0, 0, 0);
        cmplx_2_real(s, s->c_w, s->w);
        update_boundary_uvw(s, s->u, s->v, s->w);
        get_div_spec(s, s->c_u, s->c_v, s->c_qu);
        for (size_t q = 0; q < n; ++q) s->c_qu[q] = s->c_qu[q] / s->prm.dt;
        assign_abc(s, s->aa_p, s->bb_p, s->cc_p, 1);
        poisson_solver_fft_spec(s, s->c_qu, s->c_phi, 0, 1, 0, 0);
        cmplx_2_real(s, s->c_phi, s->phi);
        update_boundary_p(s, s->phi);
        calculate_new_p_spec(s);
        calculate_uvw_spec(s);
        spectral_truncation(s, s->c_u); spectral_truncation(s, s->c_v);
        spectral_truncation(s, s->c_w); spectral_truncation(s, s->c_p);
        cmplx_2_real(s, s->c_u, s->u); cmplx_2_real(s, s->c_v, s->v);
        cmplx_2_real(s, s->c_w, s->w); cmplx_2_real(s, s->c_p, s->p);
        update_boundary_p(s, s->p);
        update_boundary_uvw(s, s->u, s->v, s->w);
        if (s->prm.isscalar == 1) {
            get_temperature_cnvdiff_spec(s);
            assign_abc(s, s->aa_t, s->bb_t, s->cc_t, 0);
            poisson_solver_fft_spec(s, s->c_qu, s->c_t, 0, 0, 1, 0);
            spectral_truncation(s, s->c_t);
            cmplx_2_real(s, s->c_t, s->t);
            update_boundary_t(s, s->t);
        }
        if (screen_div_error_spec(s, 1, t_its - 1)) return 1;
    }
    calculate_mean_fields(s, 1);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* public API                                                               */
/* ------------------------------------------------------------------------ */
static double* dalloc(size_t n) { return (double*)calloc(n, sizeof(double)); }
static cplx* calloc_c(size_t n) { return (cplx*)calloc(n, sizeof(cplx)); }

or_state* or_create(const hc_params* prm, int* err)
{
    if (err) *err = 0;
    if (!prm) { if (err) *err = HC_ERR_ARG; return NULL; }
    /* initiate_parameters checks (src/module_parameters.f90:266-270) */
    if (prm->nx % 2 != 0 || prm->ny % 2 != 0 || prm->nx < 4 || prm->ny < 4 || prm->nz < 3 ||
        (prm->cds < 1 || prm->cds > 3) || (prm->dts != 1 && prm->dts != 2) ||
        (prm->isscalar != 0 && prm->isscalar != 1) || (prm->tbc_bot != 0 && prm->tbc_bot != 1)) {
        if (err) *err = HC_ERR_PARAM;
        return NULL;
    }
    or_state* s = (or_state*)calloc(1, sizeof(or_state));
    s->prm = *prm;
    s->nx = prm->nx; s->ny = prm->ny; s->nz = prm->nz;
    s->nia = s->nx + 4; s->nja = s->ny + 4; s->nka = s->nz + 4;
    s->istr3 = 3; s->iend3 = s->nx + 2; s->jstr3 = 3; s->jend3 = s->ny + 2; s->kstr3 = 3; s->kend3 = s->nz + 2;
    s->dx = prm->lx / s->nx; s->dy = prm->ly / s->ny;
    s->dx2 = s->dx * s->dx; s->dy2 = s->dy * s->dy;
    s->dpx_coef = prm->nu * 1.0;
    s->wx1 = cexp(I * 2.0 * PI / s->nx);
    s->wy1 = cexp(I * 2.0 * PI / s->ny);
    s->got = prm->got;
    if (prm->dp_opt == 1) s->dpx_drive = 1.0; else { s->dpx_drive = 0.0; s->ubar = 0.0; }
    size_t nf = (size_t)s->nia * s->nja * s->nka;
    size_t nb = (size_t)s->nx * s->ny * s->nka;
    size_t nc = (size_t)s->nx * s->ny * s->nz;
    s->dz = dalloc(s->nka + 2); s->l_t = dalloc(s->nka + 2); s->l_b = dalloc(s->nka + 2);
    s->dz_t = dalloc(s->nka + 2); s->dz_b = dalloc(s->nka + 2);
    double** fl[] = {&s->u, &s->v, &s->w, &s->p, &s->phi, &s->t, &s->ff, &s->gg, &s->hh, &s->ss,
                     &s->ff0, &s->gg0, &s->hh0, &s->ss0, &s->qu, &s->qv, &s->qw,
                     &s->uhx, &s->uhy, &s->uhz, &s->vhx, &s->vhy, &s->vhz, &s->whx, &s->why,
                     &s->thx, &s->thy, &s->thz};
    for (size_t q = 0; q < sizeof(fl) / sizeof(fl[0]); ++q) *fl[q] = dalloc(nf);
    for (int q = 0; q < 11; ++q) s->mean[q] = dalloc(nf);
    s->aa = dalloc(nb); s->cc = dalloc(nb); s->bb = calloc_c(nb);
    double** al[] = {&s->aa_u, &s->cc_u, &s->aa_w, &s->cc_w, &s->aa_p, &s->cc_p, &s->aa_t, &s->cc_t};
    for (int q = 0; q < 8; ++q) *al[q] = dalloc(s->nka + 2);
    s->bb_u = calloc_c(nb); s->bb_w = calloc_c(nb); s->bb_p = calloc_c(nb); s->bb_t = calloc_c(nb);
    s->c_src = calloc_c(nc); s->c_var = calloc_c(nc);
    if (prm->cds == 3) {
        cplx** cl[] = {&s->c_u, &s->c_v, &s->c_w, &s->c_p, &s->c_phi, &s->c_t, &s->c_qu, &s->c_qv, &s->c_qw,
                       &s->c_ff, &s->c_gg, &s->c_hh, &s->c_ss};
        for (int q = 0; q < 13; ++q) *cl[q] = calloc_c(nc);
    }
    plan_init(&s->px, s->nx);
    plan_init(&s->py, s->ny);
    get_mesh_param(s);
    get_u_eqn_coeff(s, s->aa_u, s->bb_u, s->cc_u);
    get_w_eqn_coeff(s, s->aa_w, s->bb_w, s->cc_w);
    get_p_eqn_coeff(s, s->aa_p, s->bb_p, s->cc_p);
    get_t_eqn_coeff(s, s->aa_t, s->bb_t, s->cc_t);
    return s;
}

void or_destroy(or_state* s)
{
    if (!s) return;
    double* fl[] = {s->u, s->v, s->w, s->p, s->phi, s->t, s->ff, s->gg, s->hh, s->ss, s->ff0, s->gg0, s->hh0, s->ss0,
                    s->qu, s->qv, s->qw, s->uhx, s->uhy, s->uhz, s->vhx, s->vhy, s->vhz, s->whx, s->why,
                    s->thx, s->thy, s->thz, s->aa, s->cc, s->aa_u, s->cc_u, s->aa_w, s->cc_w, s->aa_p, s->cc_p,
                    s->aa_t, s->cc_t, s->dz, s->l_t, s->l_b, s->dz_t, s->dz_b};
    for (size_t q = 0; q < sizeof(fl) / sizeof(fl[0]); ++q) free(fl[q]);
    for (int q = 0; q < 11; ++q) free(s->mean[q]);
    cplx* cl[] = {s->bb, s->bb_u, s->bb_w, s->bb_p, s->bb_t, s->c_src, s->c_var, s->c_u, s->c_v, s->c_w, s->c_p,
                  s->c_phi, s->c_t, s->c_qu, s->c_qv, s->c_qw, s->c_ff, s->c_gg, s->c_hh, s->c_ss};
    for (size_t q = 0; q < sizeof(cl) / sizeof(cl[0]); ++q) free(cl[q]);
    free(s->bfx); free(s->bfy); free(s->bfz);
    plan_free(&s->px);
    plan_free(&s->py);
    free(s);
}

/* Body force (no reference counterpart): a field added to ff, gg, hh of the
 * momentum equations (the FD right-hand side and the spectral histories alike).
 * NULL for all three removes it; a NULL component is zero. */
int or_set_body_force(or_state* s, const double* fx, const double* fy, const double* fz)
{
    free(s->bfx); free(s->bfy); free(s->bfz);
    s->bfx = s->bfy = s->bfz = NULL;
    if (!fx && !fy && !fz) return 0;
    size_t nf = (size_t)s->nia * s->nja * s->nka;
    double** dst[3] = {&s->bfx, &s->bfy, &s->bfz};
    const double* src[3] = {fx, fy, fz};
    for (int c = 0; c < 3; ++c) {
        *dst[c] = (double*)calloc(nf, sizeof(double));
        if (!src[c]) continue;
        size_t q = 0;
        for (int k = 1; k <= s->nz; ++k)
            for (int j = 1; j <= s->ny; ++j)
                for (int i = 1; i <= s->nx; ++i) F(*dst[c], i + 2, j + 2, k + 2) = src[c][q++];
    }
    return 0;
}

int or_get_grid(or_state* s, double* dz, double* l_t, double* l_b, double* dz_t, double* dz_b)
{
    for (int k = 1; k <= s->nka; ++k) {
        if (dz) dz[k - 1] = s->dz[k];
        if (l_t) l_t[k - 1] = s->l_t[k];
        if (l_b) l_b[k - 1] = s->l_b[k];
        if (dz_t) dz_t[k - 1] = s->dz_t[k];
        if (dz_b) dz_b[k - 1] = s->dz_b[k];
    }
    return 0;
}

static double* field_ptr(or_state* s, int id)
{
    switch (id) {
    case HC_FIELD_U: return s->u;
    case HC_FIELD_V: return s->v;
    case HC_FIELD_W: return s->w;
    case HC_FIELD_P: return s->p;
    case HC_FIELD_T: return s->t;
    case HC_FIELD_FF: return s->ff;
    case HC_FIELD_GG: return s->gg;
    case HC_FIELD_HH: return s->hh;
    case HC_FIELD_SS: return s->ss;
    case HC_FIELD_PHI: return s->phi;
    default:
        if (id >= HC_FIELD_MEAN_U && id <= HC_FIELD_MEAN_TW) return s->mean[id - HC_FIELD_MEAN_U];
    }
    return NULL;
}

int or_set_field(or_state* s, int id, const double* in)
{
    double* f = field_ptr(s, id);
    if (!f || !in) return HC_ERR_ARG;
    size_t q = 0;
    for (int k = 1; k <= s->nz; ++k)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) F(f, i + 2, j + 2, k + 2) = in[q++];
    return 0;
}

int or_get_field(or_state* s, int id, double* out)
{
    double* f = field_ptr(s, id);
    if (!f || !out) return HC_ERR_ARG;
    /* spectral ff..ss live in c_ff..c_ss; report their physical image */
    if (s->prm.cds == 3 && id >= HC_FIELD_FF && id <= HC_FIELD_SS && s->initialized) {
        cplx* c = id == HC_FIELD_FF ? s->c_ff : id == HC_FIELD_GG ? s->c_gg : id == HC_FIELD_HH ? s->c_hh : s->c_ss;
        size_t n = (size_t)s->nx * s->ny * s->nz;
        cplx* tmp = calloc_c(n);
        memcpy(tmp, c, n * sizeof(cplx));
        mpi_2d_fft(s, tmp, 1);
        for (size_t q = 0; q < n; ++q) out[q] = creal(tmp[q]);
        free(tmp);
        return 0;
    }
    size_t q = 0;
    for (int k = 1; k <= s->nz; ++k)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) out[q++] = F(f, i + 2, j + 2, k + 2);
    return 0;
}

/* set-up part of drive (src/module_navier_stokes.f90:61-129) */
int or_initialize(or_state* s)
{
    if (s->prm.is_ri_var == 1) update_ri(s, 0);
    if (s->prm.dp_opt == 2) calculate_ubar(s);
    if (s->prm.cds == 3) {
        real_2_cmplx(s, s->u, s->c_u); real_2_cmplx(s, s->v, s->c_v); real_2_cmplx(s, s->w, s->c_w);
        real_2_cmplx(s, s->p, s->c_p); real_2_cmplx(s, s->t, s->c_t);
        real_2_cmplx(s, s->ff, s->c_ff); real_2_cmplx(s, s->gg, s->c_gg); real_2_cmplx(s, s->hh, s->c_hh);
        real_2_cmplx(s, s->ss, s->c_ss);
        spectral_truncation(s, s->c_u); spectral_truncation(s, s->c_v); spectral_truncation(s, s->c_w);
        spectral_truncation(s, s->c_p); spectral_truncation(s, s->c_t);
        cmplx_2_real(s, s->c_u, s->u); cmplx_2_real(s, s->c_v, s->v); cmplx_2_real(s, s->c_w, s->w);
        cmplx_2_real(s, s->c_p, s->p); cmplx_2_real(s, s->c_t, s->t);
    }
    update_boundary_uvw(s, s->u, s->v, s->w);
    update_boundary_p(s, s->p);
    update_boundary_t(s, s->t);
    s->initialized = 1;
    return 0;
}

/* body of the drive loop (src/module_navier_stokes.f90:142-165) */
int or_step(or_state* s, int nsteps, hc_diag* diag)
{
    if (!s->initialized) return HC_ERR_STATE;
    for (int n = 0; n < nsteps; ++n) {
        s->stps += 1;
        screen_cpu_time(s);
        if (s->prm.is_ri_var == 1) update_ri(s, s->stps);
        double got_used = s->got;
        for (int q = 0; q < 3; ++q) { s->div_avg_sub[q] = 0; s->div_max_sub[q] = 0; }
        int bad = s->prm.cds == 3 ? time_advancement_sp(s) : time_advancement_fd(s);
        if (!bad && s->prm.dp_opt == 2) calculate_ubar(s);
        if (diag) {
            hc_diag* d = diag + n;
            memset(d, 0, sizeof(*d));
            int last = s->prm.dts == 2 ? 2 : 0;
            d->time_sim = s->time_sim;
            d->cfl = s->cfl_max;
            d->div_avg = s->div_avg_sub[last];
            d->div_max = s->div_max_sub[last];
            d->div_hist_max = s->div_hist_max;
            d->ubar = s->prm.dp_opt == 2 ? s->ubar : 0.0;
            d->dpx_drive = s->dpx_drive;
            d->got = got_used;
            for (int q = 0; q < 3; ++q) { d->div_avg_sub[q] = s->div_avg_sub[q]; d->div_max_sub[q] = s->div_max_sub[q]; }
            d->nan_flag = s->nan_flag;
            d->step = s->stps;
        }
        if (bad) return HC_ERR_NAN;
    }
    return 0;
}

/* Helmholtz solve of the u equation alone on one real right-hand side, for
 * known-answer tests of the FFT-Thomas-iFFT chain. rk_c is taken as given. */
int or_helmholtz_u(or_state* s, const double* rhs, double* out, double rk_c)
{
    double* src = dalloc((size_t)s->nia * s->nja * s->nka);
    double* dst = dalloc((size_t)s->nia * s->nja * s->nka);
    size_t q = 0;
    for (int k = 1; k <= s->nz; ++k)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) F(src, i + 2, j + 2, k + 2) = rhs[q++];
    double save = s->rk_c;
    s->rk_c = rk_c;
    int dts = s->prm.dts;
    s->prm.dts = 2;
    assign_abc(s, s->aa_u, s->bb_u, s->cc_u, 0);
    poisson_solver_fft(s, src, dst, 0, 0, 0, 1);
    s->prm.dts = dts;
    s->rk_c = save;
    q = 0;
    for (int k = 1; k <= s->nz; ++k)
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) out[q++] = F(dst, i + 2, j + 2, k + 2);
    free(src);
    free(dst);
    return 0;
}
