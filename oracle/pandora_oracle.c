/*
 * pandora_oracle.c -- CPU restatement of PANDORA 2.0's RK3 time step (FP64).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU
 * baseline; the product (the CUDA library) never links or calls it.  Only the
 * tests, the smoke check and the bench's CPU-baseline leg load it.
 *
 * The reference (Fortran 90 + MPI + PETSc + FFTW3) cannot be built here, so this
 * is a line-by-line restatement of its arithmetic in the reference's own
 * truncated spectral layout [i][j][k][re,im] (src/pf_arrays.f90:267-280).
 * FFTW's role (src/pf_fftw.f90:199-297) is taken by a self-written mixed-radix
 * FFT with FFTW's sign and normalisation conventions: BACKWARD (e^{+ikx})
 * unnormalised for spectral->physical, FORWARD (e^{-ikx}) for physical->
 * spectral with one factor 1/(NX*NY*NZ) after the last (z) pass
 * (src/pf_fftw.f90:295-297,877).  The FFT is checked against numpy.fft and the
 * transform+nonlinear path against the reference's own known-answer test
 * (src/ptf_rk3.f90:1115-1191: L1 norms 3/4, 9/8, 11/8).
 *
 * RNG: gfortran's random_number cannot be replayed, so the seeded draws use the
 * project generator (SplitMix64 finaliser over a stream index, Steele, Lea &
 * Flood, OOPSLA 2014) that the CUDA library defines too; the ORDER and COUNT of
 * draws follow the reference loops (src/pf_initialise.f90:97-512,
 * src/pf_force.f90:106-268, src/pp_control.f90:663-707).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "../include/pandora_gpu.h"

typedef struct { double re, im; } cx;

/* ------------------------------------------------------------------------- */
/* project RNG (shared definition with the CUDA library)                      */
/* ------------------------------------------------------------------------- */
#define PD_GOLDEN 0x9E3779B97F4A7C15ULL
static inline uint64_t pd_mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static inline uint64_t pd_stream_key(uint64_t seed, uint64_t tag) {
    return pd_mix64(seed * PD_GOLDEN + tag * 0xD1B54A32D192ED03ULL + 0x632BE59BD9B4E019ULL);
}
/* n-th uniform in [0,1) of a stream (53-bit mantissa). */
static inline double pd_uniform(uint64_t key, uint64_t n) {
    return (double)(pd_mix64(key + (n + 1) * PD_GOLDEN) >> 11) * 0x1.0p-53;
}
#define PD_TAG_FLUID 1ULL
#define PD_TAG_FORCE 2ULL
#define PD_TAG_PART 3ULL
#define PD_MAX_POLAR_TRIES 64

/* g_RandomNormal (src/pg_random.f90:112-151), polar Box-Muller; normal-pair call
 * number `call` draws its uniforms from its own sub-stream.  Returns 0, or -1 if
 * the bounded rejection loop gave up. */
static int pd_normal_pair(uint64_t key, uint64_t call, double* r1, double* r2) {
    uint64_t sub = pd_mix64(key + (call + 1) * PD_GOLDEN);
    double x1 = 0.0, x2 = 0.0, w = 2.0;
    int a = 0;
    while (w >= 1.0) {
        if (a >= PD_MAX_POLAR_TRIES) { *r1 = 0.0; *r2 = 0.0; return -1; }
        x1 = pd_uniform(sub, 2 * (uint64_t)a);
        x2 = pd_uniform(sub, 2 * (uint64_t)a + 1);
        x1 = 2.0 * x1 - 1.0;
        x2 = 2.0 * x2 - 1.0;
        w = x1 * x1 + x2 * x2;
        a++;
    }
    w = sqrt((-2.0 * log(w)) / w);
    *r1 = x1 * w;
    *r2 = x2 * w;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* mixed-radix FFT (FFTW conventions, unnormalised)                           */
/* ------------------------------------------------------------------------- */
typedef struct { int n, nf; int fac[40]; cx* tw; } fplan;

static int plan_init(fplan* P, int n) {
    P->n = n; P->nf = 0;
    int m = n;
    const int pr[4] = {2, 3, 5, 7};
    for (int t = 0; t < 4; t++)
        while (m % pr[t] == 0) { P->fac[P->nf++] = pr[t]; m /= pr[t]; }
    if (m != 1) { if (P->nf >= 39) return -1; P->fac[P->nf++] = m; }
    if (P->nf == 0) P->fac[P->nf++] = 1;
    P->tw = (cx*)malloc(sizeof(cx) * (size_t)n);
    if (!P->tw) return -1;
    const long double twopi = 6.283185307179586476925286766559005768L;
    for (int e = 0; e < n; e++) {
        long double a = twopi * (long double)e / (long double)n;
        P->tw[e].re = (double)cosl(a);
        P->tw[e].im = -(double)sinl(a);   /* exp(-2 pi i e / n) */
    }
    return 0;
}
static void plan_free(fplan* P) { free(P->tw); P->tw = NULL; }

static inline cx cmulw(cx v, cx w, int sign) {
    /* sign < 0: multiply by w (FORWARD); sign > 0: by conj(w) (BACKWARD) */
    double wi = sign < 0 ? w.im : -w.im;
    cx r = {v.re * w.re - v.im * wi, v.re * wi + v.im * w.re};
    return r;
}

static void fft_rec(const cx* in, long s, cx* out, int n, const fplan* P, int fi, int sign) {
    if (n == 1) { out[0] = in[0]; return; }
    int p = P->fac[fi], m = n / p, N = P->n, ts = N / n, np = N / p;
    for (int q = 0; q < p; q++) fft_rec(in + q * s, s * p, out + q * m, m, P, fi + 1, sign);
    cx t[64], y[64];
    for (int k = 0; k < m; k++) {
        for (int q = 0; q < p; q++) {
            cx v = out[q * m + k];
            if (q && k) v = cmulw(v, P->tw[((long)q * k * ts) % N], sign);
            t[q] = v;
        }
        for (int r = 0; r < p; r++) {
            cx acc = t[0];
            for (int q = 1; q < p; q++) {
                cx z = cmulw(t[q], P->tw[(long)((q * r) % p) * np], sign);
                acc.re += z.re; acc.im += z.im;
            }
            y[r] = acc;
        }
        for (int r = 0; r < p; r++) out[k + r * m] = y[r];
    }
}
/* out = DFT(in), sign -1 = FFTW_FORWARD, +1 = FFTW_BACKWARD; in != out */
static void fft_exec(const fplan* P, const cx* in, cx* out, int sign) {
    fft_rec(in, 1, out, P->n, P, 0, sign);
}

/* ------------------------------------------------------------------------- */
/* oracle state                                                                */
/* ------------------------------------------------------------------------- */
typedef struct oracle {
    pandora_params p;
    int nx, ny, nz, ki, kj, kk, nki, nkj, nkk;
    long S;               /* modes per component */
    long R;               /* physical points */
    cx* u[3];
    cx* rk[3];
    /* forcing fluid_f(0:1,-NK:NK,-NK:NK,0:NK) stored [i][j+NK][k+NK] */
    int fnk;
    cx* ff[3];
    /* geometry (src/pg_domain.f90:147-243) */
    double dx, dy, dz, lx, ly, lz;
    double bmat[3][3], binv[3][3], amat[3][3];
    int bexist[3][3], aexist[3][3];
    int shear;            /* F_TYPE == F_SHEAR_DNS */
    int rrot;             /* ... in a Rogallo form (NS_DEFORMED = NS_R_ROT or NS_R_CONV), else BF-rot */
    int rconv;            /* ... in the convective Rogallo form (NS_R_CONV) */
    /* work */
    double* phys[12];     /* physical fields [z][y][x]: u, then omega (or the nine R-conv gradients) */
    cx *wa, *wb;          /* pencil work arrays */
    cx* nl[3];            /* spectral nonlinear term (normalised) */
    fplan px, py, pz;
    /* particles */
    long np;
    double *xp, *up, *uprk, *prk, *dp;
    /* diagnostics */
    double ucfl;
    int kkmax;
    double *dens_mod;
    int status;
} oracle;

static inline double wvn(int idx, int K) { return (double)(idx <= K ? idx : idx - (2 * K + 1)); }

static double* dalloc(long n) { return (double*)calloc((size_t)n, sizeof(double)); }
static cx* calloc_cx(long n) { return (cx*)calloc((size_t)n, sizeof(cx)); }

static void mode_density(oracle* o);

oracle* oracle_create(const pandora_params* p) {
    oracle* o = (oracle*)calloc(1, sizeof(oracle));
    if (!o) return NULL;
    o->p = *p;
    o->nx = p->nodes_x; o->ny = p->nodes_y; o->nz = p->nodes_z;
    o->ki = o->nx / 3; o->kj = o->ny / 3; o->kk = o->nz / 3;
    o->nki = o->ki + 1; o->nkj = 2 * o->kj + 1; o->nkk = 2 * o->kk + 1;
    o->S = (long)o->nki * o->nkj * o->nkk;
    o->R = (long)o->nx * o->ny * o->nz;
    for (int c = 0; c < 3; c++) {
        o->u[c] = calloc_cx(o->S); o->rk[c] = calloc_cx(o->S); o->nl[c] = calloc_cx(o->S);
    }
    o->fnk = (int)p->force_kf;   /* aint(FORCE_KF), src/pf_force.f90:289 */
    long nf = (long)(o->fnk + 1) * (2 * o->fnk + 1) * (2 * o->fnk + 1);
    for (int c = 0; c < 3; c++) o->ff[c] = calloc_cx(nf);
    /* g_DomainCalc */
    const double twopi = (double)(6.283185307179586476925286766559005768L);
    o->lx = twopi; o->ly = twopi; o->lz = twopi;
    o->dx = o->lx / (double)o->nx; o->dy = o->ly / (double)o->ny; o->dz = o->lz / (double)o->nz;
    memset(o->bmat, 0, sizeof(o->bmat)); memset(o->binv, 0, sizeof(o->binv));
    memset(o->amat, 0, sizeof(o->amat)); memset(o->bexist, 0, sizeof(o->bexist));
    memset(o->aexist, 0, sizeof(o->aexist));
    o->binv[0][0] = (double)p->b110; o->binv[1][1] = (double)p->b220; o->binv[2][2] = (double)p->b330;
    o->bexist[0][0] = o->bexist[1][1] = o->bexist[2][2] = 1;
    if (p->f_type != PANDORA_F_ISOTROPIC_DEFORMED) {
        o->bexist[0][2] = 1; o->amat[0][2] = p->f_deform_s; o->aexist[0][2] = 1;
    }
    o->shear = (p->f_type == PANDORA_F_SHEAR_DNS);
    o->rrot = o->shear && (p->ns_deformed == PANDORA_NS_R_ROT || p->ns_deformed == PANDORA_NS_R_CONV);
    o->rconv = o->shear && p->ns_deformed == PANDORA_NS_R_CONV;
    o->bmat[0][0] = 1.0 / o->binv[0][0]; o->bmat[1][1] = 1.0 / o->binv[1][1];
    o->bmat[2][2] = 1.0 / o->binv[2][2];
    for (int f = 0; f < (o->rconv ? 12 : 6); f++) o->phys[f] = dalloc(o->R);
    long wa = (long)o->nki * o->nkj * o->nz, wb = (long)o->nki * o->nz * o->ny;
    o->wa = calloc_cx(wa); o->wb = calloc_cx(wb);
    if (plan_init(&o->px, o->nx) || plan_init(&o->py, o->ny) || plan_init(&o->pz, o->nz)) {
        o->status = -1;
    }
    mode_density(o);
    return o;
}

void oracle_destroy(oracle* o) {
    if (!o) return;
    for (int c = 0; c < 3; c++) { free(o->u[c]); free(o->rk[c]); free(o->nl[c]); free(o->ff[c]); }
    for (int f = 0; f < 12; f++) free(o->phys[f]);
    free(o->wa); free(o->wb); free(o->dens_mod);
    free(o->xp); free(o->up); free(o->uprk); free(o->prk); free(o->dp);
    plan_free(&o->px); plan_free(&o->py); plan_free(&o->pz);
    free(o);
}

long oracle_modes(const oracle* o) { return o->S; }
int oracle_kkmax(const oracle* o) { return o->kkmax; }
int oracle_force_nk(const oracle* o) { return o->fnk; }

void oracle_set_state(oracle* o, const double* a, const double* b, const double* c) {
    memcpy(o->u[0], a, sizeof(cx) * o->S); memcpy(o->u[1], b, sizeof(cx) * o->S);
    memcpy(o->u[2], c, sizeof(cx) * o->S);
}
void oracle_get_state(const oracle* o, double* a, double* b, double* c) {
    memcpy(a, o->u[0], sizeof(cx) * o->S); memcpy(b, o->u[1], sizeof(cx) * o->S);
    memcpy(c, o->u[2], sizeof(cx) * o->S);
}
void oracle_set_rk(oracle* o, const double* a, const double* b, const double* c) {
    memcpy(o->rk[0], a, sizeof(cx) * o->S); memcpy(o->rk[1], b, sizeof(cx) * o->S);
    memcpy(o->rk[2], c, sizeof(cx) * o->S);
}
void oracle_get_rk(const oracle* o, double* a, double* b, double* c) {
    memcpy(a, o->rk[0], sizeof(cx) * o->S); memcpy(b, o->rk[1], sizeof(cx) * o->S);
    memcpy(c, o->rk[2], sizeof(cx) * o->S);
}
void oracle_get_nl(const oracle* o, double* a, double* b, double* c) {
    memcpy(a, o->nl[0], sizeof(cx) * o->S); memcpy(b, o->nl[1], sizeof(cx) * o->S);
    memcpy(c, o->nl[2], sizeof(cx) * o->S);
}
void oracle_get_forcing(const oracle* o, double* a, double* b, double* c) {
    long nf = (long)(o->fnk + 1) * (2 * o->fnk + 1) * (2 * o->fnk + 1);
    memcpy(a, o->ff[0], sizeof(cx) * nf); memcpy(b, o->ff[1], sizeof(cx) * nf);
    memcpy(c, o->ff[2], sizeof(cx) * nf);
}
void oracle_get_physical(const oracle* o, double* a, double* b, double* c) {
    memcpy(a, o->phys[0], sizeof(double) * o->R); memcpy(b, o->phys[1], sizeof(double) * o->R);
    memcpy(c, o->phys[2], sizeof(double) * o->R);
}
double oracle_ucfl(const oracle* o) { return o->ucfl; }
int oracle_status(const oracle* o) { return o->status; }

/* one FFT of length n on a line, exposed for the numpy check */
int oracle_fft(int n, int sign, const double* in, double* out) {
    fplan P;
    if (plan_init(&P, n)) return -1;
    fft_exec(&P, (const cx*)in, (cx*)out, sign);
    plan_free(&P);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* transforms                                                                  */
/* ------------------------------------------------------------------------- */
/* spectral (truncated) -> physical [z][y][x]:
 * z: pad k, BACKWARD (f_RK3PrepareVelocity/Vorticity + f_Fftw_k_Fs2Rs,
 *    src/pf_rk3.f90:385-492,893-948, src/pf_fftw.f90:586-624);
 * y: pad j, BACKWARD (f_RK3TransformjiFs2Rs, src/pf_rk3.f90:1437-1498);
 * x: pad i to NX/2+1, c2r (src/pf_fftw.f90:693-759,646). */
static void spec_to_phys(oracle* o, const cx* spec, double* phys) {
    const int nx = o->nx, ny = o->ny, nz = o->nz, ki = o->ki, kj = o->kj, kk = o->kk;
    const int nkj = o->nkj, nkk = o->nkk, nki = o->nki;
    cx* A = o->wa;   /* [i][j][z] */
    cx* B = o->wb;   /* [i][z][y] */
#pragma omp parallel
    {
        int nmax = nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz);
        cx* line = calloc_cx(nmax);
        cx* res = calloc_cx(nmax);
        double* rl = dalloc(nmax);
#pragma omp for schedule(static)
        for (long ij = 0; ij < (long)nki * nkj; ij++) {
            const cx* src = spec + ij * nkk;
            for (int z = 0; z < nz; z++) line[z].re = line[z].im = 0.0;
            for (int k = 0; k <= kk; k++) line[k] = src[k];
            for (int k = kk + 1; k < nkk; k++) line[nz - nkk + k] = src[k];
            fft_exec(&o->pz, line, A + ij * nz, +1);
        }
#pragma omp for schedule(static)
        for (long iz = 0; iz < (long)nki * nz; iz++) {
            long i = iz / nz, z = iz % nz;
            for (int y = 0; y < ny; y++) line[y].re = line[y].im = 0.0;
            for (int j = 0; j <= kj; j++) line[j] = A[(i * nkj + j) * nz + z];
            for (int j = kj + 1; j < nkj; j++) line[ny - nkj + j] = A[(i * nkj + j) * nz + z];
            fft_exec(&o->py, line, B + (i * nz + z) * ny, +1);
        }
#pragma omp for schedule(static)
        for (long zy = 0; zy < (long)nz * ny; zy++) {
            long z = zy / ny, y = zy % ny;
            /* Hermitian extension of the half spectrum; c2r ignores Im of DC/Nyquist */
            for (int m = 0; m < nx; m++) line[m].re = line[m].im = 0.0;
            for (int m = 0; m <= nx / 2; m++) {
                cx v = {0.0, 0.0};
                if (m <= ki) v = B[((long)m * nz + z) * ny + y];
                if (m == 0 || (nx % 2 == 0 && m == nx / 2)) v.im = 0.0;
                line[m] = v;
                if (m > 0 && m < nx - m) { line[nx - m].re = v.re; line[nx - m].im = -v.im; }
            }
            fft_exec(&o->px, line, res, +1);
            for (int x = 0; x < nx; x++) rl[x] = res[x].re;
            memcpy(phys + zy * nx, rl, sizeof(double) * nx);
        }
        free(line); free(res); free(rl);
    }
}

/* physical [z][y][x] -> spectral (truncated, normalised):
 * x: r2c, truncate i (src/pf_fftw.f90:766-834, src/pf_rk3.f90:1878-1940);
 * y: FORWARD, truncate j; z: FORWARD, x 1/(NX NY NZ), truncate k
 * (src/pf_rk3.f90:2242-2316, src/pf_fftw.f90:841-879). */
static void phys_to_spec(oracle* o, const double* phys, cx* spec) {
    const int nx = o->nx, ny = o->ny, nz = o->nz, ki = o->ki, kj = o->kj, kk = o->kk;
    const int nkj = o->nkj, nkk = o->nkk, nki = o->nki;
    (void)ki; (void)kj; (void)kk;
    cx* A = o->wa;   /* [i][j][z] */
    cx* B = o->wb;   /* [i][z][y] */
    const double norm = 1.0 / ((double)nx * (double)ny * (double)nz);
#pragma omp parallel
    {
        int nmax = nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz);
        cx* line = calloc_cx(nmax);
        cx* res = calloc_cx(nmax);
#pragma omp for schedule(static)
        for (long zy = 0; zy < (long)nz * ny; zy++) {
            long z = zy / ny, y = zy % ny;
            for (int x = 0; x < nx; x++) { line[x].re = phys[zy * nx + x]; line[x].im = 0.0; }
            fft_exec(&o->px, line, res, -1);
            for (int i = 0; i < nki; i++) B[((long)i * nz + z) * ny + y] = res[i];
        }
#pragma omp for schedule(static)
        for (long iz = 0; iz < (long)nki * nz; iz++) {
            long i = iz / nz, z = iz % nz;
            fft_exec(&o->py, B + (i * nz + z) * ny, res, -1);
            for (int j = 0; j <= o->kj; j++) A[(i * nkj + j) * nz + z] = res[j];
            for (int j = o->kj + 1; j < nkj; j++) A[(i * nkj + j) * nz + z] = res[ny - nkj + j];
        }
#pragma omp for schedule(static)
        for (long ij = 0; ij < (long)nki * nkj; ij++) {
            fft_exec(&o->pz, A + ij * nz, res, -1);
            for (int z = 0; z < nz; z++) { res[z].re = res[z].re * norm; res[z].im = res[z].im * norm; }
            cx* dst = spec + ij * nkk;
            for (int k = 0; k <= o->kk; k++) dst[k] = res[k];
            for (int k = o->kk + 1; k < nkk; k++) dst[k] = res[nz - nkk + k];
        }
        free(line); free(res);
    }
}

/* spectral vorticity omega = i k x u, isotropic branch of f_RK3PrepareVelocity
 * (src/pf_rk3.f90:402-407,520-525,630-634) with f_RK3Derivative (3735-3743). */
static void vorticity_iso(oracle* o, cx* om[3]) {
#pragma omp parallel for schedule(static)
    for (long ij = 0; ij < (long)o->nki * o->nkj; ij++) {
        int i = (int)(ij / o->nkj), j = (int)(ij % o->nkj);
        double k1 = wvn(i, o->ki), k2 = wvn(j, o->kj);
        for (int k = 0; k < o->nkk; k++) {
            long m = ij * o->nkk + k;
            double k3 = wvn(k, o->kk);
            cx u = o->u[0][m], v = o->u[1][m], w = o->u[2][m];
            cx dudy = {-k2 * u.im, k2 * u.re}, dudz = {-k3 * u.im, k3 * u.re};
            cx dvdx = {-k1 * v.im, k1 * v.re}, dvdz = {-k3 * v.im, k3 * v.re};
            cx dwdx = {-k1 * w.im, k1 * w.re}, dwdy = {-k2 * w.im, k2 * w.re};
            cx o4 = {0.0, 0.0}, o5 = dudz, o6 = {-dudy.re, -dudy.im};
            o4.re = o4.re - dvdz.re; o4.im = o4.im - dvdz.im;
            o6.re = o6.re + dvdx.re; o6.im = o6.im + dvdx.im;
            o4.re = o4.re + dwdy.re; o4.im = o4.im + dwdy.im;
            o5.re = o5.re - dwdx.re; o5.im = o5.im - dwdx.im;
            om[0][m] = o4; om[1][m] = o5; om[2][m] = o6;
        }
    }
}

/* f_RK3ComputeNonlinearIsotropic (src/pf_rk3.f90:1597-1628): NL = omega x u */
static void nonlinear_iso(oracle* o) {
    double *u1 = o->phys[0], *u2 = o->phys[1], *u3 = o->phys[2];
    double *w1 = o->phys[3], *w2 = o->phys[4], *w3 = o->phys[5];
#pragma omp parallel for schedule(static)
    for (long p = 0; p < o->R; p++) {
        double n1 = u3[p] * w2[p] - u2[p] * w3[p];
        double n2 = u1[p] * w3[p] - u3[p] * w1[p];
        double n3 = u2[p] * w1[p] - u1[p] * w2[p];
        w1[p] = n1; w2[p] = n2; w3[p] = n3;
    }
}


/* BF-rot vorticity of one velocity component n, f_RK3VorticityBFRot
 * (src/pf_rk3.f90:3786-3843): accumulates into w[0..2]. */
static void vort_bf_add(const oracle* o, cx un, const double* k, int n, cx* w) {
    const double(*bm)[3] = o->bmat;
    const double(*bi)[3] = o->binv;
    const int(*ex)[3] = o->bexist;
    for (int m = 0; m < 3; m++) {
        if (ex[m][0]) {
            if (ex[2][n]) {
                w[1].im = w[1].im - (bm[m][0] * bi[2][n] * k[m] * un.re);
                w[1].re = w[1].re + (bm[m][0] * bi[2][n] * k[m] * un.im);
            }
            if (ex[1][n]) {
                w[2].im = w[2].im + (bm[m][0] * bi[1][n] * k[m] * un.re);
                w[2].re = w[2].re - (bm[m][0] * bi[1][n] * k[m] * un.im);
            }
        }
        if (ex[m][1]) {
            if (ex[2][n]) {
                w[0].im = w[0].im + (bm[m][1] * bi[2][n] * k[m] * un.re);
                w[0].re = w[0].re - (bm[m][1] * bi[2][n] * k[m] * un.im);
            }
            if (ex[0][n]) {
                w[2].im = w[2].im - (bm[m][1] * bi[0][n] * k[m] * un.re);
                w[2].re = w[2].re + (bm[m][1] * bi[0][n] * k[m] * un.im);
            }
        }
        if (ex[m][2]) {
            if (ex[1][n]) {
                w[0].im = w[0].im - (bm[m][2] * bi[1][n] * k[m] * un.re);
                w[0].re = w[0].re + (bm[m][2] * bi[1][n] * k[m] * un.im);
            }
            if (ex[0][n]) {
                w[1].im = w[1].im + (bm[m][2] * bi[0][n] * k[m] * un.re);
                w[1].re = w[1].re - (bm[m][2] * bi[0][n] * k[m] * un.im);
            }
        }
    }
}

static void vorticity_bf(oracle* o, cx* om[3]) {
#pragma omp parallel for schedule(static)
    for (long ij = 0; ij < (long)o->nki * o->nkj; ij++) {
        int i = (int)(ij / o->nkj), j = (int)(ij % o->nkj);
        for (int k = 0; k < o->nkk; k++) {
            long m = ij * o->nkk + k;
            double kv[3] = {wvn(i, o->ki), wvn(j, o->kj), wvn(k, o->kk)};
            cx w[3] = {{0, 0}, {0, 0}, {0, 0}};
            for (int n = 0; n < 3; n++) vort_bf_add(o, o->u[n][m], kv, n, w);
            om[0][m] = w[0]; om[1][m] = w[1]; om[2][m] = w[2];
        }
    }
}

/* f_RK3DerivativeRRot (src/pf_rk3.f90:3749-3780): d/dx_j = i sum_m bmat(m,j) k_m, over
 * every m (the reference's bvalexist test there guards nothing). */
static cx deriv_rrot(const oracle* o, cx u, const double* k, int j) {
    cx d = {0.0, 0.0};
    for (int m = 0; m < 3; m++) {
        d.im = d.im + (o->bmat[m][j] * k[m] * u.re);
        d.re = d.re - (o->bmat[m][j] * k[m] * u.im);
    }
    return d;
}

/* R-rot vorticity (src/pf_rk3.f90:416-421, 470-475, 585-590): w = D x u with the
 * sheared derivatives, assembled per velocity component in the reference's order. */
static void vorticity_rrot(oracle* o, cx* om[3]) {
#pragma omp parallel for schedule(static)
    for (long ij = 0; ij < (long)o->nki * o->nkj; ij++) {
        int i = (int)(ij / o->nkj), j = (int)(ij % o->nkj);
        for (int k = 0; k < o->nkk; k++) {
            long m = ij * o->nkk + k;
            double kv[3] = {wvn(i, o->ki), wvn(j, o->kj), wvn(k, o->kk)};
            cx w[3];
            cx dudy = deriv_rrot(o, o->u[0][m], kv, 1), dudz = deriv_rrot(o, o->u[0][m], kv, 2);
            w[0].re = 0.0; w[0].im = 0.0;
            w[1] = dudz;
            w[2].re = -dudy.re; w[2].im = -dudy.im;
            cx dvdx = deriv_rrot(o, o->u[1][m], kv, 0), dvdz = deriv_rrot(o, o->u[1][m], kv, 2);
            w[0].re = w[0].re - dvdz.re; w[0].im = w[0].im - dvdz.im;
            w[2].re = w[2].re + dvdx.re; w[2].im = w[2].im + dvdx.im;
            cx dwdx = deriv_rrot(o, o->u[2][m], kv, 0), dwdy = deriv_rrot(o, o->u[2][m], kv, 1);
            w[0].re = w[0].re + dwdy.re; w[0].im = w[0].im + dwdy.im;
            w[1].re = w[1].re - dwdx.re; w[1].im = w[1].im - dwdx.im;
            om[0][m] = w[0]; om[1][m] = w[1]; om[2][m] = w[2];
        }
    }
}

/* R-conv form (NS_DEFORMED = NS_R_CONV): the nine plain derivatives d u_c / d x_d =
 * i k_d u_c (f_RK3Derivative, src/pf_rk3.f90:3735-3743) held as the reference's u4..u12
 * (u4, u5, u6 = d(u, v, w)/dx, u7..u9 the y and u10..u12 the z derivatives;
 * src/pf_rk3.f90:422-428, 476-482, 538-544), into phys[3 + 3 d + c]. */
static void gradients_rconv(oracle* o) {
    cx* g = o->nl[0];
    for (int d = 0; d < 3; d++)
        for (int c = 0; c < 3; c++) {
#pragma omp parallel for schedule(static)
            for (long ij = 0; ij < (long)o->nki * o->nkj; ij++) {
                int i = (int)(ij / o->nkj), j = (int)(ij % o->nkj);
                for (int k = 0; k < o->nkk; k++) {
                    long m = ij * o->nkk + k;
                    const double kd = d == 0 ? wvn(i, o->ki) : (d == 1 ? wvn(j, o->kj) : wvn(k, o->kk));
                    const cx u = o->u[c][m];
                    g[m].im = kd * u.re;
                    g[m].re = -kd * u.im;
                }
            }
            spec_to_phys(o, g, o->phys[3 + 3 * d + c]);
        }
}

/* f_RK3ComputeNonlinearRConv (src/pf_rk3.f90:1717-1774): with duidk(k, i) = d u_i / d x_k
 * (phys[3 + 3 (k-1) + (i-1)]), NL_i = sum_j sum_k bmat(k,j) duidk(k,i) u_j over the
 * existing bmat entries, into phys[3..5]. */
static void nonlinear_rconv(oracle* o) {
    const double(*bm)[3] = o->bmat;
    const int(*ex)[3] = o->bexist;
#pragma omp parallel for schedule(static)
    for (long p = 0; p < o->R; p++) {
        const double uj[3] = {o->phys[0][p], o->phys[1][p], o->phys[2][p]};
        double du[3][3];
        for (int k = 0; k < 3; k++)
            for (int i = 0; i < 3; i++) du[k][i] = o->phys[3 + 3 * k + i][p];
        double nl[3] = {0.0, 0.0, 0.0};
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                for (int k = 0; k < 3; k++)
                    if (ex[k][j]) nl[i] = nl[i] + ((bm[k][j] * du[k][i]) * uj[j]);
        o->phys[3][p] = nl[0]; o->phys[4][p] = nl[1]; o->phys[5][p] = nl[2];
    }
}

/* f_RK3ComputeNonlinearBFRot (src/pf_rk3.f90:1634-1711) */
static void nonlinear_bf(oracle* o) {
    const double(*bi)[3] = o->binv;
    const int(*ex)[3] = o->bexist;
    double *w1 = o->phys[3], *w2 = o->phys[4], *w3 = o->phys[5];
#pragma omp parallel for schedule(static)
    for (long p = 0; p < o->R; p++) {
        double u[3] = {o->phys[0][p], o->phys[1][p], o->phys[2][p]};
        double om[3] = {w1[p], w2[p], w3[p]};
        double n1 = 0.0, n2 = 0.0, n3 = 0.0;
        for (int m = 0; m < 3; m++) {
            if (ex[0][m]) { n3 = n3 - (om[1] * bi[0][m] * u[m]); n2 = n2 + (om[2] * bi[0][m] * u[m]); }
            if (ex[1][m]) { n1 = n1 - (om[2] * bi[1][m] * u[m]); n3 = n3 + (om[0] * bi[1][m] * u[m]); }
            if (ex[2][m]) { n1 = n1 + (om[1] * bi[2][m] * u[m]); n2 = n2 - (om[0] * bi[2][m] * u[m]); }
        }
        w1[p] = n1; w2[p] = n2; w3[p] = n3;
    }
}

/* f_RK3FormFBFRot for F_SHEAR_DNS (src/pf_rk3.f90:2494-2673) with
 * f_RK3BFRotNonlinear 2864-2895, ...Viscous 2903-2937, ...Pressure 2986-3070,
 * ...Source 3167-3209, then f_RK3RungeKutta and f_RK3ContinuityFixIsotropic. */
static void form_f_bf(oracle* o, int stage, double dt) {
    double beta, gamma;
    void rk_coeffs(int, double*, double*);
    rk_coeffs(stage, &beta, &gamma);
    const double nu = o->p.f_nu;
    const double(*bm)[3] = o->bmat;
    const double(*bi)[3] = o->binv;
    const double(*am)[3] = o->amat;
    const int(*ex)[3] = o->bexist;
    const int(*ax)[3] = o->aexist;
#pragma omp parallel for schedule(static)
    for (long ij = 0; ij < (long)o->nki * o->nkj; ij++) {
        int i = (int)(ij / o->nkj), j = (int)(ij % o->nkj);
        for (int kq = 0; kq < o->nkk; kq++) {
            long m0 = ij * o->nkk + kq;
            double k[3] = {wvn(i, o->ki), wvn(j, o->kj), wvn(kq, o->kk)};
            double kmag2 = (k[0] * k[0]) + (k[1] * k[1]) + (k[2] * k[2]);
            if (!(kmag2 > 0.0)) continue;
            cx u[3] = {o->u[0][m0], o->u[1][m0], o->u[2][m0]};
            cx nlr[3] = {o->nl[0][m0], o->nl[1][m0], o->nl[2][m0]};
            cx nl[3] = {{0, 0}, {0, 0}, {0, 0}};
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++)
                    if (ex[a][b]) { nl[a].re = nl[a].re + bm[a][b] * nlr[b].re; nl[a].im = nl[a].im + bm[a][b] * nlr[b].im; }
            /* pressure */
            double p1[3] = {0, 0, 0}, p4 = 0.0;
            cx p2 = {0, 0}, p3 = {0, 0};
            for (int m = 0; m < 3; m++) {
                p2.re = p2.re + (k[m] * nl[m].re); p2.im = p2.im + (k[m] * nl[m].im);
                for (int r = 0; r < 3; r++) {
                    if (!ex[m][r]) continue;
                    for (int sx = 0; sx < 3; sx++) {
                        if (!ax[r][sx]) continue;
                        for (int q = 0; q < 3; q++) {
                            if (!ex[sx][q]) continue;
                            double c = k[m] * bm[m][r] * am[r][sx] * bi[sx][q];
                            p3.re = p3.re + (2.0 * (c * u[q].re));
                            p3.im = p3.im + (2.0 * (c * u[q].im));
                        }
                    }
                    for (int q = 0; q < 3; q++)
                        if (ex[q][r]) p4 = p4 + (k[m] * bm[m][r] * bm[q][r] * k[q]);
                }
            }
            for (int a = 0; a < 3; a++)
                for (int pp = 0; pp < 3; pp++)
                    if (ex[a][pp])
                        for (int b = 0; b < 3; b++)
                            if (ex[b][pp]) p1[a] = p1[a] + bm[a][pp] * bm[b][pp] * k[b];
            cx press[3];
            for (int a = 0; a < 3; a++) {
                if (p4 > 0.0) { press[a].re = (p1[a] / p4) * (p2.re + p3.re); press[a].im = (p1[a] / p4) * (p2.im + p3.im); }
                else { press[a].re = 0.0; press[a].im = 0.0; }
            }
            /* homogeneous source */
            cx hom[3] = {{0, 0}, {0, 0}, {0, 0}};
            for (int a = 0; a < 3; a++)
                for (int r = 0; r < 3; r++) {
                    if (!ex[a][r]) continue;
                    for (int b = 0; b < 3; b++) {
                        if (!ax[r][b]) continue;
                        for (int q = 0; q < 3; q++) {
                            if (!ex[b][q]) continue;
                            double c = bm[a][r] * am[r][b] * bi[b][q];
                            hom[a].re = hom[a].re + (2.0 * (c * u[q].re));
                            hom[a].im = hom[a].im + (2.0 * (c * u[q].im));
                        }
                    }
                }
            /* viscous */
            cx visc[3] = {{0, 0}, {0, 0}, {0, 0}};
            for (int l = 0; l < 3; l++)
                for (int jj = 0; jj < 3; jj++) {
                    if (!ex[l][jj]) continue;
                    for (int n = 0; n < 3; n++) {
                        if (!ex[n][jj]) continue;
                        double c = nu * bm[l][jj] * bm[n][jj] * k[l] * k[n];
                        for (int a = 0; a < 3; a++) { visc[a].re = visc[a].re - c * u[a].re; visc[a].im = visc[a].im - c * u[a].im; }
                    }
                }
            cx tot[3];
            for (int a = 0; a < 3; a++) {
                tot[a].re = visc[a].re - nl[a].re + press[a].re + 0.0 - hom[a].re;
                tot[a].im = visc[a].im - nl[a].im + press[a].im + 0.0 - hom[a].im;
            }
            for (int a = 0; a < 3; a++) {
                cx* r = &o->rk[a][m0];
                r->re = (beta * r->re) + tot[a].re;
                r->im = (beta * r->im) + tot[a].im;
                u[a].re = u[a].re + (gamma * dt * r->re);
                u[a].im = u[a].im + (gamma * dt * r->im);
            }
            cx kdu = {k[0] * u[0].re + k[1] * u[1].re + k[2] * u[2].re, k[0] * u[0].im + k[1] * u[1].im + k[2] * u[2].im};
            for (int a = 0; a < 3; a++) {
                u[a].re = u[a].re - (k[a] * kdu.re / kmag2);
                u[a].im = u[a].im - (k[a] * kdu.im / kmag2);
                o->u[a][m0] = u[a];
            }
        }
    }
}

/* f_RK3FormFRRot for F_SHEAR_DNS (src/pf_rk3.f90:2680-2856): f_RK3RRotPressure
 * (2986-3070 pattern, the R-rot routine of 3078-3156), f_RK3RRotSource (3218-3249),
 * f_RK3RRotViscous, then f_RK3RungeKutta and f_RK3ContinuityFixRRot (3620-3693).
 * The nonlinear term enters untransformed (the isotropic product of the R-rot
 * vorticity). */
static void form_f_rrot(oracle* o, int stage, double dt) {
    double beta, gamma;
    void rk_coeffs(int, double*, double*);
    rk_coeffs(stage, &beta, &gamma);
    const double nu = o->p.f_nu;
    const double(*bm)[3] = o->bmat;
    const double(*bi)[3] = o->binv;
    const double(*am)[3] = o->amat;
    const int(*ex)[3] = o->bexist;
    const int(*ax)[3] = o->aexist;
#pragma omp parallel for schedule(static)
    for (long ij = 0; ij < (long)o->nki * o->nkj; ij++) {
        int i = (int)(ij / o->nkj), j = (int)(ij % o->nkj);
        for (int kq = 0; kq < o->nkk; kq++) {
            long m0 = ij * o->nkk + kq;
            double k[3] = {wvn(i, o->ki), wvn(j, o->kj), wvn(kq, o->kk)};
            double kmag2 = (k[0] * k[0]) + (k[1] * k[1]) + (k[2] * k[2]);
            if (!(kmag2 > 0.0)) continue;
            cx u[3] = {o->u[0][m0], o->u[1][m0], o->u[2][m0]};
            cx nl[3] = {o->nl[0][m0], o->nl[1][m0], o->nl[2][m0]};
            /* pressure */
            double p1[3] = {0, 0, 0}, p4 = 0.0;
            cx p2 = {0, 0}, p3 = {0, 0};
            for (int m = 0; m < 3; m++)
                for (int r = 0; r < 3; r++) {
                    if (!ex[m][r]) continue;
                    p2.re = p2.re + (k[m] * bm[m][r] * nl[r].re);
                    p2.im = p2.im + (k[m] * bm[m][r] * nl[r].im);
                    for (int q = 0; q < 3; q++)
                        if (ax[r][q]) {
                            p3.re = p3.re + (k[m] * bm[m][r] * am[r][q] * u[q].re);
                            p3.im = p3.im + (k[m] * bm[m][r] * am[r][q] * u[q].im);
                        }
                    for (int q = 0; q < 3; q++)
                        if (ex[q][r]) p4 = p4 + (k[m] * bm[m][r] * k[q] * bm[q][r]);
                }
            for (int a = 0; a < 3; a++)
                for (int pp = 0; pp < 3; pp++)
                    if (ex[pp][a]) p1[a] = p1[a] + k[pp] * bm[pp][a];
            cx press[3];
            for (int a = 0; a < 3; a++) {
                if (p4 > 0.0) { press[a].re = (p1[a] / p4) * (p2.re + p3.re); press[a].im = (p1[a] / p4) * (p2.im + p3.im); }
                else { press[a].re = 0.0; press[a].im = 0.0; }
            }
            /* homogeneous source A u */
            cx hom[3] = {{0, 0}, {0, 0}, {0, 0}};
            for (int a = 0; a < 3; a++)
                for (int q = 0; q < 3; q++)
                    if (ax[a][q]) { hom[a].re = hom[a].re + (am[a][q] * u[q].re); hom[a].im = hom[a].im + (am[a][q] * u[q].im); }
            /* viscous */
            cx visc[3] = {{0, 0}, {0, 0}, {0, 0}};
            for (int l = 0; l < 3; l++)
                for (int jj = 0; jj < 3; jj++) {
                    if (!ex[l][jj]) continue;
                    for (int n = 0; n < 3; n++) {
                        if (!ex[n][jj]) continue;
                        for (int a = 0; a < 3; a++) {
                            visc[a].re = visc[a].re - nu * bm[l][jj] * bm[n][jj] * k[l] * k[n] * u[a].re;
                            visc[a].im = visc[a].im - nu * bm[l][jj] * bm[n][jj] * k[l] * k[n] * u[a].im;
                        }
                    }
                }
            cx tot[3];
            for (int a = 0; a < 3; a++) {
                tot[a].re = visc[a].re - nl[a].re + press[a].re + 0.0 - hom[a].re;
                tot[a].im = visc[a].im - nl[a].im + press[a].im + 0.0 - hom[a].im;
            }
            for (int a = 0; a < 3; a++) {
                cx* r = &o->rk[a][m0];
                r->re = (beta * r->re) + tot[a].re;
                r->im = (beta * r->im) + tot[a].im;
                u[a].re = u[a].re + (gamma * dt * r->re);
                u[a].im = u[a].im + (gamma * dt * r->im);
            }
            /* f_RK3ContinuityFixRRot: project in the moving components umov = bmat u */
            cx um[3] = {{0, 0}, {0, 0}, {0, 0}};
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++)
                    if (ex[a][b]) { um[a].re = um[a].re + (bm[a][b] * u[b].re); um[a].im = um[a].im + (bm[a][b] * u[b].im); }
            cx kdu = {k[0] * um[0].re + k[1] * um[1].re + k[2] * um[2].re, k[0] * um[0].im + k[1] * um[1].im + k[2] * um[2].im};
            for (int a = 0; a < 3; a++) {
                um[a].re = um[a].re - (k[a] * kdu.re / kmag2);
                um[a].im = um[a].im - (k[a] * kdu.im / kmag2);
            }
            cx ul[3] = {{0, 0}, {0, 0}, {0, 0}};
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++)
                    if (ex[a][b]) { ul[a].re = ul[a].re + (bi[a][b] * um[b].re); ul[a].im = ul[a].im + (bi[a][b] * um[b].im); }
            for (int a = 0; a < 3; a++) o->u[a][m0] = ul[a];
        }
    }
}

/* max |u1|+|u2|+|u3| (src/pf_fluidstats.f90:913-917,979) */
static double cfl_velocity(const oracle* o) {
    double m = 0.0;
#pragma omp parallel for reduction(max : m) schedule(static)
    for (long p = 0; p < o->R; p++) {
        double v = fabs(o->phys[0][p]) + fabs(o->phys[1][p]) + fabs(o->phys[2][p]);
        if (v > m) m = v;
    }
    return m;
}


/* ------------------------------------------------------------------------- */
/* Rogallo moving frame (shear): g_RK3UpdateB (src/pg_rk3.f90:280-385) and the */
/* wave-space remesh f_RK3Remesh / f_RK3RemeshWaveSpace (src/pf_rk3.f90:3958-4178) */
/* ------------------------------------------------------------------------- */
void oracle_update_b(oracle* o, int tstep, double simtime) {
    const pandora_params* p = &o->p;
    if (p->f_type == PANDORA_F_ISOTROPIC) return;
    double localtime = simtime;
    if (p->rk3_timestep == PANDORA_RK3_TIMESTEP_DECIDE) {
        if (tstep > p->b110 * p->f_remesh_t) {
            int a = tstep - (p->b110 * p->f_remesh_t) - 1;
            int b = 2 * (p->b110 * p->f_remesh_t);
            int localtstep = a / b;
            localtime = simtime - ((double)(localtstep + 1) / p->f_deform_s * (double)p->b110);
        }
    }
    o->bmat[0][2] = -o->bmat[0][0] * p->f_deform_s * localtime;
    o->binv[0][2] = p->f_deform_s * localtime / o->bmat[2][2];
}

int oracle_remesh_due(const oracle* o, int tstep) {
    const pandora_params* p = &o->p;
    if (p->f_type == PANDORA_F_ISOTROPIC || p->rk3_timestep != PANDORA_RK3_TIMESTEP_DECIDE) return 0;
    int a = tstep - (p->b110 * p->f_remesh_t) - 1;
    int b = 2 * p->b110 * p->f_remesh_t;
    return (a % b) == 0;
}

/* k3 <- k3 - k1 shift, modes below -KK dropped, BF-rot: u1 += u3; then the
 * frame jumps from S t = +B110/2 to -B110/2 (bmat/binv (1,3) reset). */
static void remesh_wave_space(oracle* o) {
    const int KK = o->kk, nodes = 2 * KK + 1, NKK = o->nkk;
    const double half_b = (double)o->p.b110 * 0.5;
    o->binv[0][2] = half_b / o->bmat[2][2];
    o->bmat[0][2] = -o->bmat[0][0] * (-half_b);
#pragma omp parallel
    {
        cx* r[3];
        for (int c = 0; c < 3; c++) r[c] = calloc_cx(NKK);
#pragma omp for schedule(static)
        for (long ij = 0; ij < (long)o->nki * o->nkj; ij++) {
            int i = (int)(ij / o->nkj);
            for (int c = 0; c < 3; c++) memset(r[c], 0, sizeof(cx) * NKK);
            for (int k = 0; k < NKK; k++) {
                int actualk = k > KK ? k - nodes : k;
                int knew = actualk - i;
                if (knew >= -KK) {
                    if (knew < 0) knew += nodes;
                    for (int c = 0; c < 3; c++) r[c][knew] = o->u[c][ij * NKK + k];
                }
            }
            for (int k = 0; k < NKK; k++) {
                cx a = r[0][k], b3 = r[2][k];
                if (o->rrot) { b3.re = 0.0; b3.im = 0.0; }   /* R-rot: no u1 += u3 (src/pf_rk3.f90:4155-4158) */
                o->u[0][ij * NKK + k].re = a.re + b3.re;
                o->u[0][ij * NKK + k].im = a.im + b3.im;
                o->u[1][ij * NKK + k] = r[1][k];
                o->u[2][ij * NKK + k] = r[2][k];
            }
        }
        for (int c = 0; c < 3; c++) free(r[c]);
    }
    o->binv[0][2] = (-half_b) / o->bmat[2][2];
}

void oracle_get_b(const oracle* o, double* b13, double* bi13) {
    *b13 = o->bmat[0][2];
    *bi13 = o->binv[0][2];
}

/* f_ArraysDealiasSpherical / f_ArraysLESCutoff (src/pf_arrays.f90:1865-1987):
 * DEALIASING 2 zeroes every mode whose laboratory-frame wave vector
 * k_lab(n) = sum_m bmat(m,n) k(m) is longer than KMAX = min(KI, KJ, KK)
 * (src/pg_domain.f90:231), DEALIASING 3 those longer than LES_CUTOFF * KMAX. */
static void dealias(oracle* o) {
    const int mode = o->p.dealiasing;
    if (mode != PANDORA_DEALIASING_SPHERICAL && mode != PANDORA_DEALIASING_LES) return;
    int kmin = o->ki < o->kj ? o->ki : o->kj;
    kmin = kmin < o->kk ? kmin : o->kk;
    const double kmax = (double)kmin;
    const double cutoff = mode == PANDORA_DEALIASING_SPHERICAL ? kmax : o->p.les_cutoff * kmax;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < o->nki; i++)
        for (int j = 0; j < o->nkj; j++)
            for (int k = 0; k < o->nkk; k++) {
                const double mov[3] = {(double)i, wvn(j, o->kj), wvn(k, o->kk)};
                double lab[3] = {0.0, 0.0, 0.0};
                for (int m = 0; m < 3; m++)
                    for (int n = 0; n < 3; n++)
                        if (o->bexist[m][n]) lab[n] = lab[n] + o->bmat[m][n] * mov[m];
                const double kmag = sqrt((lab[0] * lab[0]) + (lab[1] * lab[1]) + (lab[2] * lab[2]));
                if (kmag > cutoff) {
                    const long m = ((long)i * o->nkj + j) * o->nkk + k;
                    for (int c = 0; c < 3; c++) { o->u[c][m].re = 0.0; o->u[c][m].im = 0.0; }
                }
            }
}

/* transforms + nonlinear term of the current state -> o->nl (normalised); with
 * DEALIASING 2/3 the state is first truncated (f_RK3PrepareRealSpace,
 * src/pf_rk3.f90:269-277; the second truncation after the nonlinear term,
 * src/pf_rk3.f90:2101-2109, finds the state unchanged) */
static void compute_nonlinear(oracle* o, int want_cfl) {
    dealias(o);
    if (o->rconv) {   /* 12 transformed fields (src/pf_rk3.f90:254-267, 825-869) */
        for (int c = 0; c < 3; c++) spec_to_phys(o, o->u[c], o->phys[c]);
        gradients_rconv(o);
        if (want_cfl) o->ucfl = cfl_velocity(o);
        nonlinear_rconv(o);
        for (int c = 0; c < 3; c++) phys_to_spec(o, o->phys[3 + c], o->nl[c]);
        return;
    }
    cx* om[3] = {o->nl[0], o->nl[1], o->nl[2]};   /* spectral omega held in nl */
    if (o->rrot) vorticity_rrot(o, om);
    else if (o->shear) vorticity_bf(o, om);
    else vorticity_iso(o, om);
    for (int c = 0; c < 3; c++) spec_to_phys(o, o->u[c], o->phys[c]);
    for (int c = 0; c < 3; c++) spec_to_phys(o, om[c], o->phys[3 + c]);
    if (want_cfl) o->ucfl = cfl_velocity(o);
    if (o->shear && !o->rrot) nonlinear_bf(o);   /* R-rot: the isotropic product (src/pf_rk3.f90:1088-1089) */
    else nonlinear_iso(o);
    for (int c = 0; c < 3; c++) phys_to_spec(o, o->phys[3 + c], o->nl[c]);
}

/* f_FluidstatsRs2D (src/pf_fluidstats.f90:827-958) over the physical fields of the
 * current state: out[0..20] raw sums of u1u1 u2u2 u3u3 u1u2 u1u3 u2u3, u^3, u^4
 * (laboratory frame: u_lab = binv u), w^2, w^3, w^4; out[21] max |u1|+|u2|+|u3|,
 * out[22..24] max |w_i|.  The state is truncated first as at a stage's start. */
void oracle_realspace_sums(oracle* o, double* out) {
    dealias(o);
    cx* om[3] = {o->nl[0], o->nl[1], o->nl[2]};
    if (o->rconv) {   /* R-conv: u4..u6 hold d(u1,u2,u3)/dx1 (src/pf_rk3.f90:422-428, 476-482, 538-544) */
        for (long ij = 0; ij < (long)o->nki * o->nkj; ij++) {
            const double k1 = wvn((int)(ij / o->nkj), o->ki);
            for (int k = 0; k < o->nkk; k++) {
                const long m = ij * o->nkk + k;
                for (int c = 0; c < 3; c++) {
                    const cx u = o->u[c][m];
                    om[c][m].im = k1 * u.re;
                    om[c][m].re = -k1 * u.im;
                }
            }
        }
    } else if (o->rrot) vorticity_rrot(o, om);
    else if (o->shear) vorticity_bf(o, om);
    else vorticity_iso(o, om);
    for (int c = 0; c < 3; c++) spec_to_phys(o, o->u[c], o->phys[c]);
    for (int c = 0; c < 3; c++) spec_to_phys(o, om[c], o->phys[3 + c]);
    for (int a = 0; a < 25; a++) out[a] = 0.0;
    for (long x = 0; x < o->R; x++) {
        double u[3] = {o->phys[0][x], o->phys[1][x], o->phys[2][x]};
        if (o->p.f_type != PANDORA_F_ISOTROPIC) {
            double ul[3] = {0.0, 0.0, 0.0};
            for (int m = 0; m < 3; m++)
                for (int n = 0; n < 3; n++)
                    if (o->bexist[m][n]) ul[m] += o->binv[m][n] * u[n];
            u[0] = ul[0]; u[1] = ul[1]; u[2] = ul[2];
        }
        const double w[3] = {o->phys[3][x], o->phys[4][x], o->phys[5][x]};
        out[0] += u[0] * u[0]; out[1] += u[1] * u[1]; out[2] += u[2] * u[2];
        out[3] += u[0] * u[1]; out[4] += u[0] * u[2]; out[5] += u[1] * u[2];
        for (int c = 0; c < 3; c++) {
            out[6 + c] += u[c] * u[c] * u[c];
            out[9 + c] += (u[c] * u[c]) * (u[c] * u[c]);
            out[12 + c] += w[c] * w[c];
            out[15 + c] += w[c] * w[c] * w[c];
            out[18 + c] += (w[c] * w[c]) * (w[c] * w[c]);
            if (fabs(w[c]) > out[22 + c]) out[22 + c] = fabs(w[c]);
        }
        const double us = fabs(u[0]) + fabs(u[1]) + fabs(u[2]);
        if (us > out[21]) out[21] = us;
    }
}

/* TS_CORR's longitudinal autocorrelation (f_FluidstatsRs2D, src/pf_fluidstats.f90:933-945)
 * as the reference loops: per point (z slice, y, x) and ii = i .. i + (NX-1)/2 + 1,
 * temp_r1i(ii - i) += u1 * arr_u1(ii, wrapped by NX), u1 in the laboratory frame for shear
 * (binv(1,1) u1 + binv(1,3) u3) and arr_u1 the stored component; lint11 += the same product
 * times dx_laboratoryframe (2 pi B110 / NX, src/pg_domain.f90:178-183).  out[0..NX/2] =
 * temp_r1i, out[NX/2 + 1] = lint11.  The state is truncated first as at a stage's start. */
void oracle_x_correlation(oracle* o, double* out) {
    dealias(o);
    spec_to_phys(o, o->u[0], o->phys[0]);
    spec_to_phys(o, o->u[2], o->phys[2]);
    const int nx = o->nx, nl = nx / 2 + 1;
    const double dxl = ((double)(6.283185307179586476925286766559005768L) * (double)o->p.b110) / (double)nx;
    for (int l = 0; l <= nl; l++) out[l] = 0.0;
    double lint = 0.0;
    for (long zy = 0; zy < (long)o->ny * o->nz; zy++) {
        const double* a = o->phys[0] + zy * nx;
        const double* a3 = o->phys[2] + zy * nx;
        for (int i = 0; i < nx; i++) {
            double u1 = a[i];
            if (o->p.f_type != PANDORA_F_ISOTROPIC) u1 = (0.0 + o->binv[0][0] * a[i]) + o->binv[0][2] * a3[i];
            for (int ii = i; ii <= i + (nx - 1) / 2 + 1; ii++) {
                const double v = ii <= nx - 1 ? a[ii] : a[ii - nx];
                out[ii - i] = out[ii - i] + u1 * v;
                lint = lint + (u1 * v * dxl);
            }
        }
    }
    out[nl] = lint;
}

int oracle_nonlinear(oracle* o, double* a, double* b, double* c) {
    compute_nonlinear(o, 0);
    oracle_get_nl(o, a, b, c);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* forcing f_ForceCalc (src/pf_force.f90:106-268)                              */
/* ------------------------------------------------------------------------- */
static inline cx* fref(oracle* o, int c, int i, int j, int k) {
    int NK = o->fnk, W = 2 * NK + 1;
    return &o->ff[c][((long)i * W + (j + NK)) * W + (k + NK)];
}
long oracle_force_calls_per_stage(const oracle* o);
long oracle_force_calls_per_stage(const oracle* o) {
    long NK = o->fnk;
    return 3 * ((NK + 1) * (NK + 1) + NK * (NK + 1)) + 3 * NK * (2 * NK + 1) * (2 * NK + 1);
}
static void force_calc(oracle* o, int tstep, int stage, double dt) {
    const pandora_params* p = &o->p;
    int NK = o->fnk;
    long nf = (long)(NK + 1) * (2 * NK + 1) * (2 * NK + 1);
    if (tstep >= p->force_stop) {
        for (int c = 0; c < 3; c++) memset(o->ff[c], 0, sizeof(cx) * nf);
        return;
    }
    uint64_t key = pd_stream_key(p->seed_force, PD_TAG_FORCE);
    uint64_t call = ((uint64_t)tstep * 3 + (uint64_t)(stage - 1)) * (uint64_t)oracle_force_calls_per_stage(o);
    double dt_over_TF = dt / p->force_tf;
    double amp = sqrt(2.0 * (p->force_sigma * p->force_sigma) * dt_over_TF);
    double decay = 1.0 - dt_over_TF;
    double re[3], im[3];
#define DRAW3()                                                                    \
    do {                                                                           \
        for (int c = 0; c < 3; c++)                                                \
            if (pd_normal_pair(key, call++, &re[c], &im[c])) o->status |= 2;       \
    } while (0)
#define OU(i, j, k)                                                                \
    do {                                                                           \
        for (int c = 0; c < 3; c++) {                                              \
            cx* f = fref(o, c, i, j, k);                                           \
            f->re = f->re * decay + re[c] * amp;                                   \
            f->im = f->im * decay + im[c] * amp;                                   \
        }                                                                          \
    } while (0)
#define CONJ(id, jd, kd, is, js, ks)                                               \
    do {                                                                           \
        for (int c = 0; c < 3; c++) {                                              \
            cx* s = fref(o, c, is, js, ks);                                        \
            cx* d = fref(o, c, id, jd, kd);                                        \
            d->re = s->re;                                                         \
            d->im = -s->im;                                                        \
        }                                                                          \
    } while (0)
    for (int j = 0; j <= NK; j++) {
        for (int k = 0; k <= NK; k++) {
            DRAW3();
            OU(0, j, k);
            CONJ(0, -j, -k, 0, j, k);
            if (j > 0) {
                DRAW3();
                OU(0, -j, k);
                CONJ(0, j, -k, 0, -j, k);
            }
        }
    }
    for (int i = 1; i <= NK; i++)
        for (int j = -NK; j <= NK; j++)
            for (int k = -NK; k <= NK; k++) {
                DRAW3();
                OU(i, j, k);
            }
#undef DRAW3
#undef OU
#undef CONJ
}

/* ------------------------------------------------------------------------- */
/* f_RK3FormFIsotropic + f_RK3RungeKutta + f_RK3ContinuityFixIsotropic          */
/* (src/pf_rk3.f90:2323-2487, 3457-3531)                                        */
/* ------------------------------------------------------------------------- */
void rk_coeffs(int stage, double* beta, double* gamma) {
    if (stage == 1) { *beta = 0.0; *gamma = 1.0 / 3.0; }
    else if (stage == 2) { *beta = -(5.0 / 9.0); *gamma = 15.0 / 16.0; }
    else { *beta = -(153.0 / 128.0); *gamma = 8.0 / 15.0; }
}

/* Integrating-factor variant (PANDORA_VISCOUS_INTEGRATING_FACTOR, no counterpart in
 * the reference, whose viscous term is explicit): the low-storage RK3 applied to
 * v = exp(nu k^2 (t - t0)) u with u and the register stored in physical units, so stage s
 * scales both by E_s = exp(-nu k^2 (c_{s+1} - c_s) dt), c = 0, 1/3, 3/4, 1, and the
 * right-hand side drops -nu k^2 u. */
static double if_fraction(int stage) {
    return stage == 1 ? 1.0 / 3.0 : (stage == 2 ? 5.0 / 12.0 : 1.0 / 4.0);
}

static void form_f_iso(oracle* o, int stage, double dt) {
    double beta, gamma;
    rk_coeffs(stage, &beta, &gamma);
    const double nu = o->p.f_nu, kf = o->p.force_kf;
    const int ifac = o->p.rk3_viscous == PANDORA_VISCOUS_INTEGRATING_FACTOR;
    const double dcs = if_fraction(stage);
    const int NK = o->fnk;
#pragma omp parallel for schedule(static)
    for (long ij = 0; ij < (long)o->nki * o->nkj; ij++) {
        int i = (int)(ij / o->nkj), j = (int)(ij % o->nkj);
        double k1 = wvn(i, o->ki), k2 = wvn(j, o->kj);
        for (int k = 0; k < o->nkk; k++) {
            long m = ij * o->nkk + k;
            double k3 = wvn(k, o->kk);
            double kmag2 = (k1 * k1) + (k2 * k2) + (k3 * k3);
            if (!(kmag2 > 0.0)) continue;
            cx uu[3] = {o->u[0][m], o->u[1][m], o->u[2][m]};
            cx nl[3] = {o->nl[0][m], o->nl[1][m], o->nl[2][m]};
            double kv[3] = {k1, k2, k3};
            cx tot[3];
            cx kdn = {(k1 * nl[0].re) + (k2 * nl[1].re) + (k3 * nl[2].re),
                      (k1 * nl[0].im) + (k2 * nl[1].im) + (k3 * nl[2].im)};
            cx force[3] = {{0, 0}, {0, 0}, {0, 0}};
            double kmag = sqrt(kmag2);
            if (kmag <= kf && kmag > 0.0) {
                int jw = (int)k2, kw = (int)k3;
                if (jw >= -NK && jw <= NK && kw >= -NK && kw <= NK && i <= NK) {
                    cx f[3];
                    for (int c = 0; c < 3; c++) f[c] = *fref(o, c, i, jw, kw);
                    cx kdb = {k1 * f[0].re + k2 * f[1].re + k3 * f[2].re,
                              k1 * f[0].im + k2 * f[1].im + k3 * f[2].im};
                    for (int c = 0; c < 3; c++) {
                        force[c].re = f[c].re - ((kv[c] / kmag2) * kdb.re);
                        force[c].im = f[c].im - ((kv[c] / kmag2) * kdb.im);
                    }
                }
            }
            if (ifac) {
                const double ex = exp(-(nu * kmag2 * dcs * dt));
                for (int c = 0; c < 3; c++) {
                    double pr = (kv[c] / kmag2) * kdn.re, pi = (kv[c] / kmag2) * kdn.im;
                    tot[c].re = -nl[c].re + pr + force[c].re;
                    tot[c].im = -nl[c].im + pi + force[c].im;
                }
                for (int c = 0; c < 3; c++) {
                    cx* r = &o->rk[c][m];
                    r->re = ex * ((beta * r->re) + tot[c].re);
                    r->im = ex * ((beta * r->im) + tot[c].im);
                    uu[c].re = (ex * uu[c].re) + (gamma * dt * r->re);
                    uu[c].im = (ex * uu[c].im) + (gamma * dt * r->im);
                }
            } else {
                for (int c = 0; c < 3; c++) {
                    double vr = -nu * kmag2 * uu[c].re, vi = -nu * kmag2 * uu[c].im;
                    double pr = (kv[c] / kmag2) * kdn.re, pi = (kv[c] / kmag2) * kdn.im;
                    tot[c].re = vr - nl[c].re + pr + force[c].re + 0.0;
                    tot[c].im = vi - nl[c].im + pi + force[c].im + 0.0;
                }
                for (int c = 0; c < 3; c++) {
                    cx* r = &o->rk[c][m];
                    r->re = (beta * r->re) + tot[c].re;
                    r->im = (beta * r->im) + tot[c].im;
                    uu[c].re = uu[c].re + (gamma * dt * r->re);
                    uu[c].im = uu[c].im + (gamma * dt * r->im);
                }
            }
            cx kdu = {k1 * uu[0].re + k2 * uu[1].re + k3 * uu[2].re,
                      k1 * uu[0].im + k2 * uu[1].im + k3 * uu[2].im};
            for (int c = 0; c < 3; c++) {
                uu[c].re = uu[c].re - (kv[c] * kdu.re / kmag2);
                uu[c].im = uu[c].im - (kv[c] * kdu.im / kmag2);
                o->u[c][m] = uu[c];
            }
        }
    }
}

/* ------------------------------------------------------------------------- */
/* particles                                                                    */
/* ------------------------------------------------------------------------- */
void oracle_set_particles(oracle* o, long np, const double* xp, const double* up,
                          const double* uprk, const double* prk, const double* dp) {
    free(o->xp); free(o->up); free(o->uprk); free(o->prk); free(o->dp);
    o->np = np;
    o->xp = dalloc(3 * np); o->up = dalloc(3 * np); o->uprk = dalloc(3 * np);
    o->prk = dalloc(3 * np); o->dp = dalloc(np);
    if (xp) memcpy(o->xp, xp, sizeof(double) * 3 * np);
    if (up) memcpy(o->up, up, sizeof(double) * 3 * np);
    if (uprk) memcpy(o->uprk, uprk, sizeof(double) * 3 * np);
    if (prk) memcpy(o->prk, prk, sizeof(double) * 3 * np);
    if (dp) memcpy(o->dp, dp, sizeof(double) * np);
}
void oracle_get_particles(const oracle* o, double* xp, double* up, double* uprk, double* prk,
                          double* dp) {
    if (xp) memcpy(xp, o->xp, sizeof(double) * 3 * o->np);
    if (up) memcpy(up, o->up, sizeof(double) * 3 * o->np);
    if (uprk) memcpy(uprk, o->uprk, sizeof(double) * 3 * o->np);
    if (prk) memcpy(prk, o->prk, sizeof(double) * 3 * o->np);
    if (dp) memcpy(dp, o->dp, sizeof(double) * o->np);
}

/* P_INIT_RANDOM (src/pp_control.f90:663-707): xp = rn * L - dx/2 per component,
 * three draws per particle in particle order; diameter P_DIA_VALS. */
void oracle_init_particles(oracle* o) {
    long np = o->p.p_np_global;
    oracle_set_particles(o, np, NULL, NULL, NULL, NULL, NULL);
    uint64_t key = pd_stream_key(o->p.seed_particles, PD_TAG_PART);
    double L[3] = {o->lx, o->ly, o->lz}, D[3] = {o->dx, o->dy, o->dz};
    for (long n = 0; n < np; n++) {
        for (int c = 0; c < 3; c++) {
            long double rn = (long double)pd_uniform(key, (uint64_t)(3 * n + c));
            o->xp[3 * n + c] = (double)(rn * (long double)L[c] - ((long double)D[c] * 0.5L));
        }
        o->dp[n] = o->p.p_dia_vals;
    }
}

/* p_InterpFindMolecule + p_InterpNeville3D (src/pp_interp.f90:313-560) */
static void interp3d(const oracle* o, const double* xp, double* uf) {
    const int ord = o->p.p_interp_order, nh = ord / 2;
    const double D[3] = {o->dx, o->dy, o->dz};
    const int NN[3] = {o->nx, o->ny, o->nz};
    int i0[3];
    double nodes[3][16];
    for (int c = 0; c < 3; c++) {
        double halo = (double)nh * D[c];
        if (ord % 2 == 0) halo = halo - (0.5 * D[c]);
        double xd;
        if (ord % 2 == 0) xd = xp[c] + halo + D[c] + (0.5 * D[c]);
        else xd = xp[c] + halo + (0.5 * D[c]);
        int idx = (int)(xd / D[c]) - nh - nh;
        i0[c] = idx;
        for (int m = 0; m < ord; m++) nodes[c][m] = (double)(idx + m) * D[c];
    }
    /* values v[comp][xi][zi][yi] (reference array order (x, z, y)) */
    double v[3][8][8][8];
    for (int xi = 0; xi < ord; xi++)
        for (int zi = 0; zi < ord; zi++)
            for (int yi = 0; yi < ord; yi++) {
                int X = ((i0[0] + xi) % NN[0] + NN[0]) % NN[0];
                int Y = ((i0[1] + yi) % NN[1] + NN[1]) % NN[1];
                int Z = ((i0[2] + zi) % NN[2] + NN[2]) % NN[2];
                long pidx = ((long)Z * NN[1] + Y) * NN[0] + X;
                for (int c = 0; c < 3; c++) v[c][xi][zi][yi] = o->phys[c][pidx];
            }
    /* along y */
    for (int col = 1; col <= ord - 1; col++)
        for (int nv = 0; nv < ord - col; nv++) {
            double d1 = xp[1] - nodes[1][nv + col], d2 = nodes[1][nv] - xp[1];
            double d3 = nodes[1][nv] - nodes[1][nv + col];
            for (int zi = 0; zi < ord; zi++)
                for (int xi = 0; xi < ord; xi++)
                    for (int c = 0; c < 3; c++)
                        v[c][xi][zi][nv] = ((d1 * v[c][xi][zi][nv]) + (d2 * v[c][xi][zi][nv + 1])) / d3;
        }
    /* along z */
    for (int col = 1; col <= ord - 1; col++)
        for (int nv = 0; nv < ord - col; nv++) {
            double d1 = xp[2] - nodes[2][nv + col], d2 = nodes[2][nv] - xp[2];
            double d3 = nodes[2][nv] - nodes[2][nv + col];
            for (int xi = 0; xi < ord; xi++)
                for (int c = 0; c < 3; c++)
                    v[c][xi][nv][0] = ((d1 * v[c][xi][nv][0]) + (d2 * v[c][xi][nv + 1][0])) / d3;
        }
    /* along x */
    for (int col = 1; col <= ord - 1; col++)
        for (int nv = 0; nv < ord - col; nv++) {
            double d1 = xp[0] - nodes[0][nv + col], d2 = nodes[0][nv] - xp[0];
            double d3 = nodes[0][nv] - nodes[0][nv + col];
            for (int c = 0; c < 3; c++)
                v[c][nv][0][0] = ((d1 * v[c][nv][0][0]) + (d2 * v[c][nv + 1][0][0])) / d3;
        }
    for (int c = 0; c < 3; c++) uf[c] = v[c][0][0][0];
}

int oracle_interpolate(const oracle* o, long n, const double* xp, double* uf) {
    for (long q = 0; q < n; q++) interp3d(o, xp + 3 * q, uf + 3 * q);
    return 0;
}

/* p_ControlRK3 -> p_RK3SolveParticle (src/pp_rk3.f90:57-165), then the wrap of
 * p_MPICorrectPosition (src/pp_mpi.f90:1011-1057) and the inside test of
 * p_MPIFindLocalParticles (src/pp_mpi.f90:1164-1191). */
static void particles_stage(oracle* o, int stage, int tstep, double dt) {
    if (!o->p.p_track_part || tstep < o->p.p_ts_release || o->np == 0) return;
    double beta, gamma;
    rk_coeffs(stage, &beta, &gamma);
    const int init_vel = (tstep == o->p.p_ts_release && stage == 1);
    const double x1min = -0.5 * o->dx, x2min = -0.5 * o->dy, x3min = -0.5 * o->dz;
    const double x1max = x1min + o->lx, x2max = x2min + o->ly, x3max = x3min + o->lz;
    const double ymin = 0.0 * o->dy - (0.5 * o->dy), ymax = (double)o->ny * o->dy - (0.5 * o->dy);
    const double zmin = 0.0 * o->dz - (0.5 * o->dz), zmax = (double)o->nz * o->dz - (0.5 * o->dz);
    int lost = 0;
#pragma omp parallel for schedule(static) reduction(| : lost)
    for (long n = 0; n < o->np; n++) {
        double* xp = o->xp + 3 * n;
        double* up = o->up + 3 * n;
        double* ur = o->uprk + 3 * n;
        double* pr = o->prk + 3 * n;
        double uf[3];
        /* the R forms: p_RK3SolveParticleR (src/pp_rk3.f90:307-403, dispatched at
         * src/pp_control.f90:568-571) and p_ControlInitPartVelocityR (418-463) are the
         * isotropic arithmetic on the laboratory components of the sheared grid */
        if (o->shear && !o->rrot) {
            /* p_RK3SolveParticleBF (src/pp_rk3.f90:169-303): RK3 in the lab frame,
             * p_RK3Mov2Lab / p_RK3Lab2Mov (src/pp_rk3.f90:989-1042) */
            double ufm[3], xl[3] = {0, 0, 0}, ul[3] = {0, 0, 0};
            interp3d(o, xp, ufm);
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++)
                    if (o->bexist[a][b]) { xl[a] = xl[a] + o->binv[a][b] * xp[b]; ul[a] = ul[a] + o->binv[a][b] * ufm[b]; }
            if (init_vel) {   /* p_ControlInitPartVelocityBF (src/pp_control.f90:466-516) */
                for (int c = 0; c < 3; c++) { up[c] = ul[c]; pr[c] = 0.0; ur[c] = 0.0; }
            }
            double dpv = o->dp[n];
            if (dpv > 0.0) {
                double tau = ((dpv * dpv) / (18.0 * o->p.f_nu)) * (o->p.p_rho / o->p.f_rho);
                double hs[3] = {0, 0, 0};   /* p_RK3ComputeHomogeneousSourceTerm (src/pp_rk3.f90:1080-1102) */
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++)
                        if (o->aexist[a][b]) hs[a] = hs[a] + o->amat[a][b] * up[b];
                for (int c = 0; c < 3; c++) {
                    double acc = ((ul[c] - up[c]) / tau) - hs[c];
                    pr[c] = (beta * pr[c]) + acc;
                    up[c] = up[c] + (gamma * dt * pr[c]);
                }
            } else {
                for (int c = 0; c < 3; c++) up[c] = ul[c];
            }
            for (int c = 0; c < 3; c++) {
                ur[c] = (beta * ur[c]) + up[c];
                xl[c] = xl[c] + (gamma * dt * ur[c]);
            }
            double xm[3] = {0, 0, 0};
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++)
                    if (o->bexist[a][b]) xm[a] = xm[a] + o->bmat[a][b] * xl[b];
            for (int c = 0; c < 3; c++) xp[c] = xm[c];
        } else {
        if (init_vel) {   /* p_ControlInitPartVelocity (src/pp_control.f90:378-416) */
            interp3d(o, xp, uf);
            for (int c = 0; c < 3; c++) { up[c] = uf[c]; pr[c] = 0.0; ur[c] = 0.0; }
        }
        interp3d(o, xp, uf);
        double dpv = o->dp[n];
        if (dpv > 0.0) {
            double tau = ((dpv * dpv) / (18.0 * o->p.f_nu)) * (o->p.p_rho / o->p.f_rho);
            for (int c = 0; c < 3; c++) {
                double acc = (uf[c] - up[c]) / tau;
                pr[c] = (beta * pr[c]) + acc;
                up[c] = up[c] + (gamma * dt * pr[c]);
            }
        } else {
            for (int c = 0; c < 3; c++) up[c] = uf[c];
        }
        for (int c = 0; c < 3; c++) {
            ur[c] = (beta * ur[c]) + up[c];
            xp[c] = xp[c] + (gamma * dt * ur[c]);
        }
        }
        if (xp[0] < x1min) xp[0] = xp[0] + o->lx;
        if (xp[0] >= x1max) xp[0] = xp[0] - o->lx;
        if (xp[1] < x2min) xp[1] = xp[1] + o->ly;
        if (xp[1] >= x2max) xp[1] = xp[1] - o->ly;
        if (xp[2] < x3min) xp[2] = xp[2] + o->lz;
        if (xp[2] > x3max) xp[2] = xp[2] - o->lz;
        if (!(xp[1] >= ymin && xp[1] < ymax && xp[2] >= zmin && xp[2] < zmax)) lost |= 1;
    }
    if (lost) o->status |= 4;
}


/* p_ControlRemesh -> p_MPIRemeshPosition (src/pp_mpi.f90:1062-1092): x1 += x3, one wrap */
static void particles_remesh(oracle* o) {
    if (!o->p.p_track_part || o->np == 0) return;
    const double x1min = -0.5 * o->dx, x1max = x1min + o->lx;
    for (long n = 0; n < o->np; n++) {
        double* xp = o->xp + 3 * n;
        xp[0] = xp[0] + xp[2];
        if (xp[0] < x1min) xp[0] = xp[0] + o->lx;
        if (xp[0] >= x1max) xp[0] = xp[0] - o->lx;
    }
}

/* ------------------------------------------------------------------------- */
/* statistics (src/pf_fluidstats.f90:336-374, 696-780, 1423-1576)              */
/* ------------------------------------------------------------------------- */
static void mode_density(oracle* o) {
    double kmax = sqrt((double)((long)o->ki * o->ki + (long)o->kj * o->kj + (long)o->kk * o->kk));
    if (o->p.f_type != PANDORA_F_ISOTROPIC) {
        const pandora_params* p = &o->p;
        kmax = sqrt((double)((double)o->ki * o->ki / (double)(p->b110 * p->b110) +
                             (double)o->kj * o->kj / (double)(p->b220 * p->b220) +
                             (double)o->kk * o->kk / (double)(p->b330 * p->b330)));
    }
    double kmin = 1.0;
    o->kkmax = (int)lround(kmax / kmin);
    free(o->dens_mod);
    o->dens_mod = dalloc(o->kkmax + 1);
    long* cnt = (long*)calloc((size_t)o->kkmax + 2, sizeof(long));
    for (int i = 0; i < o->nki; i++)
        for (int j = 0; j < o->nkj; j++)
            for (int k = 0; k < o->nkk; k++) {
                double a = wvn(i, o->ki), b = wvn(j, o->kj), c = wvn(k, o->kk);
                double km = sqrt((a * a) + (b * b) + (c * c));
                for (int kk = 1; kk <= o->kkmax; kk++) {
                    double up = (double)kk + (kmin * 0.5), lo = (double)kk - (kmin * 0.5);
                    if (km >= lo && km < up) cnt[kk] += (i != 0) ? 2 : 1;
                }
            }
    const double pi = (double)(3.14159265358979323846264338327950288L);
    for (int kk = 1; kk <= o->kkmax; kk++) {
        double up = (double)kk + (kmin * 0.5), lo = (double)kk - (kmin * 0.5);
        o->dens_mod[kk] = (double)cnt[kk] / (4.0 / 3.0 * pi * (up * up * up - lo * lo * lo));
    }
    free(cnt);
}


/* lab-frame statistics of the moving-frame state, f_FluidstatsModeDensityBFRot
 * (src/pf_fluidstats.f90:1977-2229) and f_FluidstatsFsPrimaryQuantsBFRot
 * (src/pf_fluidstats.f90:1586-1960): k_lab = B^T k, u_lab = B^-1 u, mode density
 * recomputed for the current B and divided by B110 B220 B330. */
static void stats_bf(const oracle* o, double* ek, double* tke, double* eps) {
    const int K = o->kkmax;
    double* spec = dalloc(K + 1);
    double* dis = dalloc(K + 1);
    long* cnt = (long*)calloc((size_t)K + 2, sizeof(long));
    double s11 = 0, s22 = 0, s33 = 0;
    const double nu = o->p.f_nu;
    for (int i = 0; i < o->nki; i++)
        for (int j = 0; j < o->nkj; j++)
            for (int k = 0; k < o->nkk; k++) {
                long m = ((long)i * o->nkj + j) * o->nkk + k;
                double km_[3] = {wvn(i, o->ki), wvn(j, o->kj), wvn(k, o->kk)};
                cx um[3] = {o->u[0][m], o->u[1][m], o->u[2][m]};
                double kl[3] = {0, 0, 0};
                cx ul[3] = {{0, 0}, {0, 0}, {0, 0}};
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++)
                        if (o->bexist[a][b]) {
                            kl[b] = kl[b] + o->bmat[a][b] * km_[a];
                            ul[a].re = ul[a].re + o->binv[a][b] * um[b].re;
                            ul[a].im = ul[a].im + o->binv[a][b] * um[b].im;
                        }
                /* f_FluidstatsFsPrimaryQuantsRRot: the R-rot state already holds the
                 * laboratory components (src/pf_fluidstats.f90, ulab = umov) */
                if (o->rrot) { ul[0] = um[0]; ul[1] = um[1]; ul[2] = um[2]; }
                double km = sqrt((kl[0] * kl[0]) + (kl[1] * kl[1]) + (kl[2] * kl[2]));
                double p11 = ul[0].re * ul[0].re + ul[0].im * ul[0].im;
                double p22 = ul[1].re * ul[1].re + ul[1].im * ul[1].im;
                double p33 = ul[2].re * ul[2].re + ul[2].im * ul[2].im;
                if (i != 0) { p11 *= 2.0; p22 *= 2.0; p33 *= 2.0; }
                s11 += p11; s22 += p22; s33 += p33;
                double e = 0.5 * (p11 + p22 + p33);
                double d = 2.0 * km * km * nu * e;
                int kc = (int)floor(km + 0.5);
                for (int q = kc - 1; q <= kc + 1; q++) {
                    if (q < 1 || q > K) continue;
                    double up = 1.0 * ((double)q + 0.5), lo = 1.0 * ((double)q - 0.5);
                    if (km >= lo && km < up) { spec[q] += e; dis[q] += d; cnt[q] += (i != 0) ? 2 : 1; }
                }
            }
    const double pi = (double)(3.14159265358979323846264338327950288L);
    const double bvol = (double)o->p.b110 * (double)o->p.b220 * (double)o->p.b330;
    double fdis = 0.0;
    for (int q = 1; q <= K; q++) {
        double up = (double)q + 0.5, lo = (double)q - 0.5;
        double dm = (double)cnt[q] / (4.0 / 3.0 * pi * (up * up * up - lo * lo * lo));
        dm = dm / bvol;
        if (dm != 0.0) {
            fdis += dis[q];
            if (ek) ek[q - 1] = spec[q] / dm;
        } else if (ek) {
            ek[q - 1] = spec[q];
        }
    }
    if (tke) *tke = 0.5 * (s11 + s22 + s33);
    if (eps) *eps = fdis;
    free(spec); free(dis); free(cnt);
}

/* ek[0..kkmax-1] = E(k) for shells kk=1..kkmax; tke; eps = f_dis. */
void oracle_stats(const oracle* o, double* ek, double* tke, double* eps) {
    if (o->p.f_type != PANDORA_F_ISOTROPIC) { stats_bf(o, ek, tke, eps); return; }
    const int K = o->kkmax;
    double* spec = dalloc(K + 1);
    double* dis = dalloc(K + 1);
    double s11 = 0, s22 = 0, s33 = 0;
    const double nu = o->p.f_nu;
    for (int i = 0; i < o->nki; i++)
        for (int j = 0; j < o->nkj; j++)
            for (int k = 0; k < o->nkk; k++) {
                long m = ((long)i * o->nkj + j) * o->nkk + k;
                double a = wvn(i, o->ki), b = wvn(j, o->kj), c = wvn(k, o->kk);
                double km = sqrt((a * a) + (b * b) + (c * c));
                cx u1 = o->u[0][m], u2 = o->u[1][m], u3 = o->u[2][m];
                double p11 = u1.re * u1.re + u1.im * u1.im;
                double p22 = u2.re * u2.re + u2.im * u2.im;
                double p33 = u3.re * u3.re + u3.im * u3.im;
                if (i != 0) { p11 *= 2.0; p22 *= 2.0; p33 *= 2.0; }
                s11 += p11; s22 += p22; s33 += p33;
                double e = 0.5 * (p11 + p22 + p33);
                double d = 2.0 * km * km * nu * e;
                int kk = (int)floor(km + 0.5);
                /* bin test exactly as the reference: lo <= km < up */
                for (int q = kk - 1; q <= kk + 1; q++) {
                    if (q < 1 || q > K) continue;
                    double up = (double)q + 0.5, lo = (double)q - 0.5;
                    if (km >= lo && km < up) { spec[q] += e; dis[q] += d; }
                }
            }
    double fdis = 0.0;
    for (int q = 1; q <= K; q++) {
        if (o->dens_mod[q] != 0.0) {
            fdis += dis[q];
            if (ek) ek[q - 1] = spec[q] / o->dens_mod[q];
        } else if (ek) {
            ek[q - 1] = spec[q];
        }
    }
    if (tke) *tke = 0.5 * (s11 + s22 + s33);
    if (eps) *eps = fdis;
    free(spec); free(dis);
}

/* ------------------------------------------------------------------------- */
/* initial field f_InitialiseFluid (src/pf_initialise.f90:97-512)              */
/* ------------------------------------------------------------------------- */
static double init_spec(const pandora_params* p, double kmag) {
    const double pi = (double)(3.14159265358979323846264338327950288L);
    switch (p->f_init_type) {
    case PANDORA_F_INIT_GAUSS:
        return (p->f_init_u0 / (p->f_init_kv * sqrt(4.0 * asin(1.0)))) *
               exp(-((kmag - p->f_init_kp) * (kmag - p->f_init_kp)) / (2.0 * (p->f_init_kv * p->f_init_kv)));
    case PANDORA_F_INIT_KERR:
        return (p->f_init_u0 / (4.0 * asin(1.0))) * (kmag * kmag * kmag * kmag) *
               exp(-(2.0 * kmag * kmag) / (p->f_init_kp * p->f_init_kp));
    case PANDORA_F_INIT_PULSE:
        return (sqrt((kmag - p->f_init_kp) * (kmag - p->f_init_kp)) < p->f_init_kv) ? p->f_init_u0 : 0.0;
    case PANDORA_F_INIT_SQUARE:
        return (kmag > p->f_init_kstart && kmag < p->f_init_kend) ? 1.0 : 0.0;
    case PANDORA_F_INIT_MINUSFIVETHIRD:
        if (kmag < p->f_init_kstart)
            return 1.5 * pow(p->f_init_epsilon, 2.0 / 3.0) * pow(p->f_init_kstart, -5.0 / 3.0) *
                   ((kmag / p->f_init_kstart) * (kmag / p->f_init_kstart));
        if (kmag < p->f_init_kend)
            return 1.5 * pow(p->f_init_epsilon, 2.0 / 3.0) * pow(p->f_init_kstart, -5.0 / 3.0) *
                   pow(kmag / p->f_init_kstart, -5.0 / 3.0);
        return 0.0;
    case PANDORA_F_INIT_MATSUMOTO:
        if (kmag < p->f_init_kstart) return p->f_init_u0 * (kmag * kmag);
        if (kmag < p->f_init_kend)
            return p->f_init_u0 * pow(p->f_init_kstart, 11.0 / 3.0) * pow(kmag, -5.0 / 3.0);
        return 0.0;
    case PANDORA_F_INIT_AHMED_ELGHOBASHI: {
        double k4 = (kmag * kmag) * (kmag * kmag);
        double kp = p->f_init_kp, kp5 = kp * kp * kp * kp * kp;
        return 16.0 * pow(2.0 / pi, 0.5) * 1.5 * p->f_init_u0 * (k4 / kp5) *
               exp(-(2.0 * kmag * kmag) / (kp * kp));
    }
    default:
        return 0.0;
    }
}

/* Rogallo construction of one mode from three uniform draws (src/pf_initialise.f90:160-205) */
static void rogallo_mode(const pandora_params* p, double k1, double k2, double k3, double kmag,
                         double r1, double r2, double r3, cx t[3], double fdiv) {
    const double twopi = (double)(6.283185307179586476925286766559005768L);
    const double fourpi = (double)(12.566370614359172953850573533118011536L);
    r1 = twopi * r1; r2 = twopi * r2; r3 = twopi * r3;
    double k2d = (k1 * k1) + (k2 * k2);
    for (int c = 0; c < 3; c++) t[c].re = t[c].im = 0.0;
    if (!(kmag > 0.0)) return;
    double ek = init_spec(p, kmag);
    double factor = sqrt(ek / (fourpi * kmag * kmag));
    if (fdiv != 1.0) factor = factor / fdiv;
    cx al = {factor * cos(r1) * cos(r3), factor * sin(r1) * cos(r3)};
    cx be = {factor * cos(r2) * sin(r3), factor * sin(r2) * sin(r3)};
    if (!(k2d > 0.0)) return;
    double den = kmag * sqrt(k2d);
    t[0].re = (al.re * kmag * k2 + be.re * k1 * k3) / den;
    t[0].im = (al.im * kmag * k2 + be.im * k1 * k3) / den;
    t[1].re = (be.re * k2 * k3 - al.re * kmag * k1) / den;
    t[1].im = (be.im * k2 * k3 - al.im * kmag * k1) / den;
    t[2].re = -(be.re * sqrt(k2d)) / kmag;
    t[2].im = -(be.im * sqrt(k2d)) / kmag;
}

/* f_InitialiseFluid (src/pf_initialise.f90:97-512) and, when
 * B110+B220+B330 > 3, f_InitialiseFluidDeformed (src/pf_initialise.f90:520-990):
 * wavenumbers scaled by 1/B, amplitude by (B110 B220 B330)^-1/2, velocity mapped
 * through bmat.  Same draw order in both. */
static void deform_map(const oracle* o, cx t[3]) {
    cx d[3] = {{0, 0}, {0, 0}, {0, 0}};
    for (int m = 0; m < 3; m++)
        for (int n = 0; n < 3; n++)
            if (o->bexist[m][n]) {
                d[m].re = d[m].re + o->bmat[m][n] * t[n].re;
                d[m].im = d[m].im + o->bmat[m][n] * t[n].im;
            }
    for (int c = 0; c < 3; c++) t[c] = d[c];
}

void oracle_init_fluid(oracle* o) {
    const pandora_params* p = &o->p;
    uint64_t key = pd_stream_key(p->seed_fluid, PD_TAG_FLUID);
    uint64_t n = 0;
    const int KJ = o->kj, KK = o->kk, NKJ = o->nkj, NKK = o->nkk, KI = o->ki;
    const int deformed = (p->b110 + p->b220 + p->b330) > 3;
    const double b1 = deformed ? (double)p->b110 : 1.0, b2 = deformed ? (double)p->b220 : 1.0;
    const double b3 = deformed ? (double)p->b330 : 1.0;
    const double fdiv = deformed ? pow((double)p->b110 * (double)p->b220 * (double)p->b330, 0.5) : 1.0;
    for (int c = 0; c < 3; c++) memset(o->u[c], 0, sizeof(cx) * o->S);
#define U(c, i, j, k) o->u[c][((long)(i) * NKJ + (j)) * NKK + (k)]
    /* i = 0 plane with conjugate symmetry */
    double k1 = wvn(0, KI) / b1;
    for (int j = 0; j <= KJ; j++) {
        double k2 = wvn(j, KJ) / b2;
        for (int k = 0; k <= KK; k++) {
            double k3 = wvn(k, KK) / b3;
            double r1 = pd_uniform(key, n++), r2 = pd_uniform(key, n++), r3 = pd_uniform(key, n++);
            double kmag = sqrt((k1 * k1) + (k2 * k2) + (k3 * k3));
            cx t[3];
            rogallo_mode(p, k1, k2, k3, kmag, r1, r2, r3, t, fdiv);
            if (deformed) deform_map(o, t);
            int jj = (j != 0) ? NKJ - j : j;
            int kk = (k != 0) ? NKK - k : k;
            for (int c = 0; c < 3; c++) U(c, 0, j, k) = t[c];
            for (int c = 0; c < 3; c++) { U(c, 0, jj, kk).re = t[c].re; U(c, 0, jj, kk).im = -t[c].im; }
            if (k != 0) {
                double k2n = wvn(jj, KJ);
                if (deformed || p->b220 > 1) k2n = k2n / (double)p->b220;
                r1 = pd_uniform(key, n++); r2 = pd_uniform(key, n++); r3 = pd_uniform(key, n++);
                rogallo_mode(p, k1, k2n, k3, kmag, r1, r2, r3, t, fdiv);
                if (deformed) deform_map(o, t);
                for (int c = 0; c < 3; c++) U(c, 0, jj, k) = t[c];
                for (int c = 0; c < 3; c++) { U(c, 0, j, kk).re = t[c].re; U(c, 0, j, kk).im = -t[c].im; }
            }
        }
    }
    /* i >= 1; loops run one index past the stored range (draws consumed) */
    for (int i = 1; i <= o->nki; i++) {
        double a = wvn(i, KI) / b1;
        for (int j = 0; j <= NKJ; j++) {
            double b = wvn(j, KJ) / b2;
            for (int k = 0; k <= NKK; k++) {
                double c3 = wvn(k, KK) / b3;
                double r1 = pd_uniform(key, n++), r2 = pd_uniform(key, n++), r3 = pd_uniform(key, n++);
                if (i > KI || j >= NKJ || k >= NKK) continue;
                double kmag = sqrt((a * a) + (b * b) + (c3 * c3));
                cx t[3];
                rogallo_mode(p, a, b, c3, kmag, r1, r2, r3, t, fdiv);
                if (deformed) deform_map(o, t);
                for (int c = 0; c < 3; c++) U(c, i, j, k) = t[c];
            }
        }
    }
#undef U
    dealias(o);   /* src/pf_initialise.f90:75-83 */
}

/* tf_RK3InitTaylorGreenReverse (src/ptf_rk3.f90:1030-1105) */
void oracle_init_taylor_green_reverse(oracle* o) {
    for (int c = 0; c < 3; c++) memset(o->u[c], 0, sizeof(cx) * o->S);
    const double e8 = 1.0 / 8.0, e24 = 1.0 / 24.0;
    const int NKJ = o->nkj, NKK = o->nkk;
#define U(c, i, j, k) o->u[c][((long)(i) * NKJ + (j)) * NKK + (k)]
    if (o->nki < 2 || o->kj < 2 || o->kk < 3) return;
    U(0, 1, 2, 3).re = -e8; U(1, 1, 2, 3).re = e8; U(2, 1, 2, 3).re = -e24;
    U(0, 1, 2, NKK - 3).re = e8; U(1, 1, 2, NKK - 3).re = -e8; U(2, 1, 2, NKK - 3).re = -e24;
    U(0, 1, NKJ - 2, 3).re = e8; U(1, 1, NKJ - 2, 3).re = e8; U(2, 1, NKJ - 2, 3).re = e24;
    U(0, 1, NKJ - 2, NKK - 3).re = -e8; U(1, 1, NKJ - 2, NKK - 3).re = -e8;
    U(2, 1, NKJ - 2, NKK - 3).re = e24;
#undef U
}

/* ------------------------------------------------------------------------- */
/* dt (f_RK3Tstep, src/pf_rk3.f90:3852-3948)                                    */
/* ------------------------------------------------------------------------- */
static double tstep_dt(const oracle* o, double ucfl) {
    const pandora_params* p = &o->p;
    double dt = p->rk3_dt;
    switch (p->rk3_timestep) {
    case PANDORA_RK3_TIMESTEP_FIXED: dt = p->rk3_dt; break;
    case PANDORA_RK3_TIMESTEP_CFL:
        dt = (ucfl == 0.0) ? 0.02 : p->rk3_cfl * o->dx / ucfl;
        break;
    case PANDORA_RK3_TIMESTEP_DECIDE:
        if (p->f_type == PANDORA_F_ISOTROPIC) {
            if (ucfl == 0.0) dt = 0.02;
            else { dt = p->rk3_cfl * o->dx / ucfl; if (dt > p->force_tf) dt = p->force_tf; }
        } else if (p->f_type == PANDORA_F_ISOTROPIC_DEFORMED) {
            double m = o->dx < o->dy ? o->dx : o->dy; m = m < o->dz ? m : o->dz;
            if (ucfl == 0.0) dt = 0.02;
            else { dt = p->rk3_cfl * m / ucfl; if (dt > p->force_tf) dt = p->force_tf; }
        } else {
            dt = ((0.5 / p->f_deform_s) / (double)p->f_remesh_t);
        }
        break;
    }
    return dt;
}

/* ------------------------------------------------------------------------- */
/* stages and step                                                              */
/* ------------------------------------------------------------------------- */
/* f_RK3Stage{1,2,3} (src/pf_rk3.f90:40-200); *dt in/out */
int oracle_stage(oracle* o, int stage, int tstep, double* dt) {
    if (o->p.f_type != PANDORA_F_ISOTROPIC && o->p.f_type != PANDORA_F_SHEAR_DNS) return PANDORA_ERR_UNSUPPORTED;
    if (o->p.rk3_viscous == PANDORA_VISCOUS_INTEGRATING_FACTOR && o->p.f_type != PANDORA_F_ISOTROPIC)
        return PANDORA_ERR_UNSUPPORTED;
    if (stage == 1 && o->shear && oracle_remesh_due(o, tstep)) {   /* src/pf_rk3.f90:3990-4025 */
        dealias(o);
        particles_remesh(o);
        remesh_wave_space(o);
        dealias(o);
    }
    compute_nonlinear(o, stage == 1);
    if (stage == 1) *dt = tstep_dt(o, o->ucfl);
    particles_stage(o, stage, tstep, *dt);
    if (o->rrot) {
        form_f_rrot(o, stage, *dt);
    } else if (o->shear) {
        form_f_bf(o, stage, *dt);
    } else {
        force_calc(o, tstep, stage, *dt);
        form_f_iso(o, stage, *dt);
    }
    return o->status ? PANDORA_ERR_NAN : 0;
}

/* g_RK3Calc (src/pg_rk3.f90:82-129) */
int oracle_step(oracle* o, int tstep, double* simtime, double* dt) {
    double t0 = *simtime;
    double sim_dt = 99999.0;
    int rc;
    if ((rc = oracle_stage(o, 1, tstep, &sim_dt))) return rc;
    *simtime = t0 + (1.0 / 3.0) * sim_dt;
    oracle_update_b(o, tstep, *simtime);
    if ((rc = oracle_stage(o, 2, tstep, &sim_dt))) return rc;
    *simtime = t0 + (3.0 / 4.0) * sim_dt;
    oracle_update_b(o, tstep, *simtime);
    if ((rc = oracle_stage(o, 3, tstep, &sim_dt))) return rc;
    *simtime = t0 + sim_dt;
    oracle_update_b(o, tstep, *simtime);
    *dt = sim_dt;
    return 0;
}

int oracle_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
