/*
 * CPU oracle for the BigDFT Daubechies-16 local-Hamiltonian path.
 *
 * TEST INFRASTRUCTURE ONLY: this file is the checker the parity tests and the
 * benchmark's CPU-baseline leg compare against.  Nothing in the product
 * library links or calls it.
 *
 * It restates, loop for loop and in FP64, the reference's CPU convolutions
 * (Fortran, not compilable in this environment: no Fortran compiler) and the
 * compositions its OpenCL accelerator backend performs.  Each routine cites
 * the reference file:line it follows (paths relative to the reference root).
 * The filter constants come from the generated header wvl_filters.h, which is
 * parsed from the reference sources.
 *
 * Conventions follow the Fortran sources:
 *   - n1,n2,n3 are the maximum coarse indices (n+1 coarse cells per dim);
 *   - keys are 1-based: keyg[2*iseg+0..1] = first/last linear coarse index,
 *     keyv[iseg] = first compressed position;
 *   - psig(0:n1,2,0:n2,2,0:n3,2) is the wavelet-basis box, i1 fastest;
 *   - "rot" 1D passes read x(0:L-1,ndat) and write y(ndat,0:L'-1).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../bigdft-suite_b200/csrc/wvl_filters.h"

#define IMOD(a, m) ((((a) % (m)) + (m)) % (m))

/* ------------------------------------------------------------------------ */
/* keys: num_segkeys / segkeys, bigdft/src/locregs/initlocregs.f90:1573,1633 */
/* ------------------------------------------------------------------------ */
void wo_num_segkeys(int n1, int n2, int n3, const uint8_t *logrid, int *mseg, int *mvctr)
{
    int nsrt = 0, nend = 0, nv = 0;
    for (int i3 = 0; i3 <= n3; ++i3)
        for (int i2 = 0; i2 <= n2; ++i2) {
            int p = 0;
            for (int i1 = 0; i1 <= n1; ++i1) {
                int on = logrid[(i3 * (n2 + 1) + i2) * (n1 + 1) + i1] != 0;
                if (on) {
                    nv++;
                    if (!p) nsrt++;
                } else if (p) {
                    nend++;
                }
                p = on;
            }
            if (p) nend++;
        }
    *mseg = nend;
    *mvctr = nv;
    (void)nsrt;
}

void wo_segkeys(int n1, int n2, int n3, const uint8_t *logrid, int32_t *keyg, int32_t *keyv)
{
    int mvctr = 0, nsrt = 0, nend = 0;
    int n1p1 = n1 + 1, np = n1p1 * (n2 + 1);
    for (int i3 = 0; i3 <= n3; ++i3)
        for (int i2 = 0; i2 <= n2; ++i2) {
            int p = 0, ngridp = 0;
            for (int i1 = 0; i1 <= n1; ++i1) {
                ngridp = i3 * np + i2 * n1p1 + i1 + 1;
                int on = logrid[(i3 * (n2 + 1) + i2) * (n1 + 1) + i1] != 0;
                if (on) {
                    mvctr++;
                    if (!p) {
                        keyg[2 * nsrt] = ngridp;
                        keyv[nsrt] = mvctr;
                        nsrt++;
                    }
                } else if (p) {
                    keyg[2 * nend + 1] = ngridp - 1;
                    nend++;
                }
                p = on;
            }
            if (p) {
                keyg[2 * nend + 1] = ngridp;
                nend++;
            }
        }
}

/* segment decode shared by every (un)compress loop, un-compress.f90:896-905 */
static inline void seg_decode(int n1, int n2, const int32_t *keyg, int iseg,
                              int *i0, int *i1e, int *i2, int *i3)
{
    int j0 = keyg[2 * iseg], j1 = keyg[2 * iseg + 1];
    int ii = j0 - 1;
    *i3 = ii / ((n1 + 1) * (n2 + 1));
    ii = ii - (*i3) * (n1 + 1) * (n2 + 1);
    *i2 = ii / (n1 + 1);
    *i0 = ii - (*i2) * (n1 + 1);
    *i1e = *i0 + j1 - j0;
}

/* psig(i1,s1,i2,s2,i3,s3), s in {0,1} */
static inline size_t gidx(int n1, int n2, int n3, int i1, int s1, int i2, int s2, int i3, int s3)
{
    size_t N1 = n1 + 1, N2 = n2 + 1, N3 = n3 + 1;
    return (size_t)i1 + N1 * (s1 + 2 * ((size_t)i2 + N2 * (s2 + 2 * ((size_t)i3 + N3 * s3))));
}

/* fine component c (1..7) -> (s1,s2,s3), un-compress.f90:930-936 */
static const int FS1[8] = {0, 1, 0, 1, 0, 1, 0, 1};
static const int FS2[8] = {0, 0, 1, 1, 0, 0, 1, 1};
static const int FS3[8] = {0, 0, 0, 0, 1, 1, 1, 1};

/* uncompress into psig (zeroed), optional per-component scaling;
 * un-compress.f90:877-940 (uncompress_per scatter) and 953-1010 (scal) */
void wo_uncompress(int n1, int n2, int n3,
                   int nseg_c, const int32_t *keyg_c, const int32_t *keyv_c,
                   int nseg_f, const int32_t *keyg_f, const int32_t *keyv_f,
                   const double *psi_c, const double *psi_f, const double *scal,
                   double *psig)
{
    size_t ntot = (size_t)8 * (n1 + 1) * (n2 + 1) * (n3 + 1);
    memset(psig, 0, ntot * sizeof(double));
    for (int iseg = 0; iseg < nseg_c; ++iseg) {
        int i0, i1e, i2, i3;
        seg_decode(n1, n2, keyg_c, iseg, &i0, &i1e, &i2, &i3);
        int jj = keyv_c[iseg];
        for (int i = i0; i <= i1e; ++i)
            psig[gidx(n1, n2, n3, i, 0, i2, 0, i3, 0)] = psi_c[i - i0 + jj - 1] * (scal ? scal[0] : 1.0);
    }
    for (int iseg = 0; iseg < nseg_f; ++iseg) {
        int i0, i1e, i2, i3;
        seg_decode(n1, n2, keyg_f, iseg, &i0, &i1e, &i2, &i3);
        int jj = keyv_f[iseg];
        for (int i = i0; i <= i1e; ++i)
            for (int c = 1; c <= 7; ++c)
                psig[gidx(n1, n2, n3, i, FS1[c], i2, FS2[c], i3, FS3[c])] =
                    psi_f[7 * (size_t)(i - i0 + jj - 1) + c - 1] * (scal ? scal[c] : 1.0);
    }
}

/* gather from psig; acc=1 accumulates (compress_and_accumulate_mixed,
 * un-compress.f90:2174-2238), acc=0 overwrites (OpenCL compress_d,
 * OpenCL/Uncompress.c:612); optional scaling (compress_sd_scal :1023) */
void wo_compress(int n1, int n2, int n3,
                 int nseg_c, const int32_t *keyg_c, const int32_t *keyv_c,
                 int nseg_f, const int32_t *keyg_f, const int32_t *keyv_f,
                 const double *psig, const double *scal, int acc,
                 double *psi_c, double *psi_f)
{
    for (int iseg = 0; iseg < nseg_c; ++iseg) {
        int i0, i1e, i2, i3;
        seg_decode(n1, n2, keyg_c, iseg, &i0, &i1e, &i2, &i3);
        int jj = keyv_c[iseg];
        for (int i = i0; i <= i1e; ++i) {
            double v = psig[gidx(n1, n2, n3, i, 0, i2, 0, i3, 0)] * (scal ? scal[0] : 1.0);
            double *o = &psi_c[i - i0 + jj - 1];
            *o = acc ? *o + v : v;
        }
    }
    for (int iseg = 0; iseg < nseg_f; ++iseg) {
        int i0, i1e, i2, i3;
        seg_decode(n1, n2, keyg_f, iseg, &i0, &i1e, &i2, &i3);
        int jj = keyv_f[iseg];
        for (int i = i0; i <= i1e; ++i)
            for (int c = 1; c <= 7; ++c) {
                double v = psig[gidx(n1, n2, n3, i, FS1[c], i2, FS2[c], i3, FS3[c])] * (scal ? scal[c] : 1.0);
                double *o = &psi_f[7 * (size_t)(i - i0 + jj - 1) + c - 1];
                *o = acc ? *o + v : v;
            }
    }
}

/* ------------------------------------------------------------------------ */
/* periodic 1D rotated passes, orbitals/convolut_simple_per.f90             */
/* ------------------------------------------------------------------------ */

/* ana_rot_per, convolut_simple_per.f90:11-57 */
void wo_ana_rot_per(int n, int ndat, const double *x, double *y)
{
    int L = 2 * n + 2;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ndat; ++j)
        for (int i = 0; i <= n; ++i) {
            double ci = 0.0, di = 0.0;
            for (int l = -7; l <= 8; ++l) {
                int k = IMOD(l + 2 * i, L);
                ci += WVL_CH[l + 7] * x[(size_t)j * L + k];
                di += WVL_CG[l + 7] * x[(size_t)j * L + k];
            }
            y[(size_t)i * ndat + j] = ci;
            y[(size_t)(n + 1 + i) * ndat + j] = di;
        }
}

/* ch(-8:9)/cg(-8:9) of syn_rot_per: the analysis taps shifted by one with a
 * zero at each end, convolut_simple_per.f90:70-87 */
static inline double syn_ch(int m) { return (m >= -7 && m <= 8) ? WVL_CH[m + 7] : 0.0; }
static inline double syn_cg(int m) { return (m >= -7 && m <= 8) ? WVL_CG[m + 7] : 0.0; }

/* syn_rot_per main loop, convolut_simple_per.f90:89-103 */
void wo_syn_rot_per(int n, int ndat, const double *x, double *y)
{
    int L = 2 * n + 2;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ndat; ++j)
        for (int i = 0; i <= n; ++i) {
            double se = 0.0, so = 0.0;
            for (int l = -4; l <= 4; ++l) {
                int k = IMOD(i - l, n + 1);
                se += syn_ch(2 * l) * x[(size_t)j * L + k] + syn_cg(2 * l) * x[(size_t)j * L + n + 1 + k];
                so += syn_ch(2 * l + 1) * x[(size_t)j * L + k] + syn_cg(2 * l + 1) * x[(size_t)j * L + n + 1 + k];
            }
            y[(size_t)(2 * i) * ndat + j] = se;
            y[(size_t)(2 * i + 1) * ndat + j] = so;
        }
}

/* convrot_n_per, convolut_simple_per.f90:200-243 */
void wo_convrot_n_per(int n1, int ndat, const double *x, double *y)
{
    int L = n1 + 1;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ndat; ++j)
        for (int i = 0; i <= n1; ++i) {
            double tt = 0.0;
            for (int l = -8; l <= 7; ++l) tt += x[(size_t)j * L + IMOD(i + l, L)] * WVL_MF[l + 8];
            y[(size_t)i * ndat + j] = tt;
        }
}

/* convrot_t_per, convolut_simple_per.f90:246-291 (fil(-7:8) is fil_n mirrored) */
void wo_convrot_t_per(int n1, int ndat, const double *x, double *y)
{
    int L = n1 + 1;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ndat; ++j)
        for (int i = 0; i <= n1; ++i) {
            double tt = 0.0;
            for (int l = -7; l <= 8; ++l) tt += x[(size_t)j * L + IMOD(i + l, L)] * WVL_MF[-l + 8];
            y[(size_t)i * ndat + j] = tt;
        }
}

/* convolut_kinetic_per_T, convolut_simple_per.f90:377-460: y += T x on the
 * (n1+1)(n2+1)(n3+1) fine grid, ekin = sum_d <x|T_d x>; hgrid = fine spacing */
void wo_kinetic_per_T(int n1, int n2, int n3, const double *hgrid, const double *x, double *y, double *ekin)
{
    double fil[3][29];
    for (int d = 0; d < 3; ++d) {
        double scale = -0.5 / (hgrid[d] * hgrid[d]);
        for (int l = 0; l <= 14; ++l) fil[d][14 + l] = fil[d][14 - l] = WVL_KIN[l] * scale;
    }
    size_t N1 = n1 + 1, N2 = n2 + 1, N3 = n3 + 1;
    double ek = 0.0;
#pragma omp parallel for reduction(+ : ek) schedule(static)
    for (int i3 = 0; i3 <= n3; ++i3) {
        for (int i2 = 0; i2 <= n2; ++i2)
            for (int i1 = 0; i1 <= n1; ++i1) {
                double tt = 0.0;
                for (int l = -14; l <= 14; ++l)
                    tt += x[(i3 * N2 + i2) * N1 + IMOD(i1 + l, (int)N1)] * fil[0][l + 14];
                y[(i3 * N2 + i2) * N1 + i1] += tt;
                ek += x[(i3 * N2 + i2) * N1 + i1] * tt;
            }
        for (int i1 = 0; i1 <= n1; ++i1)
            for (int i2 = 0; i2 <= n2; ++i2) {
                double tt = 0.0;
                for (int l = -14; l <= 14; ++l)
                    tt += x[(i3 * N2 + IMOD(i2 + l, (int)N2)) * N1 + i1] * fil[1][l + 14];
                y[(i3 * N2 + i2) * N1 + i1] += tt;
                ek += x[(i3 * N2 + i2) * N1 + i1] * tt;
            }
    }
    double ek3 = 0.0;
#pragma omp parallel for reduction(+ : ek3) schedule(static)
    for (int i2 = 0; i2 <= n2; ++i2)
        for (int i1 = 0; i1 <= n1; ++i1)
            for (int i3 = 0; i3 <= n3; ++i3) {
                double tt = 0.0;
                for (int l = -14; l <= 14; ++l)
                    tt += x[(IMOD(i3 + l, (int)N3) * N2 + i2) * N1 + i1] * fil[2][l + 14];
                y[(i3 * N2 + i2) * N1 + i1] += tt;
                ek3 += x[(i3 * N2 + i2) * N1 + i1] * tt;
            }
    *ekin = ek + ek3;
}

/* synthese_per_self / analyse_per_self / convolut_magic_n_per / _t_per_self,
 * orbitals/convolut_common_per.f90:38,87,112,166: three rotated passes */
void wo_synthese_per(int n1, int n2, int n3, const double *psig, double *psifscf, double *w)
{
    wo_syn_rot_per(n1, (2 * n2 + 2) * (2 * n3 + 2), psig, psifscf);
    wo_syn_rot_per(n2, (2 * n3 + 2) * (2 * n1 + 2), psifscf, w);
    wo_syn_rot_per(n3, (2 * n1 + 2) * (2 * n2 + 2), w, psifscf);
}
void wo_analyse_per(int n1, int n2, int n3, const double *y, double *psig, double *w)
{
    wo_ana_rot_per(n1, (2 * n2 + 2) * (2 * n3 + 2), y, psig);
    wo_ana_rot_per(n2, (2 * n3 + 2) * (2 * n1 + 2), psig, w);
    wo_ana_rot_per(n3, (2 * n1 + 2) * (2 * n2 + 2), w, psig);
}
/* magic filter on an (m1+1)(m2+1)(m3+1) grid */
void wo_magic_n_per(int m1, int m2, int m3, const double *x, double *y, double *w)
{
    wo_convrot_n_per(m1, (m2 + 1) * (m3 + 1), x, y);
    wo_convrot_n_per(m2, (m3 + 1) * (m1 + 1), y, w);
    wo_convrot_n_per(m3, (m1 + 1) * (m2 + 1), w, y);
}
void wo_magic_t_per(int m1, int m2, int m3, const double *x, double *y, double *w)
{
    wo_convrot_t_per(m1, (m2 + 1) * (m3 + 1), x, y);
    wo_convrot_t_per(m2, (m3 + 1) * (m1 + 1), y, w);
    wo_convrot_t_per(m3, (m1 + 1) * (m2 + 1), w, y);
}

/* apply_potential_lr_nobounds scalar branch, orbitals/potential.f90:1011-1031 */
double wo_apply_potential(size_t npts, const double *pot, double *psir)
{
    double epot = 0.0;
#pragma omp parallel for reduction(+ : epot) schedule(static)
    for (size_t i = 0; i < npts; ++i) {
        double tt = pot[i] * psir[i];
        epot += tt * psir[i];
        psir[i] = tt;
    }
    return epot;
}

/* Local Hamiltonian of one periodic orbital: daub_to_isf_locham case 'P'
 * (orbitals/daubisf.f90:303-311), psir_to_vpsi (locregs/locreg_operations.f90:2502),
 * isf_to_daub_kinetic case 'P' (:2836-2865).  hpsi is ACCUMULATED into, as
 * compress_and_accumulate_mixed does.  hgrid = coarse grid spacing. */
void wo_locham_per(int n1, int n2, int n3, const double *hgrid,
                   int nseg_c, const int32_t *keyg_c, const int32_t *keyv_c,
                   int nseg_f, const int32_t *keyg_f, const int32_t *keyv_f,
                   const double *psi_c, const double *psi_f, const double *pot,
                   double *hpsi_c, double *hpsi_f, double *ekin, double *epot)
{
    size_t nf = (size_t)8 * (n1 + 1) * (n2 + 1) * (n3 + 1);
    double *psig = malloc(nf * sizeof(double));
    double *xc = malloc(nf * sizeof(double));
    double *psir = malloc(nf * sizeof(double));
    double *yc = malloc(nf * sizeof(double));
    wo_uncompress(n1, n2, n3, nseg_c, keyg_c, keyv_c, nseg_f, keyg_f, keyv_f, psi_c, psi_f, NULL, psig);
    wo_synthese_per(n1, n2, n3, psig, xc, yc);                   /* x_c = psifscf */
    int m1 = 2 * n1 + 1, m2 = 2 * n2 + 1, m3 = 2 * n3 + 1;
    wo_magic_n_per(m1, m2, m3, xc, psir, yc);                    /* psir = MF^3 x_c */
    *epot = wo_apply_potential(nf, pot, psir);                   /* psir = V psir */
    wo_magic_t_per(m1, m2, m3, psir, yc, psig);                  /* y_c = MF^T^3 psir */
    double hh[3] = {0.5 * hgrid[0], 0.5 * hgrid[1], 0.5 * hgrid[2]};
    wo_kinetic_per_T(m1, m2, m3, hh, xc, yc, ekin);              /* y_c += T x_c */
    wo_analyse_per(n1, n2, n3, yc, psig, psir);
    wo_compress(n1, n2, n3, nseg_c, keyg_c, keyv_c, nseg_f, keyg_f, keyv_f, psig, NULL, 1, hpsi_c, hpsi_f);
    free(psig); free(xc); free(psir); free(yc);
}

/* local_partial_density + partial_density for one periodic orbital:
 * sumrho.f90:422-440 and 472-577: rho += hfac * psir^2 */
void wo_locden_per(int n1, int n2, int n3,
                   int nseg_c, const int32_t *keyg_c, const int32_t *keyv_c,
                   int nseg_f, const int32_t *keyg_f, const int32_t *keyv_f,
                   const double *psi_c, const double *psi_f, double hfac, double *rho)
{
    size_t nf = (size_t)8 * (n1 + 1) * (n2 + 1) * (n3 + 1);
    double *psig = malloc(nf * sizeof(double));
    double *xc = malloc(nf * sizeof(double));
    double *w = malloc(nf * sizeof(double));
    wo_uncompress(n1, n2, n3, nseg_c, keyg_c, keyv_c, nseg_f, keyg_f, keyv_f, psi_c, psi_f, NULL, psig);
    wo_synthese_per(n1, n2, n3, psig, xc, w);
    wo_magic_n_per(2 * n1 + 1, 2 * n2 + 1, 2 * n3 + 1, xc, psig, w);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < nf; ++i) rho[i] += hfac * psig[i] * psig[i];
    free(psig); free(xc); free(w);
}

/* ------------------------------------------------------------------------ */
/* free boundary conditions: the grown-box formulation of the OpenCL backend */
/* (syngrow1d / magicfiltergrow1d / magicfiltershrink1d / kinetic1d_f /      */
/* anashrink1d, OpenCL/Wavelet.c:238-330, MagicFilter.c, Kinetic.c:240-270), */
/* whose fine grid -7..2N+6 and ISF grid -14..2N+14 are those of the CPU     */
/* comb_grow_all / comb_shrink path (orbitals/growshrink.f90:12,310).        */
/* N = coarse cells, grown fine length 2N+14, ISF length 2N+29.              */
/* ------------------------------------------------------------------------ */

/* syn grow: x(0:2N-1,ndat) -> y(ndat, 0:2N+13), y index q = f+7 */
void wo_syn_grow_rot(int N, int ndat, const double *x, double *y)
{
    int L = 2 * N, Lo = 2 * N + 14;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ndat; ++j)
        for (int q = 0; q < Lo; ++q) {
            int f = q - 7;
            int i = (f >= 0) ? f / 2 : -((-f + 1) / 2); /* floor(f/2) */
            int odd = f - 2 * i;
            double s = 0.0;
            for (int l = -4; l <= 4; ++l) {
                int k = i - l;
                if (k < 0 || k >= N) continue;
                int m = 2 * l + odd;
                s += syn_ch(m) * x[(size_t)j * L + k] + syn_cg(m) * x[(size_t)j * L + N + k];
            }
            y[(size_t)q * ndat + j] = s;
        }
}

/* ana shrink: x(0:2N+13,ndat) -> y(ndat,0:2N-1) */
void wo_ana_shrink_rot(int N, int ndat, const double *x, double *y)
{
    int L = 2 * N + 14;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ndat; ++j)
        for (int i = 0; i < N; ++i) {
            double ci = 0.0, di = 0.0;
            for (int l = -7; l <= 8; ++l) {
                double v = x[(size_t)j * L + 2 * i + l + 7];
                ci += WVL_CH[l + 7] * v;
                di += WVL_CG[l + 7] * v;
            }
            y[(size_t)i * ndat + j] = ci;
            y[(size_t)(N + i) * ndat + j] = di;
        }
}

/* MF grow: x(0:Lf-1,ndat) (fine, q=f+7) -> y(ndat,0:Lf+14), r index = rr+14 */
void wo_mf_grow_rot(int Lf, int ndat, const double *x, double *y)
{
    int Lo = Lf + 15;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ndat; ++j)
        for (int r = 0; r < Lo; ++r) {
            int rr = r - 14;
            double tt = 0.0;
            for (int l = -8; l <= 7; ++l) {
                int q = rr + l + 7;
                if (q >= 0 && q < Lf) tt += x[(size_t)j * Lf + q] * WVL_MF[l + 8];
            }
            y[(size_t)r * ndat + j] = tt;
        }
}

/* MF^T shrink: x(0:Lf+14,ndat) -> y(ndat,0:Lf-1) */
void wo_mf_shrink_rot(int Lf, int ndat, const double *x, double *y)
{
    int Li = Lf + 15;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ndat; ++j)
        for (int q = 0; q < Lf; ++q) {
            int f = q - 7;
            double tt = 0.0;
            for (int l = -7; l <= 8; ++l) tt += x[(size_t)j * Li + (f + l + 14)] * WVL_MF[-l + 8];
            y[(size_t)q * ndat + j] = tt;
        }
}

/* kinetic on an L1 x L2 x L3 fine grid, zero outside (free) or periodic per
 * dimension; y += T x, ekin = <x|T x>.  hgrid = fine spacing. */
void wo_kinetic_generic(int L1, int L2, int L3, const int *periodic, const double *hgrid,
                        const double *x, double *y, double *ekin)
{
    double fil[3][29];
    int L[3] = {L1, L2, L3};
    for (int d = 0; d < 3; ++d) {
        double scale = -0.5 / (hgrid[d] * hgrid[d]);
        for (int l = 0; l <= 14; ++l) fil[d][14 + l] = fil[d][14 - l] = WVL_KIN[l] * scale;
    }
    double ek = 0.0;
#pragma omp parallel for reduction(+ : ek) schedule(static)
    for (int i3 = 0; i3 < L3; ++i3)
        for (int i2 = 0; i2 < L2; ++i2)
            for (int i1 = 0; i1 < L1; ++i1) {
                int c[3] = {i1, i2, i3};
                size_t p = ((size_t)i3 * L2 + i2) * L1 + i1;
                double tot = 0.0;
                for (int d = 0; d < 3; ++d) {
                    double tt = 0.0;
                    for (int l = -14; l <= 14; ++l) {
                        int cc[3] = {c[0], c[1], c[2]};
                        int v = c[d] + l;
                        if (periodic[d]) v = IMOD(v, L[d]);
                        else if (v < 0 || v >= L[d]) continue;
                        cc[d] = v;
                        tt += x[((size_t)cc[2] * L2 + cc[1]) * L1 + cc[0]] * fil[d][l + 14];
                    }
                    tot += tt;
                    ek += x[p] * tt;
                }
                y[p] += tot;
            }
    *ekin = ek;
}

/* generic 3D helpers for mixed periodic/free: apply a 1D rotated pass along
 * each dimension in x->y->z order (the layout returns to natural after 3). */
typedef void (*pass_fn)(int, int, const double *, double *);

/* Synthesis: psig (2N1,2N2,2N3) -> fine (F1,F2,F3), F = 2N (per) or 2N+14 (free) */
void wo_synthese_generic(const int *N, const int *per, const double *psig, double *out, double *w)
{
    int F[3];
    for (int d = 0; d < 3; ++d) F[d] = per[d] ? 2 * N[d] : 2 * N[d] + 14;
    /* x: in (2N1, 2N2*2N3) -> (2N2*2N3, F1) */
    if (per[0]) wo_syn_rot_per(N[0] - 1, 4 * N[1] * N[2], psig, w); else wo_syn_grow_rot(N[0], 4 * N[1] * N[2], psig, w);
    if (per[1]) wo_syn_rot_per(N[1] - 1, 2 * N[2] * F[0], w, out); else wo_syn_grow_rot(N[1], 2 * N[2] * F[0], w, out);
    if (per[2]) wo_syn_rot_per(N[2] - 1, F[0] * F[1], out, w); else wo_syn_grow_rot(N[2], F[0] * F[1], out, w);
    memcpy(out, w, (size_t)F[0] * F[1] * F[2] * sizeof(double));
}

void wo_analyse_generic(const int *N, const int *per, const double *in, double *psig, double *w)
{
    int F[3];
    for (int d = 0; d < 3; ++d) F[d] = per[d] ? 2 * N[d] : 2 * N[d] + 14;
    if (per[0]) wo_ana_rot_per(N[0] - 1, F[1] * F[2], in, w); else wo_ana_shrink_rot(N[0], F[1] * F[2], in, w);
    if (per[1]) wo_ana_rot_per(N[1] - 1, F[2] * 2 * N[0], w, psig); else wo_ana_shrink_rot(N[1], F[2] * 2 * N[0], w, psig);
    if (per[2]) wo_ana_rot_per(N[2] - 1, 4 * N[0] * N[1], psig, w); else wo_ana_shrink_rot(N[2], 4 * N[0] * N[1], psig, w);
    memcpy(psig, w, (size_t)8 * N[0] * N[1] * N[2] * sizeof(double));
}

/* magic filter fine (F) -> ISF (I = F per, F+15 free) */
void wo_magic_generic(const int *F, const int *per, const double *in, double *out, double *w)
{
    int I[3];
    for (int d = 0; d < 3; ++d) I[d] = per[d] ? F[d] : F[d] + 15;
    if (per[0]) wo_convrot_n_per(F[0] - 1, F[1] * F[2], in, w); else wo_mf_grow_rot(F[0], F[1] * F[2], in, w);
    if (per[1]) wo_convrot_n_per(F[1] - 1, F[2] * I[0], w, out); else wo_mf_grow_rot(F[1], F[2] * I[0], w, out);
    if (per[2]) wo_convrot_n_per(F[2] - 1, I[0] * I[1], out, w); else wo_mf_grow_rot(F[2], I[0] * I[1], out, w);
    memcpy(out, w, (size_t)I[0] * I[1] * I[2] * sizeof(double));
}

void wo_magic_t_generic(const int *F, const int *per, const double *in, double *out, double *w)
{
    int I[3];
    for (int d = 0; d < 3; ++d) I[d] = per[d] ? F[d] : F[d] + 15;
    if (per[0]) wo_convrot_t_per(F[0] - 1, I[1] * I[2], in, w); else wo_mf_shrink_rot(F[0], I[1] * I[2], in, w);
    if (per[1]) wo_convrot_t_per(F[1] - 1, I[2] * F[0], w, out); else wo_mf_shrink_rot(F[1], I[2] * F[0], w, out);
    if (per[2]) wo_convrot_t_per(F[2] - 1, F[0] * F[1], out, w); else wo_mf_shrink_rot(F[2], F[0] * F[1], out, w);
    memcpy(out, w, (size_t)F[0] * F[1] * F[2] * sizeof(double));
}

/* Generic (per-dimension periodic or free) local Hamiltonian for one orbital,
 * the composition of ocl_fulllocham_generic (OpenCL/Hamiltonian.c:41-72):
 * uncompress -> syn -> MF -> xV (epot) -> MF^T -> + T x (ekin) -> ana ->
 * compress.  hpsi is OVERWRITTEN (compress_d semantics).  hgrid = coarse. */
void wo_locham_generic(const int *N, const int *per, const double *hgrid,
                       int nseg_c, const int32_t *keyg_c, const int32_t *keyv_c,
                       int nseg_f, const int32_t *keyg_f, const int32_t *keyv_f,
                       const double *psi_c, const double *psi_f, const double *pot,
                       double *hpsi_c, double *hpsi_f, double *ekin, double *epot)
{
    int F[3], I[3];
    for (int d = 0; d < 3; ++d) {
        F[d] = per[d] ? 2 * N[d] : 2 * N[d] + 14;
        I[d] = per[d] ? F[d] : F[d] + 15;
    }
    size_t ni = (size_t)I[0] * I[1] * I[2];
    size_t nf = (size_t)F[0] * F[1] * F[2];
    double *psig = malloc(ni * sizeof(double));
    double *x = malloc(ni * sizeof(double));
    double *r = malloc(ni * sizeof(double));
    double *y = malloc(ni * sizeof(double));
    double *w = malloc(ni * sizeof(double));
    wo_uncompress(N[0] - 1, N[1] - 1, N[2] - 1, nseg_c, keyg_c, keyv_c, nseg_f, keyg_f, keyv_f,
                  psi_c, psi_f, NULL, psig);
    wo_synthese_generic(N, per, psig, x, w);
    wo_magic_generic(F, per, x, r, w);
    *epot = wo_apply_potential(ni, pot, r);
    wo_magic_t_generic(F, per, r, y, w);
    double hh[3] = {0.5 * hgrid[0], 0.5 * hgrid[1], 0.5 * hgrid[2]};
    wo_kinetic_generic(F[0], F[1], F[2], per, hh, x, y, ekin);
    wo_analyse_generic(N, per, y, psig, w);
    wo_compress(N[0] - 1, N[1] - 1, N[2] - 1, nseg_c, keyg_c, keyv_c, nseg_f, keyg_f, keyv_f,
                psig, NULL, 0, hpsi_c, hpsi_f);
    (void)nf;
    free(psig); free(x); free(r); free(y); free(w);
}

/* Density of one orbital on the ISF grid, ocl_locden_generic
 * (OpenCL/Density.c:37-54; CPU: sumrho.f90:472-577, partial_density_free :579) */
void wo_locden_generic(const int *N, const int *per,
                       int nseg_c, const int32_t *keyg_c, const int32_t *keyv_c,
                       int nseg_f, const int32_t *keyg_f, const int32_t *keyv_f,
                       const double *psi_c, const double *psi_f, double hfac, double *rho)
{
    int F[3], I[3];
    for (int d = 0; d < 3; ++d) {
        F[d] = per[d] ? 2 * N[d] : 2 * N[d] + 14;
        I[d] = per[d] ? F[d] : F[d] + 15;
    }
    size_t ni = (size_t)I[0] * I[1] * I[2];
    double *psig = malloc(ni * sizeof(double));
    double *x = malloc(ni * sizeof(double));
    double *w = malloc(ni * sizeof(double));
    wo_uncompress(N[0] - 1, N[1] - 1, N[2] - 1, nseg_c, keyg_c, keyv_c, nseg_f, keyg_f, keyv_f,
                  psi_c, psi_f, NULL, psig);
    wo_synthese_generic(N, per, psig, x, w);
    wo_magic_generic(F, per, x, psig, w);
    for (size_t i = 0; i < ni; ++i) rho[i] += hfac * psig[i] * psig[i];
    free(psig); free(x); free(w);
}

/* Wavelet-basis kinetic for a full coarse box, the ConvolkineticT filter set
 * (orbitals/convolut_ib_optim.f90:921-1064) without the bound arrays:
 * y(i,s) += sum over directions of the 2x2 block filters a,b,c,e scaled by
 * -1/(2 h_d^2) (h = coarse spacing), periodic or zero boundaries. */
void wo_kinetic_wavelet(const int *N, const int *per, const double *hgrid, const double *psig,
                        double *y, double *ekin)
{
    double A[29], B[29], C[29], E[29];
    for (int l = 0; l <= 14; ++l) {
        A[14 + l] = A[14 - l] = WVL_KIN[l];
        E[14 + l] = E[14 - l] = WVL_KIN_E[l];
    }
    for (int l = -14; l <= 14; ++l) {
        C[l + 14] = WVL_KIN_C[l + 14];
        B[l + 14] = WVL_KIN_C[-l + 14];
    }
    double ek = 0.0;
    int n1 = N[0] - 1, n2 = N[1] - 1, n3 = N[2] - 1;
    for (int i3 = 0; i3 < N[2]; ++i3)
        for (int s3 = 0; s3 < 2; ++s3)
            for (int i2 = 0; i2 < N[1]; ++i2)
                for (int s2 = 0; s2 < 2; ++s2)
                    for (int i1 = 0; i1 < N[0]; ++i1)
                        for (int s1 = 0; s1 < 2; ++s1) {
                            int ii[3] = {i1, i2, i3}, ss[3] = {s1, s2, s3};
                            double tot = 0.0;
                            for (int d = 0; d < 3; ++d) {
                                double sc = -0.5 / (hgrid[d] * hgrid[d]);
                                for (int l = -14; l <= 14; ++l) {
                                    int v = ii[d] + l;
                                    if (per[d]) v = IMOD(v, N[d]);
                                    else if (v < 0 || v >= N[d]) continue;
                                    for (int t = 0; t < 2; ++t) {
                                        /* offset l = input - output; a (out s=0, in t=0),
                                         * b (s=0 <- t=1, x_f1), c (s=1 <- t=0), e (s=1 <- t=1),
                                         * ConvolkineticT, convolut_ib_optim.f90:1183-1290 */
                                        double f = (ss[d] == 0) ? (t == 0 ? A[l + 14] : B[l + 14])
                                                                : (t == 0 ? C[l + 14] : E[l + 14]);
                                        int jj[3] = {ii[0], ii[1], ii[2]}, tt[3] = {ss[0], ss[1], ss[2]};
                                        jj[d] = v;
                                        tt[d] = t;
                                        tot += sc * f * psig[gidx(n1, n2, n3, jj[0], tt[0], jj[1], tt[1], jj[2], tt[2])];
                                    }
                                }
                            }
                            size_t p = gidx(n1, n2, n3, i1, s1, i2, s2, i3, s3);
                            y[p] += tot;
                            ek += psig[p] * tot;
                        }
    *ekin = ek;
}

/* ------------------------------------------------------------------------ */
/* preconditioner: ocl_preconditioner_generic (OpenCL/Preconditioner.c:130-195)
 * with apply_hp_generic (:98-128): A = D^{-1/2} ana (c + T) syn D^{-1/2},
 * D^{-1/2} from GPUscal0..7 (OpenCL/Uncompress.c:380-470, h = hgrid/2).   */
/* ------------------------------------------------------------------------ */
void wo_precond_scal(const double *h, double c, double *scal)
{
    double hh[3];
    for (int d = 0; d < 3; ++d) hh[d] = 0.125 / (h[d] * h[d]);
    for (int k = 0; k < 8; ++k) {
        double s = c;
        s += ((k & 1) ? WVL_B2 : WVL_A2) * hh[0];
        s += ((k & 2) ? WVL_B2 : WVL_A2) * hh[1];
        s += ((k & 4) ? WVL_B2 : WVL_A2) * hh[2];
        scal[k] = 1.0 / sqrt(s);
    }
}

typedef struct {
    const int *N, *per;
    const double *h; /* fine spacing = hgrid/2, as the OpenCL host passes */
    double c;
    int nseg_c, nseg_f;
    const int32_t *keyg_c, *keyv_c, *keyg_f, *keyv_f;
} wo_prec_ctx;

static void apply_hp(const wo_prec_ctx *p, const double *scal, const double *xc, const double *xf,
                     double *oc, double *of)
{
    int F[3];
    for (int d = 0; d < 3; ++d) F[d] = p->per[d] ? 2 * p->N[d] : 2 * p->N[d] + 14;
    size_t nf = (size_t)F[0] * F[1] * F[2];
    double *psig = malloc(nf * sizeof(double));
    double *x = malloc(nf * sizeof(double));
    double *y = malloc(nf * sizeof(double));
    double *w = malloc(nf * sizeof(double));
    wo_uncompress(p->N[0] - 1, p->N[1] - 1, p->N[2] - 1, p->nseg_c, p->keyg_c, p->keyv_c,
                  p->nseg_f, p->keyg_f, p->keyv_f, xc, xf, scal, psig);
    wo_synthese_generic(p->N, p->per, psig, x, w);
    for (size_t i = 0; i < nf; ++i) y[i] = p->c * x[i];
    double ek;
    wo_kinetic_generic(F[0], F[1], F[2], p->per, p->h, x, y, &ek);
    wo_analyse_generic(p->N, p->per, y, psig, w);
    wo_compress(p->N[0] - 1, p->N[1] - 1, p->N[2] - 1, p->nseg_c, p->keyg_c, p->keyv_c,
                p->nseg_f, p->keyg_f, p->keyv_f, psig, scal, 0, oc, of);
    free(psig); free(x); free(y); free(w);
}

static double dotv(size_t n, const double *a, const double *b)
{
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* x (in: initial guess, out: preconditioned), b right-hand side (overwritten
 * as in the OpenCL routine), rnorm[0..ncong] residual norms squared seen by
 * the CG (rnorm[0] initial, rnorm[i] after iteration i, the last one computed
 * on the final residual for reporting). */
void wo_precond_generic(const int *N, const int *per, const double *h, double c, int ncong,
                        int nseg_c, int nvctr_c, const int32_t *keyg_c, const int32_t *keyv_c,
                        int nseg_f, int nvctr_f, const int32_t *keyg_f, const int32_t *keyv_f,
                        double *x, double *b, double *rnorm)
{
    wo_prec_ctx p = {N, per, h, c, nseg_c, nseg_f, keyg_c, keyv_c, keyg_f, keyv_f};
    double scal[8];
    wo_precond_scal(h, c, scal);
    size_t n = (size_t)nvctr_c + 7 * (size_t)nvctr_f;
    double *r = malloc(n * sizeof(double));
    double *d = malloc(n * sizeof(double));
    /* x, b are laid out [psi_c | psi_f] */
    apply_hp(&p, scal, x, x + nvctr_c, d, d + nvctr_c);
    for (size_t i = 0; i < n; ++i) r[i] = -d[i] + b[i];
    memcpy(d, r, n * sizeof(double));
    double norm_sq = dotv(n, r, r);
    if (rnorm) rnorm[0] = norm_sq;
    for (int it = 0; it < ncong; ++it) {
        apply_hp(&p, scal, d, d + nvctr_c, b, b + nvctr_c);
        double alpha = norm_sq / dotv(n, d, b);
        for (size_t i = 0; i < n; ++i) x[i] += alpha * d[i];
        if (it != ncong - 1) {
            for (size_t i = 0; i < n; ++i) r[i] -= alpha * b[i];
            double ns = dotv(n, r, r);
            double beta = ns / norm_sq;
            for (size_t i = 0; i < n; ++i) d[i] = beta * d[i] + r[i];
            norm_sq = ns;
            if (rnorm) rnorm[it + 1] = norm_sq;
        } else if (rnorm) {
            for (size_t i = 0; i < n; ++i) r[i] -= alpha * b[i];
            rnorm[it + 1] = dotv(n, r, r);
        }
    }
    /* scale_psi_d: x *= D^{-1/2} */
    for (size_t i = 0; i < (size_t)nvctr_c; ++i) x[i] *= scal[0];
    for (size_t i = 0; i < (size_t)nvctr_f; ++i)
        for (int k = 1; k <= 7; ++k) x[nvctr_c + 7 * i + k - 1] *= scal[k];
    free(r); free(d);
}

/* ------------------------------------------------------------------------ */
/* overlap S = Psi^T Psi (lower triangle, syrk('L','T'), wfn_opt/orthogonality.f90:2675),
 * Cholesky (dpotrf, :2351) and Loewdin S^{-1/2} (dsyev, :2486).             */
/* ------------------------------------------------------------------------ */
void wo_overlap(int nvctr, int norb, const double *psi, double *S)
{
    /* psi(nvctr, norb) column-major; S(norb,norb) column-major, full symmetric */
#pragma omp parallel for schedule(dynamic)
    for (int j = 0; j < norb; ++j)
        for (int i = j; i < norb; ++i) {
            double s = 0.0;
            const double *a = psi + (size_t)i * nvctr, *b = psi + (size_t)j * nvctr;
            for (int k = 0; k < nvctr; ++k) s += a[k] * b[k];
            S[(size_t)j * norb + i] = s;
            S[(size_t)i * norb + j] = s;
        }
}

/* lower Cholesky in place (column-major), returns 0 on success */
int wo_cholesky(int n, double *S)
{
    for (int j = 0; j < n; ++j) {
        double d = S[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) d -= S[(size_t)k * n + j] * S[(size_t)k * n + j];
        if (d <= 0.0) return j + 1;
        d = sqrt(d);
        S[(size_t)j * n + j] = d;
        for (int i = j + 1; i < n; ++i) {
            double s = S[(size_t)j * n + i];
            for (int k = 0; k < j; ++k) s -= S[(size_t)k * n + i] * S[(size_t)k * n + j];
            S[(size_t)j * n + i] = s / d;
        }
        for (int i = 0; i < j; ++i) S[(size_t)j * n + i] = 0.0;
    }
    return 0;
}

/* ------------------------------------------------------------------ wpdot
 * Scalar product of two compressed vectors a and b with different keys of the
 * same box (wpdot, wavelib/scalprod.f90:3222-3420), as the reference runs it
 * with one OpenMP thread.  For each b segment [kbs, kbe] (in order):
 *   jb0 = max(kbs, first a start); the a segment s holding jb0 is found by
 *   hunt_inline (:3427-3501: the last s with start(s) <= jb0);
 *   if s reaches jb0 the overlap [jb0, min(kbe, end(s))] is summed, else the
 *   next a segment, if it starts before kbe, contributes its overlap (:3300-3322);
 *   only one a segment counts per b segment (the loop exits at the first
 *   overlap, :3313);
 *   once a b segment starting after the last a start has been handled with s
 *   the last a segment, the search index runs past the end and every later b
 *   segment is skipped (:3323 with hunt_inline's "jlo > n" return, :3439).
 * Coarse products go to one FP64 sum and each of the 7 fine components to its
 * own, added at the end (:3404).  Keys are 1-based, keyv the 1-based offset. */
static int wp_hunt(const int32_t *keyg, int n, int x, int jlo)
{
    /* hunt_inline: the last 1-based s with start(s) <= x, 0 when x is below
     * start(1), the input unchanged when it is past the end (disabled) */
    if (jlo > n) return jlo;
    if (x < keyg[0]) return 0;
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (keyg[2 * mid] <= x) lo = mid; else hi = mid - 1;
    }
    return lo + 1;
}

static void wp_part(int nseg_a, const int32_t *keyg_a, const int32_t *keyv_a, const double *pa,
                    int nseg_b, const int32_t *keyg_b, const int32_t *keyv_b, const double *pb,
                    int ncomp, double *sums)
{
    int iaseg0 = 1;
    if (nseg_a <= 0) return;
    const int first_a = keyg_a[0], last_a = keyg_a[2 * (nseg_a - 1)];
    for (int ib = 0; ib < nseg_b; ++ib) {
        const int kbs = keyg_b[2 * ib], jb1 = keyg_b[2 * ib + 1];
        int jbj = keyv_b[ib];
        int jb0 = kbs > first_a ? kbs : first_a;
        const int iboff = jb0 - kbs > 0 ? jb0 - kbs : 0;
        iaseg0 = wp_hunt(keyg_a, nseg_a, jb0, iaseg0);
        if (iaseg0 == 0) { iaseg0 = 1; continue; }
        while (iaseg0 <= nseg_a) {
            const int ja0 = keyg_a[2 * (iaseg0 - 1)];
            const int ea = keyg_a[2 * (iaseg0 - 1) + 1];
            const int ja1 = jb1 < ea ? jb1 : ea;
            const int length = ja1 - jb0;
            const int iaoff = jb0 - ja0 > 0 ? jb0 - ja0 : 0;
            const int jaj = keyv_a[iaseg0 - 1];
            for (int i = 0; i <= length; ++i)
                for (int k = 0; k < ncomp; ++k)
                    sums[k] += pa[(size_t)(jaj + iaoff + i - 1) * ncomp + k] *
                               pb[(size_t)(jbj + i + iboff - 1) * ncomp + k];
            if ((ja1 <= jb1 && length >= 0) || iaseg0 == nseg_a) break;
            iaseg0 += 1;
            const int sa = keyg_a[2 * (iaseg0 - 1)];
            jb0 = kbs > sa ? kbs : sa;
            if (sa > jb1) break;
            jbj += jb0 - kbs > 0 ? jb0 - kbs : 0;
        }
        if (iaseg0 == nseg_a && kbs > last_a) iaseg0 += 1;
    }
}

/* Update through the same pairing of segments: a[jaj..] += s * b[jbj..] on
 * every common run (waxpy_mask_unpack, locregs/scalar_product.f90:953-1008,
 * over the masks of fill_wblas_segs, :1095-1187, which walk the loop above). */
static void wp_axpy_part(int nseg_a, const int32_t *keyg_a, const int32_t *keyv_a, double *pa,
                         int nseg_b, const int32_t *keyg_b, const int32_t *keyv_b, const double *pb,
                         int ncomp, double scal)
{
    int iaseg0 = 1;
    if (nseg_a <= 0) return;
    const int first_a = keyg_a[0], last_a = keyg_a[2 * (nseg_a - 1)];
    for (int ib = 0; ib < nseg_b; ++ib) {
        const int kbs = keyg_b[2 * ib], jb1 = keyg_b[2 * ib + 1];
        int jbj = keyv_b[ib];
        int jb0 = kbs > first_a ? kbs : first_a;
        const int iboff = jb0 - kbs > 0 ? jb0 - kbs : 0;
        iaseg0 = wp_hunt(keyg_a, nseg_a, jb0, iaseg0);
        if (iaseg0 == 0) { iaseg0 = 1; continue; }
        while (iaseg0 <= nseg_a) {
            const int ja0 = keyg_a[2 * (iaseg0 - 1)];
            const int ea = keyg_a[2 * (iaseg0 - 1) + 1];
            const int ja1 = jb1 < ea ? jb1 : ea;
            const int length = ja1 - jb0;
            const int iaoff = jb0 - ja0 > 0 ? jb0 - ja0 : 0;
            const int jaj = keyv_a[iaseg0 - 1];
            for (int i = 0; i <= length; ++i)
                for (int k = 0; k < ncomp; ++k)
                    pa[(size_t)(jaj + iaoff + i - 1) * ncomp + k] += scal * pb[(size_t)(jbj + i + iboff - 1) * ncomp + k];
            if ((ja1 <= jb1 && length >= 0) || iaseg0 == nseg_a) break;
            iaseg0 += 1;
            const int sa = keyg_a[2 * (iaseg0 - 1)];
            jb0 = kbs > sa ? kbs : sa;
            if (sa > jb1) break;
            jbj += jb0 - kbs > 0 ? jb0 - kbs : 0;
        }
        if (iaseg0 == nseg_a && kbs > last_a) iaseg0 += 1;
    }
}

/* a += s * b on the common points of a's keys and b's keys (coarse, then the
 * 7 fine components): the projector update of cproj_pr_p_psi
 * (locregs/compression.f90:562-589) for one projector vector b. */
void wo_mask_axpy(int nseg_ac, const int32_t *keyg_ac, const int32_t *keyv_ac, int nseg_af, const int32_t *keyg_af,
                  const int32_t *keyv_af, double *a_c, double *a_f,
                  int nseg_bc, const int32_t *keyg_bc, const int32_t *keyv_bc, int nseg_bf, const int32_t *keyg_bf,
                  const int32_t *keyv_bf, const double *b_c, const double *b_f, double s)
{
    wp_axpy_part(nseg_ac, keyg_ac, keyv_ac, a_c, nseg_bc, keyg_bc, keyv_bc, b_c, 1, s);
    wp_axpy_part(nseg_af, keyg_af, keyv_af, a_f, nseg_bf, keyg_bf, keyv_bf, b_f, 7, s);
}

double wo_wpdot(int nseg_ac, const int32_t *keyg_ac, const int32_t *keyv_ac, int nseg_af, const int32_t *keyg_af,
                const int32_t *keyv_af, const double *a_c, const double *a_f,
                int nseg_bc, const int32_t *keyg_bc, const int32_t *keyv_bc, int nseg_bf, const int32_t *keyg_bf,
                const int32_t *keyv_bf, const double *b_c, const double *b_f)
{
    double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    wp_part(nseg_ac, keyg_ac, keyv_ac, a_c, nseg_bc, keyg_bc, keyv_bc, b_c, 1, s);
    wp_part(nseg_af, keyg_af, keyv_af, a_f, nseg_bf, keyg_bf, keyv_bf, b_f, 7, s + 1);
    return s[0] + s[1] + s[2] + s[3] + s[4] + s[5] + s[6] + s[7];
}
