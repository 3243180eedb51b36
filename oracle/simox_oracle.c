/*
 * simox_oracle.c -- FP64 CPU restatement of SIMOX's per-step force and charge
 * path.  TEST INFRASTRUCTURE ONLY: the GPU library never links or calls this;
 * tests/, the smoke check and the bench's CPU-baseline leg use it as the
 * checker.
 *
 * Parity status: the reference is Fortran 90 and no Fortran compiler exists
 * in this image (nor on the GPU hosts, which run the same image), and the
 * reference ships no tests, inputs or golden outputs.  Parity against the
 * reference's own outputs is therefore UNPINNED.  This restatement follows the
 * Fortran statement by statement (file:line cited per routine) and is pinned
 * instead to independent known answers in tests/: the NaCl and CsCl Madelung
 * constants through FORCE(Edir)+PME(Erec)+PME_SELF, the FFT against a naive
 * DFT, finite-difference forces, and the published Al fit (a = 4.05 A).
 *
 * Reference semantics reproduced on purpose:
 *  - INT() truncates toward zero, MOD() takes the sign of the dividend,
 *    DNINT() rounds half away from zero (C round()), DINT() is trunc().
 *  - force.f90:406 and ctip.f90:359 build the spread value with
 *    CMPLX(x, 0.0D0), which has default (single) kind: the B-spline weight
 *    product is rounded to FP32 before it is spread.  The gather uses the
 *    FP64 weights.  (Controlled by or_set_spread_round.)
 *  - same-species CTIP terms use the as-written formulas, whose energy and
 *    force are not consistent (force.f90:101-118, ctip.f90:87-93).
 *  - PME_SELF's Esum uses 2w for the charge-bound penalty, CTIP_SOLVER's w.
 *  - psi(1,1,1) (k = 0) is never assigned by PME_SELF: set to 0 here.
 * Deliberate deviations: the neighbour-overflow check tests the atom's list
 * length (the reference tests the loop counters, force.f90:78); errors are
 * returned as status codes instead of STOP.
 *
 * Build with -O2 -ffp-contract=off (no FMA contraction, IEEE division) so
 * that the binning arithmetic is the IEEE FP64 arithmetic of the Fortran.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include "simox_gpu.h"

#define KC     14.399644154020082    /* datafmt.f90:23 */
#define TFM    10.180505306645389    /* datafmt.f90:24 */
#define PI_    3.1415926535897931    /* datafmt.f90:25 */
#define SQRTPI 1.7724538509055159    /* datafmt.f90:26 */
#define KB     8.617343e-5           /* datafmt.f90:27 */
#define WPEN   20.0                  /* datafmt.f90:28 */

typedef struct { double re, im; } cplx;

static int g_spread_round = 1;   /* reproduce CMPLX default-kind rounding */
void or_set_spread_round(int on) { g_spread_round = on; }
static double spread_value(double w) { return g_spread_round ? (double)(float)w : w; }

/* ====================================================================== */
/* POTENTIAL_SETUP  datafmt.f90:142-262                                   */
/* ====================================================================== */
void or_potential_setup(simox_potential* P)
{
    memset(P, 0, sizeof(*P));
    simox_metl* e = P->eam;
    e[0].r_e = 2.86392;  e[1].r_e = 2.48875;  e[2].r_e = 2.48199;
    e[0].f_e = 1.20378;  e[1].f_e = 2.21149;  e[2].f_e = 2.31453;
    e[0].rho_e = 17.51747; e[1].rho_e = 30.37003; e[2].rho_e = 24.59573;
    e[0].rho_s = 19.90041; e[1].rho_s = 30.37137; e[2].rho_s = 24.59573;
    e[0].alpha = 6.61317; e[1].alpha = 8.38345; e[2].alpha = 9.81827;
    e[0].beta  = 3.52702; e[1].beta  = 4.47117; e[2].beta  = 5.23641;
    e[0].A = 0.31487; e[1].A = 0.42905; e[2].A = 0.39281;
    e[0].B = 0.36555; e[1].B = 0.63353; e[2].B = 0.64624;
    e[0].kappa = 0.37985; e[1].kappa = 0.44360; e[2].kappa = 0.17031;
    e[0].lambda = 0.75969; e[1].lambda = 0.82066; e[2].lambda = 0.34061;
    e[0].Fn[0] = -2.80760; e[1].Fn[0] = -2.69351; e[2].Fn[0] = -2.53499;
    e[0].Fn[1] = -0.30144; e[1].Fn[1] = -0.07644; e[2].Fn[1] = -0.05960;
    e[0].Fn[2] =  1.25856; e[1].Fn[2] =  0.24144; e[2].Fn[2] =  0.19306;
    e[0].Fn[3] = -1.24760; e[1].Fn[3] = -2.37563; e[2].Fn[3] = -2.28232;
    e[0].Fm[0] = -2.83000; e[1].Fm[0] = -2.70000; e[2].Fm[0] = -2.54000;
    e[0].Fm[1] =  0.0;     e[1].Fm[1] =  0.0;     e[2].Fm[1] =  0.0;
    e[0].Fm[2] =  0.62225; e[1].Fm[2] =  0.26539; e[2].Fm[2] =  0.20027;
    e[0].Fm[3] = -2.48824; e[1].Fm[3] = -0.15286; e[2].Fm[3] = -0.14877;
    e[0].Fp[0] = -2.83000; e[1].Fp[0] = -2.70000; e[2].Fp[0] = -2.54000;
    e[0].Fp[1] =  0.0;     e[1].Fp[1] =  0.0;     e[2].Fp[1] =  0.0;
    e[0].Fp[2] =  0.62225; e[1].Fp[2] =  0.26539; e[2].Fp[2] =  0.20027;
    e[0].Fp[3] = -2.48824; e[1].Fp[3] =  4.58568; e[2].Fp[3] =  6.69465;
    e[0].eta = 0.78591; e[1].eta = 1.01318; e[2].eta = 1.18290;
    e[0].Fe = -2.82453; e[1].Fe = -2.70839; e[2].Fe = -2.55187;

    simox_potn* p = P->param;
    p[0].xm = 26.981539; p[1].xm = 58.6934; p[2].xm = 55.84500;
    p[0].qmin = 0.0; p[1].qmin = 0.0; p[2].qmin = 0.0;
    p[0].qmax = 3.0; p[1].qmax = 2.0; p[2].qmax = 3.0;
    p[0].chi = -1.47914; p[1].chi = -1.70804; p[2].chi = -1.90587;
    p[0].J = 9.07222; p[1].J = 9.10954; p[2].J = 8.99819;
    p[0].xi = 0.968; p[1].xi = 1.087; p[2].xi = 1.024;
    p[0].Z = 1.07514; p[1].Z = 1.44450; p[2].Z = 1.28612;
    p[3].xm = 15.9994; p[4].xm = 1.00794;
    p[3].qmin = -2.0; p[4].qmin = 0.0;
    p[3].qmax = 0.0;  p[4].qmax = 0.0;
    p[3].chi = 2.000; p[4].chi = 0.0;
    p[3].J = 14.99523; p[4].J = 0.0;
    p[3].xi = 2.144; p[4].xi = 0.0;
    p[3].Z = 0.00; p[4].Z = 0.0;
    for (int i = 0; i < SIMOX_NATOM; i++) {
        for (int j = 0; j < SIMOX_NATOM; j++) {
            double* f = p[i].fafb[j];
            if (i == j) {
                double xi = p[i].xi;
                f[0] = 1.0;
                f[1] = 11.0 * xi / 8.0;
                f[2] = 0.75 * (xi * xi);
                f[3] = (xi * xi * xi) / 6.0;
            } else {
                double a = p[i].xi, b = p[j].xi;
                double apb = a + b, amb = a - b, bma = b - a;
                double a2 = a * a, b2 = b * b, a4 = a2 * a2, b4 = b2 * b2;
                f[0] = a * b4 / (apb * apb) / (amb * amb);
                f[1] = b * a4 / (apb * apb) / (bma * bma);
                f[2] = (3.0 * a2 * b4 - b4 * b2) / (apb * apb * apb) / (amb * amb * amb);
                f[3] = (3.0 * b2 * a4 - a4 * a2) / (apb * apb * apb) / (bma * bma * bma);
            }
        }
    }
    simox_oxid* o = &P->oxygn;
    o->r_e[0] = 2.98520; o->r_e[1] = 2.95732; o->r_e[2] = 3.07992;
    o->alph[0] = 8.49741; o->alph[1] = 7.96528; o->alph[2] = 7.52309;
    o->beta[0] = 4.52114; o->beta[1] = 4.42411; o->beta[2] = 4.13330;
    o->A[0] = 0.09738; o->A[1] = 0.13521; o->A[2] = 0.17108;
    o->B[0] = 0.38121; o->B[1] = 0.25332; o->B[2] = 0.39869;
    o->kapp[0] = 0.18967; o->kapp[1] = 0.47077; o->kapp[2] = 0.22335;
    o->lamb[0] = 0.95234; o->lamb[1] = 0.65524; o->lamb[2] = 0.34380;
    o->r_e[3] = 3.64857; o->r_e[4] = 1.0;
    o->alph[3] = 5.44072; o->beta[3] = 3.59746; o->A[3] = 0.34900;
    o->B[3] = 0.57438; o->kapp[3] = 0.08007; o->lamb[3] = 0.39310;
    o->F0[0] = -1.56489; o->F1[0] = -1.58967; o->F2[0] = -1.54116;
    o->F0[1] = -1.39123; o->F1[1] =  1.30636; o->F2[1] =  2.02821;
    o->F0[2] =  1.77199; o->F1[2] =  9.81033; o->F2[2] =  6.56240;
    o->F0[3] =  1.59833; o->F1[3] =  0.0;     o->F2[3] =  0.0;
    o->F3[0] = -1.51798; o->F4[0] = -1.19082;
    o->F3[1] =  2.30979; o->F4[1] =  4.12936;
    o->F3[2] =  7.69582; o->F4[2] = 10.32338;
    o->F3[3] =  0.0;     o->F4[3] =  0.0;
    o->re[0] = 54.62910; o->rmax[0] = 54.62910;
    o->re[1] = 64.26953; o->rmax[1] = 65.24078;
    o->re[2] = 66.21202; o->rmax[2] = 66.56797;
    o->re[3] = 66.92391; o->rmax[3] = 70.57748;
    o->re[4] = 74.23105; o->rmax[4] = 99.99999e9;
    o->fe = 1.39478; o->gamm = 2.11725; o->nu = 0.37457;
}

/* ====================================================================== */
/* Cells  cellsort.f90                                                    */
/* ====================================================================== */
/* ID_CELL cellsort.f90:39-50 (1-based i,j,k in, 1-based id out) */
static int id_cell(const int nc[3], int i, int j, int k)
{
    int l = (i - 1 + nc[0]) % nc[0];
    int m = (j - 1 + nc[1]) % nc[1];
    int n = (k - 1 + nc[2]) % nc[2];
    return l + m * nc[0] + n * nc[0] * nc[1] + 1;
}

/* CELL_HIERARCHY cellsort.f90:3-36; pair[(id-1)*13 + n] */
void or_cell_hierarchy(const int nc[3], int* pair)
{
    for (int i = 1; i <= nc[0]; i++)
        for (int j = 1; j <= nc[1]; j++)
            for (int k = 1; k <= nc[2]; k++) {
                int id = id_cell(nc, i, j, k);
                int* p = pair + (id - 1) * 13;
                p[0]  = id_cell(nc, i - 1, j - 1, k - 1);
                p[1]  = id_cell(nc, i,     j - 1, k - 1);
                p[2]  = id_cell(nc, i + 1, j - 1, k - 1);
                p[3]  = id_cell(nc, i - 1, j,     k - 1);
                p[4]  = id_cell(nc, i,     j,     k - 1);
                p[5]  = id_cell(nc, i + 1, j,     k - 1);
                p[6]  = id_cell(nc, i - 1, j + 1, k - 1);
                p[7]  = id_cell(nc, i,     j + 1, k - 1);
                p[8]  = id_cell(nc, i + 1, j + 1, k - 1);
                p[9]  = id_cell(nc, i - 1, j - 1, k);
                p[10] = id_cell(nc, i,     j - 1, k);
                p[11] = id_cell(nc, i + 1, j - 1, k);
                p[12] = id_cell(nc, i - 1, j,     k);
            }
}

/* Cell grid of READ_INPUT main.f90:269-274. Returns 0 or SIMOX_E_CELL_TOO_SMALL. */
int or_cell_grid(const double box[3], double rcut, int nc[3], double lc[3])
{
    for (int d = 0; d < 3; d++) {
        nc[d] = (int)(box[d] / rcut);
        lc[d] = box[d] / (double)nc[d];
    }
    if (nc[0] < 3 && nc[1] < 3 && nc[2] < 3) return SIMOX_E_CELL_TOO_SMALL;
    return 0;
}

/* CELL_SORT cellsort.f90:53-80.  link[c*npt_max + k] = 1-based atom id. */
int or_cell_sort(int n, const double* x, const double box[3], const int nc[3],
                 const double lc[3], int npt_max, int* npt, int* link)
{
    int ncall = nc[0] * nc[1] * nc[2];
    double hbox[3] = {0.5 * box[0], 0.5 * box[1], 0.5 * box[2]};
    for (int c = 0; c < ncall; c++) npt[c] = 0;
    for (int i = 0; i < n; i++) {
        int id[3];
        for (int d = 0; d < 3; d++) {
            double xx = x[3 * i + d] + hbox[d];
            double t = xx / lc[d];
            if (!(fabs(t) < 1.0e9)) return SIMOX_E_POSITION;
            id[d] = (int)t;
            id[d] = (id[d] + nc[d]) % nc[d];
            if (id[d] < 0) return SIMOX_E_POSITION;
        }
        int c = id[0] + id[1] * nc[0] + id[2] * nc[0] * nc[1];
        npt[c]++;
        if (npt[c] > npt_max) return SIMOX_E_CELL_OVERFLOW;
        link[(size_t)c * npt_max + npt[c] - 1] = i + 1;
    }
    return 0;
}

/* ====================================================================== */
/* Pair forms  eam.f90                                                    */
/* ====================================================================== */
static inline double pow20(double t)
{
    double t2 = t * t, t4 = t2 * t2, t5 = t4 * t, t10 = t5 * t5;
    return t10 * t10;
}

/* METAL_HOMO eam.f90:3-35 */
static void metal_homo(const simox_metl* e, double r, double fj[2], double dfjdr[2],
                       double* phi, double* df)
{
    double re = e->r_e, fe = e->f_e, alpha = e->alpha, beta = e->beta;
    double lambda = e->lambda, kappa = e->kappa, A = e->A, B = e->B;
    double r_re = r / re, r_re_1 = r_re - 1.0;
    double l20 = pow20(r_re - lambda), l19 = l20 / (r_re - lambda);
    double k20 = pow20(r_re - kappa), k19 = k20 / (r_re - kappa);
    double ea = exp(-alpha * r_re_1), eb = exp(-beta * r_re_1);
    double ftn = eb / (1.0 + l20);
    double dftndr = eb * (-beta * (1.0 + l20) - 20.0 * l19) / re / ((1.0 + l20) * (1.0 + l20));
    fj[0] = fe * ftn; fj[1] = fj[0];
    dfjdr[0] = fe * dftndr / r; dfjdr[1] = dfjdr[0];
    *phi = A * ea / (1.0 + k20) - B * ftn;
    double dphidr = A * ea * (-alpha * (1.0 + k20) - 20.0 * k19) / re / ((1.0 + k20) * (1.0 + k20))
                    - B * dftndr;
    *df = -dphidr / r;
}

/* one Zhou-form term of eam.f90 and its radial derivative */
static void zhou_term(double r, double re, double c, double lam, double* g, double* dg)
{
    double r_re = r / re, r_re_1 = r_re - 1.0;
    double l20 = pow20(r_re - lam), l19 = l20 / (r_re - lam);
    double ex = exp(-c * r_re_1);
    *g = ex / (1.0 + l20);
    *dg = ex * (-c * (1.0 + l20) - 20.0 * l19) / re / ((1.0 + l20) * (1.0 + l20));
}

/* METAL_HETERO eam.f90:38-98 */
static void metal_hetero(const simox_metl* ei, const simox_metl* ej, double r,
                         double fj[2], double dfjdr[2], double* phi, double* df)
{
    double ftn, dftn, ga, dga;
    zhou_term(r, ei->r_e, ei->beta, ei->lambda, &ftn, &dftn);
    zhou_term(r, ei->r_e, ei->alpha, ei->kappa, &ga, &dga);
    fj[0] = ei->f_e * ftn; dfjdr[0] = ei->f_e * dftn / r;
    double phi_i = ei->A * ga - ei->B * ftn;
    double dphi_i = ei->A * dga - ei->B * dftn;
    zhou_term(r, ej->r_e, ej->beta, ej->lambda, &ftn, &dftn);
    zhou_term(r, ej->r_e, ej->alpha, ej->kappa, &ga, &dga);
    fj[1] = ej->f_e * ftn; dfjdr[1] = ej->f_e * dftn / r;
    double phi_j = ej->A * ga - ej->B * ftn;
    double dphi_j = ej->A * dga - ej->B * dftn;
    *phi = 0.5 * (phi_i * fj[1] / fj[0] + phi_j * fj[0] / fj[1]);
    *df = -0.5 * ((dphi_i * fj[1] * fj[0] + phi_i * dfjdr[1] * r * fj[0] - phi_i * fj[1] * dfjdr[0] * r) / (fj[0] * fj[0])
                + (dphi_j * fj[0] * fj[1] + phi_j * dfjdr[0] * r * fj[1] - phi_j * fj[0] * dfjdr[1] * r) / (fj[1] * fj[1])) / r;
}

/* AL_NI eam.f90:101-168 (uninitialised alpha/kappa of the density blocks are unused) */
static void al_ni(const simox_metl* ei, const simox_metl* ej, double r,
                  double fj[2], double dfjdr[2], double* phi, double* df)
{
    double g, dg;
    zhou_term(r, ei->r_e, ei->beta, ei->lambda, &g, &dg);
    fj[0] = ei->f_e * g; dfjdr[0] = ei->f_e * dg / r;
    zhou_term(r, ej->r_e, ej->beta, ej->lambda, &g, &dg);
    fj[1] = ej->f_e * g; dfjdr[1] = ej->f_e * dg / r;
    double ga, dga, gb, dgb;
    zhou_term(r, 2.71579, 8.00443, 0.63279, &ga, &dga);
    zhou_term(r, 2.71579, 4.75970, 0.81777, &gb, &dgb);
    *phi = 0.44254 * ga - 0.68349 * gb;
    *df = -(0.44254 * dga - 0.68349 * dgb) / r;
}

/* METAL_OXYGEN eam.f90:171-225 (metal i, oxygen j) and OXYGEN_METAL
 * eam.f90:228-283 (oxygen i, metal j): metal_first selects which slot of fj
 * holds the metal density. */
static void metal_oxygen(const simox_metl* em, int id_m, const simox_oxid* o, double r,
                         int metal_first, double fj[2], double dfjdr[2],
                         double* phi, double* df)
{
    double g, dg;
    zhou_term(r, em->r_e, em->beta, em->lambda, &g, &dg);
    double fm = em->f_e * g, dfm = em->f_e * dg / r;
    int m = id_m - 1;
    double re = o->r_e[m];
    double r_re = r / re, r_re_1 = r_re - 1.0;
    double l20 = pow20(r_re - o->lamb[m]), l19 = l20 / (r_re - o->lamb[m]);
    double k20 = pow20(r_re - o->kapp[m]), k19 = k20 / (r_re - o->kapp[m]);
    double ea = exp(-o->alph[m] * r_re_1), eb = exp(-o->beta[m] * r_re_1);
    double dphidr = o->A[m] * ea * (-o->alph[m] * (1.0 + k20) - 20.0 * k19) / re / ((1.0 + k20) * (1.0 + k20))
                  - o->B[m] * eb * (-o->beta[m] * (1.0 + l20) - 20.0 * l19) / re / ((1.0 + l20) * (1.0 + l20));
    *phi = o->A[m] * ea / (1.0 + k20) - o->B[m] * eb / (1.0 + l20);
    *df = -dphidr / r;
    double eg = exp(-o->gamm * r_re_1);
    double n20 = pow20(r_re - o->nu), n19 = n20 / (r_re - o->nu);
    double fo = o->fe * eg / (1.0 + n20);
    double dfo = o->fe * eg * (-o->gamm * (1.0 + n20) - 20.0 * n19) / re / ((1.0 + n20) * (1.0 + n20)) / r;
    if (metal_first) { fj[0] = fm; dfjdr[0] = dfm; fj[1] = fo; dfjdr[1] = dfo; }
    else             { fj[1] = fm; dfjdr[1] = dfm; fj[0] = fo; dfjdr[0] = dfo; }
}

/* OXYGEN_ONLY eam.f90:286-328 */
static void oxygen_only(const simox_oxid* o, double r, double fj[2], double dfjdr[2],
                        double* phi, double* df)
{
    double re = o->r_e[3];
    double r_re = r / re, r_re_1 = r_re - 1.0;
    double l20 = pow20(r_re - o->lamb[3]), l19 = l20 / (r_re - o->lamb[3]);
    double k20 = pow20(r_re - o->kapp[3]), k19 = k20 / (r_re - o->kapp[3]);
    double ea = exp(-o->alph[3] * r_re_1), eb = exp(-o->beta[3] * r_re_1);
    double dphidr = o->A[3] * ea * (-o->alph[3] * (1.0 + k20) - 20.0 * k19) / re / ((1.0 + k20) * (1.0 + k20))
                  - o->B[3] * eb * (-o->beta[3] * (1.0 + l20) - 20.0 * l19) / re / ((1.0 + l20) * (1.0 + l20));
    *phi = o->A[3] * ea / (1.0 + k20) - o->B[3] * eb / (1.0 + l20);
    *df = -dphidr / r;
    double eg = exp(-o->gamm * r_re_1);
    double n20 = pow20(r_re - o->nu), n19 = n20 / (r_re - o->nu);
    fj[0] = o->fe * eg / (1.0 + n20); fj[1] = fj[0];
    dfjdr[0] = o->fe * eg * (-o->gamm * (1.0 + n20) - 20.0 * n19) / re / ((1.0 + n20) * (1.0 + n20)) / r;
    dfjdr[1] = dfjdr[0];
}

/* dispatch of force.f90:58-74 */
static int pair_form(const simox_potential* P, int id_i, int id_j, double r,
                     double fj[2], double dfjdr[2], double* phi, double* df)
{
    if ((id_i < 4 && id_j < 4) && id_i == id_j) metal_homo(&P->eam[id_i - 1], r, fj, dfjdr, phi, df);
    else if (id_i == 1 && id_j == 2) al_ni(&P->eam[id_i - 1], &P->eam[id_j - 1], r, fj, dfjdr, phi, df);
    else if (id_i == 2 && id_j == 1) al_ni(&P->eam[id_j - 1], &P->eam[id_i - 1], r, fj, dfjdr, phi, df);
    else if ((id_i < 4 && id_j < 4) && id_i != id_j) metal_hetero(&P->eam[id_i - 1], &P->eam[id_j - 1], r, fj, dfjdr, phi, df);
    else if (id_i == 4 && id_j < 4) metal_oxygen(&P->eam[id_j - 1], id_j, &P->oxygn, r, 0, fj, dfjdr, phi, df);
    else if (id_i < 4 && id_j == 4) metal_oxygen(&P->eam[id_i - 1], id_i, &P->oxygn, r, 1, fj, dfjdr, phi, df);
    else if (id_i == 4 && id_j == 4) oxygen_only(&P->oxygn, r, fj, dfjdr, phi, df);
    else return SIMOX_E_UNKNOWN_PAIR;
    return 0;
}

/* ====================================================================== */
/* FORCE  force.f90:3-361                                                 */
/* ====================================================================== */
typedef struct {
    int n;
    const int* id; const double* x; const double* q;
    const int* npt; const int* link; const int* pair;
    int ncall, npt_max;
    double box[3], rcut2, a;
} or_pairs;

/* CTIP same-/different-species terms force.f90:101-140 */
static void ctip_pair(const simox_potential* P, int id_i, int id_j, double r, double r2,
                      double q_i, double q_j, double* df, double* e)
{
    double xi_i = P->param[id_i - 1].xi, xi_j = P->param[id_j - 1].xi;
    double Z_i = P->param[id_i - 1].Z, Z_j = P->param[id_j - 1].Z;
    const double* f = P->param[id_i - 1].fafb[id_j - 1];
    double jfi, ifj, djfidr, difjdr, fifj, dfifjdr;
    if (id_i == id_j) {
        double xir_i = 2.0 * xi_i * r, ex = exp(-xir_i);
        jfi = -ex * (xi_i + 1.0 / r); ifj = jfi;
        djfidr = ex * (2.0 * (xi_i * xi_i) + (1.0 + xir_i) / r2); difjdr = djfidr;
        fifj = -ex * (1.0 + f[1] * r + f[2] * r2 + f[3] * r2 * r);
        dfifjdr = ex * ((xir_i + 1.0) * (1.0 / r2 + f[1] / r + f[2] + f[3] * r)
                        - (f[1] / r + f[2] * 2.0 + f[3] * 3.0 * r));
    } else {
        double xir_i = 2.0 * xi_i * r, exi = exp(-xir_i);
        double xir_j = 2.0 * xi_j * r, exj = exp(-xir_j);
        jfi = -exi * (xi_i + 1.0 / r);
        ifj = -exj * (xi_j + 1.0 / r);
        djfidr = exi * (2.0 * (xi_i * xi_i) + (1.0 + xir_i) / r2);
        difjdr = exj * (2.0 * (xi_j * xi_j) + (1.0 + xir_j) / r2);
        fifj = -f[0] * exi - f[1] * exj - f[2] * exi / r - f[3] * exj / r;
        dfifjdr = f[0] * exi * 2.0 * xi_i + f[1] * exj * 2.0 * xi_j
                + f[2] * exi * (1.0 + xir_i) / r2 + f[3] * exj * (1.0 + xir_j) / r2;
    }
    *df = KC * ((q_i * Z_j + q_j * Z_i - q_i * q_j) * dfifjdr - q_i * Z_j * djfidr - q_j * Z_i * difjdr) / r;
    *e = q_i * Z_j * (jfi - fifj) + q_j * Z_i * (ifj - fifj) + q_i * q_j * fifj;
}

/* Embedding F(rho), F'(rho)  force.f90:256-351 */
static int embed(const simox_potential* P, int id, double rho, double* F, double* dF)
{
    double F_sum = 0.0, d = 0.0;
    const double* c = NULL;
    double rr = 0.0;
    if (id < 4) {
        const simox_metl* e = &P->eam[id - 1];
        double rho_n = 0.85 * e->rho_e, rho_0 = 1.15 * e->rho_e;
        if (rho < rho_n) { c = e->Fn; rr = rho_n; }
        else if (rho < e->rho_e) { c = e->Fm; rr = e->rho_e; }
        else if (rho < rho_0) { c = e->Fp; rr = e->rho_e; }
        else if (rho > 1.0e-6) {
            double t = pow(rho / e->rho_s, e->eta);
            F_sum = e->Fe * (1.0 - log(t)) * t;
            d = -e->Fe * e->eta * log(t) * t / rho;
        }
    } else if (id == 4) {
        const simox_oxid* o = &P->oxygn;
        if (rho < o->rmax[0]) { c = o->F0; rr = o->re[0]; }
        else if (rho < o->rmax[1]) { c = o->F1; rr = o->re[1]; }
        else if (rho < o->rmax[2]) { c = o->F2; rr = o->re[2]; }
        else if (rho < o->rmax[3]) { c = o->F3; rr = o->re[3]; }
        else { c = o->F4; rr = o->re[4]; }
    } else {
        return SIMOX_E_UNKNOWN_ELEMENT;
    }
    if (c) {
        double t = rho / rr - 1.0;
        double tp[4] = {1.0, t, t * t, t * t * t};
        for (int j = 0; j < 4; j++) F_sum = F_sum + c[j] * tp[j];
        for (int j = 1; j < 4; j++) d = d + c[j] * (double)j * tp[j - 1] / rr;
    }
    *F = F_sum; *dF = d;
    return 0;
}

/* E[0..3] = Epair, Edir(*kc), Ectip(*kc), Egroup.  f overwritten. */
int or_force(int n, const double box[3], double rcut, const int nc[3], int npt_max, int nnb_max,
             const simox_potential* P, const int* id, const double* x, const double* q,
             const int* npt, const int* link, const int* pair,
             double* f, double* E, int* rdf, double* rho_out, double* dFdrho_out)
{
    int ncall = nc[0] * nc[1] * nc[2];
    double rcut2 = rcut * rcut, a = 3.8 / rcut, a2 = a * a, dr = rcut / (double)SIMOX_NRDF;
    int* nlist = (int*)calloc(n, sizeof(int));
    int* list = (int*)calloc((size_t)n * nnb_max, sizeof(int));
    double* drho_list = (double*)calloc((size_t)n * nnb_max * 3, sizeof(double));
    double* rho = (double*)calloc(n, sizeof(double));
    double* drhodx = (double*)calloc((size_t)n * 3, sizeof(double));
    double* dFdrho = (double*)calloc(n, sizeof(double));
    int st = 0;
    if (!nlist || !list || !drho_list || !rho || !drhodx || !dFdrho) { st = SIMOX_E_NOMEM; goto done; }
    for (int i = 0; i < 3 * n; i++) f[i] = 0.0;
    double Edir = 0.0, Epair = 0.0, Egroup = 0.0, Ectip = 0.0;

    for (int m = 0; m < ncall; m++) {
        int Nloc = npt[m];
        const int* lk = link + (size_t)m * npt_max;
        /* in-cell pairs force.f90:45-143, then 13 stencil cells force.f90:146-248 */
        for (int pass = 0; pass < 14; pass++) {
            int cj = pass == 0 ? m : pair[m * 13 + pass - 1] - 1;
            const int* lkj = link + (size_t)cj * npt_max;
            int Nj = npt[cj];
            int outer_n = pass == 0 ? Nloc - 1 : Nj;
            for (int oi = 0; oi < outer_n; oi++) {
                int inner_lo = pass == 0 ? oi + 1 : 0;
                int inner_hi = pass == 0 ? Nloc : Nloc;
                for (int ii = inner_lo; ii < inner_hi; ii++) {
                    int li, lj;
                    if (pass == 0) { li = lk[oi] - 1; lj = lk[ii] - 1; }
                    else           { lj = lkj[oi] - 1; li = lk[ii] - 1; }
                    double rx[3];
                    for (int d = 0; d < 3; d++) {
                        double dx = x[3 * li + d] - x[3 * lj + d];
                        rx[d] = dx - box[d] * round(dx / box[d]);
                    }
                    double r2 = rx[0] * rx[0] + rx[1] * rx[1] + rx[2] * rx[2];
                    if (!(r2 < rcut2)) continue;
                    double r = sqrt(r2);
                    int id_r = (int)(r / dr);
                    int id_i = id[li], id_j = id[lj];
                    double q_i = q[li], q_j = q[lj];
                    double fj[2], dfjdr[2], phi, df;
                    st = pair_form(P, id_i, id_j, r, fj, dfjdr, &phi, &df);
                    if (st) goto done;
                    if (rdf) rdf[(id_i - 1) + 5 * (id_j - 1) + 25 * id_r] += 2;
                    nlist[li]++; nlist[lj]++;
                    if (nlist[li] > nnb_max || nlist[lj] > nnb_max) { st = SIMOX_E_NBR_OVERFLOW; goto done; }
                    list[(size_t)li * nnb_max + nlist[li] - 1] = lj;
                    list[(size_t)lj * nnb_max + nlist[lj] - 1] = li;
                    for (int d = 0; d < 3; d++) {
                        drho_list[((size_t)li * nnb_max + nlist[li] - 1) * 3 + d] = rx[d] * dfjdr[0];
                        drho_list[((size_t)lj * nnb_max + nlist[lj] - 1) * 3 + d] = -rx[d] * dfjdr[1];
                    }
                    rho[li] += fj[1];
                    rho[lj] += fj[0];
                    for (int d = 0; d < 3; d++) {
                        drhodx[3 * li + d] += rx[d] * dfjdr[1];
                        drhodx[3 * lj + d] -= rx[d] * dfjdr[0];
                        f[3 * li + d] += rx[d] * df;
                        f[3 * lj + d] -= rx[d] * df;
                    }
                    Epair += phi;
                    /* Ewald real space force.f90:94-98 */
                    double tmp = erfc(a * r);
                    Edir += q_i * q_j * tmp / r;
                    df = KC * q_i * q_j * (2.0 * exp(-a2 * r2) * a * r / SQRTPI + tmp) / r2 / r;
                    for (int d = 0; d < 3; d++) { f[3 * li + d] += df * rx[d]; f[3 * lj + d] -= df * rx[d]; }
                    /* CTIP force.f90:101-140 */
                    double ect;
                    ctip_pair(P, id_i, id_j, r, r2, q_i, q_j, &df, &ect);
                    for (int d = 0; d < 3; d++) { f[3 * li + d] += df * rx[d]; f[3 * lj + d] -= df * rx[d]; }
                    Ectip += ect;
                }
            }
        }
    }
    E[0] = Epair; E[1] = Edir * KC; E[2] = Ectip * KC;
    for (int i = 0; i < n; i++) {
        double F;
        st = embed(P, id[i], rho[i], &F, &dFdrho[i]);
        if (st) goto done;
        for (int d = 0; d < 3; d++) f[3 * i + d] -= drhodx[3 * i + d] * dFdrho[i];
        Egroup += F;
    }
    E[3] = Egroup;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < nlist[i]; j++) {
            int jj = list[(size_t)i * nnb_max + j];
            for (int d = 0; d < 3; d++)
                f[3 * i + d] -= dFdrho[jj] * drho_list[((size_t)i * nnb_max + j) * 3 + d];
        }
    if (rho_out) memcpy(rho_out, rho, n * sizeof(double));
    if (dFdrho_out) memcpy(dFdrho_out, dFdrho, n * sizeof(double));
done:
    free(nlist); free(list); free(drho_list); free(rho); free(drhodx); free(dFdrho);
    return st;
}

/* ====================================================================== */
/* FFT: ZFFT3D(A,NX,NY,NZ,IOPT) semantics of FFTE (force.f90:412-426).    */
/* IOPT = -1: forward, sum a(j) exp(-2 pi i jk/n).  IOPT = +1: inverse,   */
/* (1/N) sum a(j) exp(+2 pi i jk/n).  Own self-sorting (Stockham)         */
/* mixed-radix 2/3/4/5 algorithm; checked against a naive DFT in tests.   */
/* ====================================================================== */
/* Plan for one length and direction: radix list and per-stage twiddles. */
typedef struct {
    int n, sign, nf, f[64];
    cplx* tw;            /* per stage: m*r twiddles w_len^(p*j) */
    cplx roots[6][5];    /* roots[r][e] = exp(sign 2 pi i e / r) */
} fftplan;

static int factor_radix(int n, int* f)
{
    int nf = 0;
    while (n % 4 == 0) { f[nf++] = 4; n /= 4; }
    while (n % 2 == 0) { f[nf++] = 2; n /= 2; }
    while (n % 3 == 0) { f[nf++] = 3; n /= 3; }
    while (n % 5 == 0) { f[nf++] = 5; n /= 5; }
    return n == 1 ? nf : -1;
}

static void plan_init(fftplan* P, int n, int sign)
{
    P->n = n; P->sign = sign;
    P->nf = factor_radix(n, P->f);
    for (int r = 2; r <= 5; r++)
        for (int e = 0; e < r; e++) {
            double ang = sign * 2.0 * PI_ * (double)e / (double)r;
            P->roots[r][e].re = cos(ang); P->roots[r][e].im = sin(ang);
        }
    P->tw = NULL;
    if (P->nf < 0) return;
    size_t tot = 0; int len = n;
    for (int t = 0; t < P->nf; t++) { tot += (size_t)len; len /= P->f[t]; }
    P->tw = (cplx*)malloc(sizeof(cplx) * (tot + 1));
    size_t off = 0; len = n;
    for (int t = 0; t < P->nf; t++) {
        int r = P->f[t], m = len / r;
        double th = sign * 2.0 * PI_ / (double)len;
        for (int p = 0; p < m; p++)
            for (int j = 0; j < r; j++) {
                double ang = th * (double)((long)p * j);
                P->tw[off + (size_t)p * r + j].re = cos(ang);
                P->tw[off + (size_t)p * r + j].im = sin(ang);
            }
        off += (size_t)len; len = m;
    }
}

static void plan_free(fftplan* P) { free(P->tw); P->tw = NULL; }

/* one 1-D complex transform of length n in place (x), work y of length n */
static void fft1d(const fftplan* P, cplx* x, cplx* y)
{
    int n = P->n, sign = P->sign;
    if (P->nf < 0) { /* length not 2/3/5-smooth: naive DFT */
        for (int k = 0; k < n; k++) {
            double sr = 0.0, si = 0.0;
            for (int j = 0; j < n; j++) {
                double ang = sign * 2.0 * PI_ * (double)(((long)j * k) % n) / (double)n;
                sr += x[j].re * cos(ang) - x[j].im * sin(ang);
                si += x[j].re * sin(ang) + x[j].im * cos(ang);
            }
            y[k].re = sr; y[k].im = si;
        }
        memcpy(x, y, n * sizeof(cplx));
        return;
    }
    /* self-sorting (Stockham) decimation in frequency: a stage of radix r
     * over sub-length len with stride s maps x[q + s(p + k m)] to
     * y[q + s(r p + j)] = (sum_k x_k root_r^{jk}) * w_len^{p j}. */
    cplx* src = x; cplx* dst = y;
    int len = n, s = 1;
    size_t off = 0;
    cplx a[5];
    for (int t = 0; t < P->nf; t++) {
        int r = P->f[t], m = len / r;
        const cplx* rt = P->roots[r];
        for (int p = 0; p < m; p++) {
            const cplx* w = P->tw + off + (size_t)p * r;
            for (int qq = 0; qq < s; qq++) {
                for (int k = 0; k < r; k++) a[k] = src[qq + s * (p + k * m)];
                for (int j = 0; j < r; j++) {
                    double sr = 0.0, si = 0.0;
                    for (int k = 0; k < r; k++) {
                        cplx c = rt[(j * k) % r];
                        sr += a[k].re * c.re - a[k].im * c.im;
                        si += a[k].re * c.im + a[k].im * c.re;
                    }
                    cplx o;
                    o.re = sr * w[j].re - si * w[j].im;
                    o.im = sr * w[j].im + si * w[j].re;
                    dst[qq + s * (r * p + j)] = o;
                }
            }
        }
        cplx* tt = src; src = dst; dst = tt;
        off += (size_t)len; len = m; s *= r;
    }
    if (src != x) memcpy(x, src, n * sizeof(cplx));
}

void or_zfft3d(double* A, int nx, int ny, int nz, int iopt)
{
    if (iopt == 0) return;
    int sign = iopt > 0 ? +1 : -1;
    cplx* g = (cplx*)A;
    int nmax = nx > ny ? nx : ny; if (nz > nmax) nmax = nz;
    const int B = 16;
    fftplan px, py, pz;
    plan_init(&px, nx, sign); plan_init(&py, ny, sign); plan_init(&pz, nz, sign);
    cplx* line = (cplx*)malloc(sizeof(cplx) * nmax * B);
    cplx* work = (cplx*)malloc(sizeof(cplx) * nmax);
    /* x lines (contiguous) */
    for (int l = 0; l < ny * nz; l++) fft1d(&px, g + (size_t)l * nx, work);
    /* y lines: batches of B consecutive x */
    for (int k = 0; k < nz; k++)
        for (int i0 = 0; i0 < nx; i0 += B) {
            int bb = nx - i0 < B ? nx - i0 : B;
            for (int j = 0; j < ny; j++)
                for (int b = 0; b < bb; b++) line[b * ny + j] = g[i0 + b + (size_t)nx * (j + (size_t)ny * k)];
            for (int b = 0; b < bb; b++) fft1d(&py, line + b * ny, work);
            for (int j = 0; j < ny; j++)
                for (int b = 0; b < bb; b++) g[i0 + b + (size_t)nx * (j + (size_t)ny * k)] = line[b * ny + j];
        }
    /* z lines */
    for (int j = 0; j < ny; j++)
        for (int i0 = 0; i0 < nx; i0 += B) {
            int bb = nx - i0 < B ? nx - i0 : B;
            for (int k = 0; k < nz; k++)
                for (int b = 0; b < bb; b++) line[b * nz + k] = g[i0 + b + (size_t)nx * (j + (size_t)ny * k)];
            for (int b = 0; b < bb; b++) fft1d(&pz, line + b * nz, work);
            for (int k = 0; k < nz; k++)
                for (int b = 0; b < bb; b++) g[i0 + b + (size_t)nx * (j + (size_t)ny * k)] = line[b * nz + k];
        }
    if (sign > 0) {
        double s = 1.0 / ((double)nx * ny * nz);
        size_t N = (size_t)nx * ny * nz;
        for (size_t i = 0; i < N; i++) { g[i].re *= s; g[i].im *= s; }
    }
    free(line); free(work);
    plan_free(&px); plan_free(&py); plan_free(&pz);
}

/* naive DFT along all axes (for FFT tests) with the same conventions */
void or_dft3d_naive(const double* in, double* out, int nx, int ny, int nz, int iopt)
{
    int sign = iopt > 0 ? +1 : -1;
    const cplx* a = (const cplx*)in; cplx* o = (cplx*)out;
    size_t N = (size_t)nx * ny * nz;
    for (int kz = 0; kz < nz; kz++) for (int ky = 0; ky < ny; ky++) for (int kx = 0; kx < nx; kx++) {
        double sr = 0.0, si = 0.0;
        for (int z = 0; z < nz; z++) for (int y = 0; y < ny; y++) for (int x = 0; x < nx; x++) {
            double ang = sign * 2.0 * PI_ * ((double)(kx * x % nx) / nx + (double)(ky * y % ny) / ny + (double)(kz * z % nz) / nz);
            const cplx v = a[x + (size_t)nx * (y + (size_t)ny * z)];
            sr += v.re * cos(ang) - v.im * sin(ang);
            si += v.re * sin(ang) + v.im * cos(ang);
        }
        if (sign > 0) { sr /= (double)N; si /= (double)N; }
        o[kx + (size_t)nx * (ky + (size_t)ny * kz)].re = sr;
        o[kx + (size_t)nx * (ky + (size_t)ny * kz)].im = si;
    }
}

/* ====================================================================== */
/* B-spline weights: force.f90:388-400 (order 4), generalised to order p  */
/* ====================================================================== */
/* Stencil point n (0..p-1) of coordinate u is INT(u) - p/2 + 1 + n (0-based
 * grid index before wrapping); w[n] its weight and dw[n] = dw/du. */
static void bspline_ref4(double u, double* w, double* dw)
{
    double z = trunc(u) - u + 1.0;   /* DINT(u) - u + 1 */
    w[0] = z * z * z / 6.0;
    dw[0] = -3.0 * (z * z) / 6.0;
    z = z + 1.0;
    w[1] = (-3.0 * (z * z * z) + 12.0 * (z * z) - 12.0 * z + 4.0) / 6.0;
    dw[1] = (9.0 * (z * z) - 24.0 * z + 12.0) / 6.0;
    z = z + 1.0;
    w[2] = (3.0 * (z * z * z) - 24.0 * (z * z) + 60.0 * z - 44.0) / 6.0;
    dw[2] = (-9.0 * (z * z) + 48.0 * z - 60.0) / 6.0;
    z = z + 1.0;
    w[3] = (-(z * z * z) + 12.0 * (z * z) - 48.0 * z + 64.0) / 6.0;
    dw[3] = (3.0 * (z * z) - 24.0 * z + 48.0) / 6.0;
}

/* cardinal B-spline recursion M_n(x) = (x M_{n-1}(x) + (n-x) M_{n-1}(x-1))/(n-1) */
void or_bspline_gen(int p, double u, double* w, double* dw)
{
    double fr = u - trunc(u);
    double M[16] = {0}, Mn[16];
    M[0] = fr; M[1] = 1.0 - fr;       /* M_2(fr + k), k = 0, 1 */
    double dA[16] = {0};
    for (int n = 3; n <= p; n++) {
        if (n == p)
            for (int k = 0; k < p; k++) dA[k] = (k < p - 1 ? M[k] : 0.0) - (k >= 1 ? M[k - 1] : 0.0);
        for (int k = 0; k < n; k++) {
            double xk = fr + k;
            double a1 = k < n - 1 ? M[k] : 0.0;
            double a0 = k >= 1 ? M[k - 1] : 0.0;
            Mn[k] = (xk * a1 + ((double)n - xk) * a0) / (double)(n - 1);
        }
        for (int k = 0; k < n; k++) M[k] = Mn[k];
    }
    for (int s = 0; s < p; s++) { w[s] = M[p - 1 - s]; dw[s] = dA[p - 1 - s]; }
}

static void bspline(int p, double u, double* w, double* dw)
{
    if (p == 4) bspline_ref4(u, w, dw);
    else or_bspline_gen(p, u, w, dw);
}

/* 1/|b(theta)|^2 per dimension: order 4 as force.f90:415-420; order p from
 * the centred B-spline values beta(j) = M_p(j + p/2). */
static double bmod_inv(int p, int k, int K)
{
    double th = 2.0 * PI_ * (double)k / (double)K;
    double w[16], dw[16];
    or_bspline_gen(p, (double)(p / 2), w, dw);   /* fr = 0: w[s] = beta at offset */
    /* at u integer, stencil point s has offset t = u - g = p/2 - 1 - s */
    double b = 0.0;
    for (int s = 0; s < p; s++) {
        int t = p / 2 - 1 - s;
        b += w[s] * cos(th * t);
    }
    return 1.0 / (b * b);
}

/* ====================================================================== */
/* PME_SELF force.f90:467-517                                             */
/* ====================================================================== */
void or_pme_self(int n, const double box[3], double rcut, const int fft[3], const simox_potential* P,
                 const int* id, const double* q, double* psi, double* Eself_out)
{
    double a = 3.8 / rcut, a2 = a * a;
    double Eself = 0.0, Esum = 0.0;
    for (int i = 0; i < n; i++) {
        double qi = q[i];
        Eself = Eself - qi * qi;
        const simox_potn* pp = &P->param[id[i] - 1];
        Esum = Esum + pp->chi * qi + 0.5 * pp->J * (qi * qi);
        double dq = qi - pp->qmin;
        if (dq < 0.0) Esum = Esum + 2.0 * WPEN * (dq * dq);
        dq = qi - pp->qmax;
        if (dq > 0.0) Esum = Esum + 2.0 * WPEN * (dq * dq);
    }
    *Eself_out = Eself * a / SQRTPI * KC + Esum;
    if (!psi) return;
    for (int i = 1; i <= fft[0]; i++) {
        int ix = (i - 1 + fft[0] / 2) % fft[0] - fft[0] / 2;
        for (int j = 1; j <= fft[1]; j++) {
            int iy = (j - 1 + fft[1] / 2) % fft[1] - fft[1] / 2;
            for (int k = 1; k <= fft[2]; k++) {
                int iz = (k - 1 + fft[2] / 2) % fft[2] - fft[2] / 2;
                int m = ix * ix + iy * iy + iz * iz;
                double v = 0.0;
                if (m != 0) {
                    double m2 = (double)(ix * ix) / (box[0] * box[0]) + (double)(iy * iy) / (box[1] * box[1])
                              + (double)(iz * iz) / (box[2] * box[2]);
                    v = exp(-m2 * (PI_ * PI_) / a2) / m2;
                }
                psi[(i - 1) + (size_t)fft[0] * ((j - 1) + (size_t)fft[1] * (k - 1))] = v;
            }
        }
    }
}

/* grid point index (0-based, wrapped) of stencil point s along one axis */
static inline int stencil_index(double u, int s, int p, int K)
{
    int v = (int)u - p / 2 + 1 + s + K;
    v %= K;
    if (v < 0) v += K;
    return v;
}

/* Q <- spread of charges (real parts of a complex grid). */
static void spread(int n, const double* x, const double* q, const double box[3], const int fft[3], int p, double* Q)
{
    size_t N = (size_t)fft[0] * fft[1] * fft[2];
    memset(Q, 0, sizeof(double) * 2 * N);
    for (int i = 0; i < n; i++) {
        double u[3], w[3][16], dw[3][16];
        int ix[3][16];
        for (int d = 0; d < 3; d++) {
            u[d] = (double)fft[d] * (x[3 * i + d] + box[d] * 0.5) / box[d];
            bspline(p, u[d], w[d], dw[d]);
            for (int s = 0; s < p; s++) ix[d][s] = stencil_index(u[d], s, p, fft[d]);
        }
        for (int a = 0; a < p; a++)
            for (int b = 0; b < p; b++)
                for (int c = 0; c < p; c++) {
                    size_t g = ix[0][a] + (size_t)fft[0] * (ix[1][b] + (size_t)fft[1] * ix[2][c]);
                    Q[2 * g] += q[i] * spread_value(w[0][a] * w[1][b] * w[2][c]);
                }
    }
}

/* Qfin = FFT_-1( G * FFT_+1(Qbas) ), G = psi * prod bmod (force.f90:411-426) */
static void convolve(const int fft[3], int p, const double* psi, const double* Qbas, double* Qfin)
{
    size_t N = (size_t)fft[0] * fft[1] * fft[2];
    memcpy(Qfin, Qbas, sizeof(double) * 2 * N);
    or_zfft3d(Qfin, fft[0], fft[1], fft[2], 0);
    or_zfft3d(Qfin, fft[0], fft[1], fft[2], +1);
    double* b[3];
    for (int d = 0; d < 3; d++) {
        b[d] = (double*)malloc(sizeof(double) * fft[d]);
        for (int i = 0; i < fft[d]; i++) {
            if (p == 4) {   /* z = (4 + 2 cos(2 pi (i-1)/K))**2 */
                double c = 4.0 + 2.0 * cos(2.0 * PI_ * (double)i / (double)fft[d]);
                b[d][i] = c * c;
            } else {
                b[d][i] = bmod_inv(p, i, fft[d]);
            }
        }
    }
    for (int k = 0; k < fft[2]; k++)
        for (int j = 0; j < fft[1]; j++)
            for (int i = 0; i < fft[0]; i++) {
                size_t g = i + (size_t)fft[0] * (j + (size_t)fft[1] * k);
                for (int c = 0; c < 2; c++) {
                    double v = Qfin[2 * g + c];
                    if (p == 4) {
                        v = v * psi[g] * 46656.0 / b[0][i] / b[1][j] / b[2][k];
                    } else {
                        v = v * psi[g] * b[0][i] * b[1][j] * b[2][k];
                    }
                    Qfin[2 * g + c] = v;
                }
            }
    for (int d = 0; d < 3; d++) free(b[d]);
    or_zfft3d(Qfin, fft[0], fft[1], fft[2], 0);
    or_zfft3d(Qfin, fft[0], fft[1], fft[2], -1);
}

/* PME force.f90:364-464: f += reciprocal forces - mean; *Erec set */
int or_pme(int n, const double box[3], const int fft[3], int p, const double* psi,
           const double* x, const double* q, double* f, double* Erec)
{
    size_t N = (size_t)fft[0] * fft[1] * fft[2];
    double* Qbas = (double*)malloc(sizeof(double) * 2 * N);
    double* Qfin = (double*)malloc(sizeof(double) * 2 * N);
    double* ff = (double*)calloc((size_t)n * 3, sizeof(double));
    if (!Qbas || !Qfin || !ff) { free(Qbas); free(Qfin); free(ff); return SIMOX_E_NOMEM; }
    double V = box[0] * box[1] * box[2];
    spread(n, x, q, box, fft, p, Qbas);
    convolve(fft, p, psi, Qbas, Qfin);
    double Epme = 0.0;
    for (int i = 0; i < fft[0]; i++)
        for (int j = 0; j < fft[1]; j++)
            for (int k = 0; k < fft[2]; k++) {
                size_t g = i + (size_t)fft[0] * (j + (size_t)fft[1] * k);
                Epme = Epme + (Qbas[2 * g] * Qfin[2 * g] - Qbas[2 * g + 1] * Qfin[2 * g + 1]);
            }
    Epme = Epme * (double)fft[0] * (double)fft[1] * (double)fft[2];
    double cst = KC * (double)fft[0] * (double)fft[1] * (double)fft[2] / V / PI_;
    double kx[3] = {fft[0] / box[0], fft[1] / box[1], fft[2] / box[2]};
    double Fsum[3] = {0, 0, 0};
    for (int i = 0; i < n; i++) {
        double u[3], w[3][16], dw[3][16];
        int ix[3][16];
        for (int d = 0; d < 3; d++) {
            u[d] = (double)fft[d] * (x[3 * i + d] + box[d] * 0.5) / box[d];
            bspline(p, u[d], w[d], dw[d]);
            for (int s = 0; s < p; s++) ix[d][s] = stencil_index(u[d], s, p, fft[d]);
        }
        double qi = q[i];
        for (int a = 0; a < p; a++)
            for (int b = 0; b < p; b++)
                for (int c = 0; c < p; c++) {
                    double d0 = qi * dw[0][a] * w[1][b] * w[2][c] * kx[0];
                    double d1 = qi * w[0][a] * dw[1][b] * w[2][c] * kx[1];
                    double d2 = qi * w[0][a] * w[1][b] * dw[2][c] * kx[2];
                    size_t g = ix[0][a] + (size_t)fft[0] * (ix[1][b] + (size_t)fft[1] * ix[2][c]);
                    double Qf = Qfin[2 * g];
                    ff[3 * i + 0] = ff[3 * i + 0] - cst * d0 * Qf;
                    ff[3 * i + 1] = ff[3 * i + 1] - cst * d1 * Qf;
                    ff[3 * i + 2] = ff[3 * i + 2] - cst * d2 * Qf;
                }
        for (int d = 0; d < 3; d++) Fsum[d] += ff[3 * i + d];
    }
    for (int d = 0; d < 3; d++) Fsum[d] /= (double)n;
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) f[3 * i + d] = f[3 * i + d] + ff[3 * i + d] - Fsum[d];
    *Erec = KC * Epme / V / PI_ / 2.0;
    free(Qbas); free(Qfin); free(ff);
    return 0;
}

/* ====================================================================== */
/* CTIP_SOLVER ctip.f90:3-396                                             */
/* ====================================================================== */
typedef struct {
    int n, p, nnb_max;
    int fft[3];
    const double* psi;
    double c_pme;
    double* XJZ;      /* [n][3] */
    double* qmx;      /* [n][2] */
    double* Qlocal;   /* [n][p^3] */
    int* grid;        /* [n][p^3] flattened grid index */
    double* asym; double* sym; int* list; int* nlist;
    double* Qbas; double* Qfin;
    long n_eval;
} ctip_ws;

/* PHI_MESH ctip.f90:336-396 (phi unscaled) */
static void phi_mesh(ctip_ws* w, const double* q, double* phi)
{
    size_t N = (size_t)w->fft[0] * w->fft[1] * w->fft[2];
    int p3 = w->p * w->p * w->p;
    memset(w->Qbas, 0, sizeof(double) * 2 * N);
    for (int i = 0; i < w->n; i++)
        for (int s = 0; s < p3; s++)
            w->Qbas[2 * (size_t)w->grid[(size_t)i * p3 + s]] += q[i] * spread_value(w->Qlocal[(size_t)i * p3 + s]);
    convolve(w->fft, w->p, w->psi, w->Qbas, w->Qfin);
    for (int i = 0; i < w->n; i++) {
        double E = 0.0;
        for (int s = 0; s < p3; s++)
            E = E + w->Qlocal[(size_t)i * p3 + s] * w->Qfin[2 * (size_t)w->grid[(size_t)i * p3 + s]];
        phi[i] = E;
    }
    w->n_eval++;
}

/* dUdq ctip.f90:307-333: g = -dU/dq */
static void dudq(ctip_ws* w, const double* q, const double* phi, double* g)
{
    for (int i = 0; i < w->n; i++) {
        double dqmin = q[i] - w->qmx[2 * i], dqmax = q[i] - w->qmx[2 * i + 1];
        if (dqmin >= 0.0) dqmin = 0.0;
        if (dqmax <= 0.0) dqmax = 0.0;
        g[i] = -(w->XJZ[3 * i] + w->XJZ[3 * i + 1] * q[i] + phi[i] + 2.0 * WPEN * (dqmin + dqmax));
    }
    for (int i = 0; i < w->n; i++)
        for (int j = 0; j < w->nlist[i]; j++) {
            int jj = w->list[(size_t)i * w->nnb_max + j];
            g[i] = g[i] - w->XJZ[3 * jj + 2] * w->asym[(size_t)i * w->nnb_max + j]
                        - q[jj] * w->sym[(size_t)i * w->nnb_max + j];
        }
}

/* -sum g(q + b p) p */
static double line_fn(ctip_ws* w, const double* q, const double* pv, double b,
                      double* ql, double* phi, double* g)
{
    for (int i = 0; i < w->n; i++) ql[i] = q[i] + b * pv[i];
    phi_mesh(w, ql, phi);
    for (int i = 0; i < w->n; i++) phi[i] = phi[i] * w->c_pme;
    dudq(w, ql, phi, g);
    double s = 0.0;
    for (int i = 0; i < w->n; i++) s = s - g[i] * pv[i];
    return s;
}

/* BRENT_SOLVER ctip.f90:216-304 */
static int brent(ctip_ws* w, const double* q, const double* pv, double* alpha,
                 double* ql, double* phi, double* g)
{
    const int Nmax = 100;
    const double E_crit = 1.0e-8, E_end = 1.0e-11;
    double a = -1.0, b = 1.0, c, d = 0.0, e = 0.0, fa, fb, fc, xm, s, x, y, z;
    fa = line_fn(w, q, pv, a, ql, phi, g);
    fb = line_fn(w, q, pv, b, ql, phi, g);
    c = b; fc = fb;
    for (int n = 1; n <= Nmax; n++) {
        if ((fb > 0.0 && fc > 0.0) || (fb < 0.0 && fc < 0.0)) { c = a; fc = fa; d = b - a; e = d; }
        if (fabs(fc) < fabs(fb)) { a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
        xm = 0.5 * (c - b);
        if (fabs(xm) < E_crit || fabs(fb) < E_end) { *alpha = b; return 0; }
        if (fabs(e) >= E_crit && fabs(fa) > fabs(fb)) {
            s = fb / fa;
            if (a == c) { x = 2.0 * xm * s; y = 1.0 - s; }
            else {
                y = fa / fc; z = fb / fc;
                x = s * (2.0 * xm * y * (y - z) - (b - a) * (z - 1.0));
                y = (y - 1.0) * (z - 1.0) * (s - 1.0);
            }
            if (x > 0.0) y = -y;
            x = fabs(x);
            double m1 = 3.0 * xm * y - fabs(E_crit * y), m2 = fabs(e * y);
            if (2.0 * x < (m1 < m2 ? m1 : m2)) { e = d; d = x / y; }
            else { d = xm; e = d; }
        } else { d = xm; e = d; }
        a = b; fa = fb;
        if (fabs(d) > E_crit) b = b + d;
        else b = b + (xm >= 0.0 ? E_crit : -E_crit);
        fb = line_fn(w, q, pv, b, ql, phi, g);
    }
    return SIMOX_E_BRENT;
}

/* The whole CTIP_SOLVER. q in/out (original order). Returns status. */
int or_ctip(int n, const double box[3], double rcut, const int nc[3], int npt_max, int nnb_max,
            const int fft[3], int p, const simox_potential* P, const int* id, const double* x,
            double* q, const int* npt, const int* link, const int* pair, const double* psi,
            int max_cg, double* Eself_out, int* n_cg_out, long* n_eval_out, double* err_out)
{
    ctip_ws W; memset(&W, 0, sizeof(W));
    W.n = n; W.p = p; W.nnb_max = nnb_max; W.psi = psi;
    memcpy(W.fft, fft, sizeof(W.fft));
    int p3 = p * p * p, st = 0;
    size_t Ng = (size_t)fft[0] * fft[1] * fft[2];
    double a = 3.8 / rcut, V = box[0] * box[1] * box[2];
    double kc_const = KC * 2.0 * a / SQRTPI, rcut2 = rcut * rcut;
    int ncall = nc[0] * nc[1] * nc[2];
    W.XJZ = (double*)malloc(sizeof(double) * 3 * n);
    W.qmx = (double*)malloc(sizeof(double) * 2 * n);
    W.Qlocal = (double*)malloc(sizeof(double) * (size_t)n * p3);
    W.grid = (int*)malloc(sizeof(int) * (size_t)n * p3);
    W.asym = (double*)calloc((size_t)n * nnb_max, sizeof(double));
    W.sym = (double*)calloc((size_t)n * nnb_max, sizeof(double));
    W.list = (int*)calloc((size_t)n * nnb_max, sizeof(int));
    W.nlist = (int*)calloc(n, sizeof(int));
    W.Qbas = (double*)malloc(sizeof(double) * 2 * Ng);
    W.Qfin = (double*)malloc(sizeof(double) * 2 * Ng);
    double* qi = (double*)malloc(sizeof(double) * n);
    double* d = (double*)malloc(sizeof(double) * n);
    double* pv = (double*)calloc(n, sizeof(double));
    double* g = (double*)malloc(sizeof(double) * n);
    double* phi = (double*)malloc(sizeof(double) * n);
    double* ql = (double*)malloc(sizeof(double) * n);
    double* g2 = (double*)malloc(sizeof(double) * n);
    double* phi2 = (double*)malloc(sizeof(double) * n);
    if (!W.XJZ || !W.qmx || !W.Qlocal || !W.grid || !W.asym || !W.sym || !W.list || !W.nlist ||
        !W.Qbas || !W.Qfin || !qi || !d || !pv || !g || !phi || !ql || !g2 || !phi2) { st = SIMOX_E_NOMEM; goto done; }
    /* ctip.f90:33-59 */
    for (int i = 0; i < n; i++) {
        const simox_potn* pp = &P->param[id[i] - 1];
        qi[i] = q[i];
        W.XJZ[3 * i] = pp->chi; W.XJZ[3 * i + 1] = pp->J - kc_const; W.XJZ[3 * i + 2] = pp->Z;
        W.qmx[2 * i] = pp->qmin; W.qmx[2 * i + 1] = pp->qmax;
        double u[3], w[3][16], dw[3][16]; int ix[3][16];
        for (int dd = 0; dd < 3; dd++) {
            u[dd] = (double)fft[dd] * (x[3 * i + dd] + box[dd] * 0.5) / box[dd];
            bspline(p, u[dd], w[dd], dw[dd]);
            for (int s = 0; s < p; s++) ix[dd][s] = stencil_index(u[dd], s, p, fft[dd]);
        }
        int s = 0;
        for (int aa = 0; aa < p; aa++) for (int bb = 0; bb < p; bb++) for (int cc = 0; cc < p; cc++, s++) {
            W.grid[(size_t)i * p3 + s] = ix[0][aa] + fft[0] * (ix[1][bb] + fft[1] * ix[2][cc]);
            W.Qlocal[(size_t)i * p3 + s] = w[0][aa] * w[1][bb] * w[2][cc];
        }
    }
    W.c_pme = KC * (double)fft[0] * (double)fft[1] * (double)fft[2] / V / PI_;
    /* pair matrices ctip.f90:64-165 */
    for (int m = 0; m < ncall; m++) {
        const int* lk = link + (size_t)m * npt_max;
        int Nloc = npt[m];
        for (int pass = 0; pass < 14; pass++) {
            int cj = pass == 0 ? m : pair[m * 13 + pass - 1] - 1;
            const int* lkj = link + (size_t)cj * npt_max;
            int outer_n = pass == 0 ? Nloc - 1 : npt[cj];
            for (int oi = 0; oi < outer_n; oi++) {
                int inner_lo = pass == 0 ? oi + 1 : 0;
                for (int ii = inner_lo; ii < Nloc; ii++) {
                    int li, lj;
                    if (pass == 0) { li = lk[oi] - 1; lj = lk[ii] - 1; }
                    else           { lj = lkj[oi] - 1; li = lk[ii] - 1; }
                    double rx[3];
                    for (int dd = 0; dd < 3; dd++) {
                        double dx = x[3 * li + dd] - x[3 * lj + dd];
                        rx[dd] = dx - box[dd] * round(dx / box[dd]);
                    }
                    double r2 = rx[0] * rx[0] + rx[1] * rx[1] + rx[2] * rx[2];
                    if (!(r2 < rcut2)) continue;
                    double r = sqrt(r2), ar = a * r;
                    int id_i = id[li], id_j = id[lj];
                    double xi_i = P->param[id_i - 1].xi, xi_j = P->param[id_j - 1].xi;
                    double ej = exp(-2.0 * xi_j * r), ej_r = ej / r;
                    double afb_j = -xi_j * ej - ej_r, afb_i, fifj;
                    const double* fa = P->param[id_i - 1].fafb[id_j - 1];
                    if (id_i == id_j) {
                        afb_i = afb_j;
                        double xir = xi_i * r;
                        const double* fs = P->param[id_i - 1].fafb[id_i - 1];
                        fifj = -ej * (1.0 + xir * (fs[1] + xir * (fs[2] + xir * fs[3]))) / r;
                    } else {
                        double ei = exp(-2.0 * xi_i * r), ei_r = ei / r;
                        afb_i = -xi_i * ei - ei_r;
                        fifj = -ei * (fa[0] + fa[2] / r) - ej * (fa[1] + fa[3] / r);
                    }
                    W.nlist[li]++; W.nlist[lj]++;
                    if (W.nlist[li] > nnb_max || W.nlist[lj] > nnb_max) { st = SIMOX_E_NBR_OVERFLOW; goto done; }
                    size_t ki = (size_t)li * nnb_max + W.nlist[li] - 1;
                    size_t kj = (size_t)lj * nnb_max + W.nlist[lj] - 1;
                    W.list[ki] = lj; W.list[kj] = li;
                    W.asym[ki] = KC * (afb_i - fifj);
                    W.asym[kj] = KC * (afb_j - fifj);
                    double tmp = KC * (fifj + erfc(ar) / r);
                    W.sym[ki] = tmp; W.sym[kj] = tmp;
                }
            }
        }
    }
    /* CG loop ctip.f90:168-190 */
    {
        double Error = 1.0, g_sum = 1.0, g_sum_old, d_sum, alpha = 0.0;
        int k = 0;
        while (Error > 1.0e-3) {
            if (max_cg > 0 && k >= max_cg) { st = SIMOX_E_CG_LIMIT; break; }
            phi_mesh(&W, qi, phi);
            for (int i = 0; i < n; i++) phi[i] = phi[i] * W.c_pme;
            dudq(&W, qi, phi, g);
            g_sum_old = g_sum; g_sum = 0.0;
            for (int i = 0; i < n; i++) g_sum = g_sum + g[i];
            for (int i = 0; i < n; i++) d[i] = g[i] + pv[i] * g_sum / g_sum_old;
            d_sum = 0.0;
            for (int i = 0; i < n; i++) d_sum = d_sum + d[i];
            d_sum = d_sum / (double)n;
            for (int i = 0; i < n; i++) pv[i] = d[i] - d_sum;
            st = brent(&W, qi, pv, &alpha, ql, phi2, g2);
            if (st) break;
            for (int i = 0; i < n; i++) qi[i] = qi[i] + alpha * pv[i];
            double mx = 0.0;
            for (int i = 0; i < n; i++) if (fabs(pv[i]) > mx) mx = fabs(pv[i]);
            Error = mx * fabs(alpha);
            k++;
        }
        if (n_cg_out) *n_cg_out = k;
        if (err_out) *err_out = Error;
    }
    if (st == 0 || st == SIMOX_E_CG_LIMIT) {
        /* energies ctip.f90:194-209 */
        double Eself = 0.0, Esum = 0.0;
        for (int i = 0; i < n; i++) {
            q[i] = qi[i];
            Eself = Eself - q[i] * q[i];
            Esum = Esum + W.XJZ[3 * i] * qi[i] + 0.5 * W.XJZ[3 * i + 1] * (qi[i] * qi[i]);
            double dq = qi[i] - W.qmx[2 * i];
            if (dq < 0.0) Esum = Esum + WPEN * (dq * dq);
            dq = qi[i] - W.qmx[2 * i + 1];
            if (dq > 0.0) Esum = Esum + WPEN * (dq * dq);
        }
        *Eself_out = Eself * KC * a / SQRTPI + Esum;
    }
    if (n_eval_out) *n_eval_out = W.n_eval;
done:
    free(W.XJZ); free(W.qmx); free(W.Qlocal); free(W.grid); free(W.asym); free(W.sym);
    free(W.list); free(W.nlist); free(W.Qbas); free(W.Qfin);
    free(qi); free(d); free(pv); free(g); free(phi); free(ql); free(g2); free(phi2);
    return st;
}

/* ====================================================================== */
/* Integrators vverlet.f90                                                */
/* ====================================================================== */
/* VV_NVE1 vverlet.f90:74-96 */
void or_vv_nve1(int n, const double box[3], const simox_potential* P, const int* id,
                double* x, double* v, const double* f, double dt)
{
    for (int i = 0; i < n; i++) {
        double xm = P->param[id[i] - 1].xm;
        for (int d = 0; d < 3; d++) {
            v[3 * i + d] = v[3 * i + d] + 0.5 * dt * f[3 * i + d] / xm;
            double xx = x[3 * i + d] + dt * v[3 * i + d];
            x[3 * i + d] = xx - box[d] * round(xx / box[d]);
        }
    }
}

/* VV_NVE1_REFLECT vverlet.f90:100-129 */
void or_vv_nve1_reflect(int n, const double box[3], const simox_potential* P, const int* id,
                        double* x, double* v, const double* f, double dt)
{
    double box_z = box[2] / 2.0;
    for (int i = 0; i < n; i++) {
        double xm = P->param[id[i] - 1].xm, xx[3];
        for (int d = 0; d < 3; d++) {
            v[3 * i + d] = v[3 * i + d] + 0.5 * dt * f[3 * i + d] / xm;
            xx[d] = x[3 * i + d] + dt * v[3 * i + d];
        }
        for (int d = 0; d < 2; d++) x[3 * i + d] = xx[d] - box[d] * round(xx[d] / box[d]);
        if (xx[2] > box_z) { xx[2] = box[2] - xx[2]; v[3 * i + 2] = -fabs(v[3 * i + 2]); }
        x[3 * i + 2] = xx[2];
    }
}

/* VV_NVE2 vverlet.f90:132-157; returns mv2 */
double or_vv_nve2(int n, const simox_potential* P, const int* id, double* v, const double* f, double dt)
{
    double mv2 = 0.0;
    for (int i = 0; i < n; i++) {
        double xm = P->param[id[i] - 1].xm, t = 0.0;
        for (int d = 0; d < 3; d++) {
            v[3 * i + d] = v[3 * i + d] + 0.5 * dt * f[3 * i + d] / xm;
            t = t + v[3 * i + d] * v[3 * i + d];
        }
        mv2 = mv2 + xm * t;
    }
    return mv2;
}

/* VV_NVT2_BEREND vverlet.f90:160-208; returns mv2 */
double or_vv_nvt2_berend(int n, const simox_potential* P, const int* id, double* v, const double* f,
                         double dt, double T_given)
{
    double mv2_sum[SIMOX_NATOM] = {0}, lambda[SIMOX_NATOM] = {0};
    int Npt[SIMOX_NATOM] = {0};
    for (int i = 0; i < n; i++) {
        double xm = P->param[id[i] - 1].xm, t = 0.0;
        for (int d = 0; d < 3; d++) {
            v[3 * i + d] = v[3 * i + d] + 0.5 * dt * f[3 * i + d] / xm;
            t = t + xm * (v[3 * i + d] * v[3 * i + d]);
        }
        mv2_sum[id[i] - 1] += t;
        Npt[id[i] - 1]++;
    }
    for (int s = 0; s < SIMOX_NATOM; s++)
        if (Npt[s] > 0) {
            double T0 = mv2_sum[s] / (double)(3 * Npt[s]);
            lambda[s] = sqrt(1.0 + 0.025 * (T_given / T0 - 1.0));
        }
    double mv2 = 0.0;
    for (int i = 0; i < n; i++) {
        double xm = P->param[id[i] - 1].xm, t = 0.0;
        for (int d = 0; d < 3; d++) {
            v[3 * i + d] = v[3 * i + d] * lambda[id[i] - 1];
            t = t + xm * (v[3 * i + d] * v[3 * i + d]);
        }
        mv2 = mv2 + t;
    }
    return mv2;
}

/* ---------------------------------------------------------------------- */
/* Random numbers of VINIT and the stochastic thermostat.  The reference  */
/* draws from Fortran's RANDOM_NUMBER after RANDOM_SEED (main.f90:28),    */
/* which no other program can reproduce; both this oracle and the GPU     */
/* library use the same seeded counter-based generator instead: the       */
/* SplitMix64 output mix (Steele, Lea & Flood, OOPSLA 2014) applied to    */
/* (seed, stream a, counter b), 53 bits scaled into [0, 1).               */
/* ---------------------------------------------------------------------- */
static uint64_t or_mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

double or_rng_uniform(uint64_t seed, uint64_t a, uint64_t b)
{
    const uint64_t g = 0x9E3779B97F4A7C15ULL;
    uint64_t z = or_mix64(or_mix64(seed + g * (a + 1)) + g * (b + 1));
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

/* fluct (util.f90:84-101): Marsaglia's polar method, v1 kept.  The draw of
 * component d of atom i at step `step` uses stream (step << 32 | i) and
 * counters 2 (256 d + k) and 2 (256 d + k) + 1 for attempt k < 100; after 100
 * rejected attempts (probability (1 - pi/4)^100) it returns 0 and sets *bad. */
double or_fluct(uint64_t seed, uint64_t step, int i, int d, double x, int* bad)
{
    const uint64_t a = (step << 32) | (uint64_t)(uint32_t)i;
    for (int k = 0; k < 100; k++) {
        const uint64_t b = 2 * (uint64_t)(256 * d + k);
        double v1 = 2.0 * or_rng_uniform(seed, a, b) - 1.0;
        double v2 = 2.0 * or_rng_uniform(seed, a, b + 1) - 1.0;
        double r = v1 * v1 + v2 * v2;
        if (r < 1.0 && r > 0.0) return v1 * sqrt(-2.0 * log(r) / r) * x;
    }
    *bad = 1;
    return 0.0;
}

/* VINIT velocities (vverlet.f90:19-55; VINIT is vverlet.f90:2-71): uniform in [-0.5, 0.5) from stream
 * (1 << 62 | i), counter d; the mean removed; scaled per species to T_given.
 * Returns the as-written mv2 of vverlet.f90:64-69, which multiplies every
 * atom's v^2 by the mass left in xm by the previous loop (the last atom's). */
double or_vinit_velocities(int n, const simox_potential* P, const int* id, double* v, uint64_t seed,
                           double T_given)
{
    double sumv[3] = {0.0, 0.0, 0.0}, mv2[SIMOX_NATOM] = {0}, lambda[SIMOX_NATOM] = {0};
    int Npt[SIMOX_NATOM] = {0};
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) {
            v[3 * i + d] = or_rng_uniform(seed, (1ULL << 62) | (uint64_t)(uint32_t)i, (uint64_t)d) - 0.5;
            sumv[d] = sumv[d] + v[3 * i + d];
        }
    for (int d = 0; d < 3; d++) sumv[d] = sumv[d] / (double)n;
    double xm = 0.0;
    for (int i = 0; i < n; i++) {
        for (int d = 0; d < 3; d++) v[3 * i + d] = v[3 * i + d] - sumv[d];
        xm = P->param[id[i] - 1].xm;
        mv2[id[i] - 1] += xm * (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
        Npt[id[i] - 1]++;
    }
    for (int s = 0; s < SIMOX_NATOM; s++)
        if (Npt[s] > 0) {
            double T0 = mv2[s] / (double)(Npt[s] * 3);
            lambda[s] = sqrt(T_given / T0);
        }
    double out = 0.0;
    for (int i = 0; i < n; i++) {
        for (int d = 0; d < 3; d++) v[3 * i + d] = v[3 * i + d] * lambda[id[i] - 1];
        out = out + xm * (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
    }
    return out;
}

/* VV_NVT1_STOCH vverlet.f90:237-260 */
void or_vv_nvt1_stoch(int n, const double box[3], const simox_potential* P, const int* id,
                      double* x, double* v, const double* f, double dt, double alpha)
{
    for (int i = 0; i < n; i++) {
        double xm = P->param[id[i] - 1].xm;
        for (int d = 0; d < 3; d++) {
            v[3 * i + d] = v[3 * i + d] * (1.0 - 0.5 * alpha * dt / xm) + 0.5 * dt * f[3 * i + d] / xm;
            double xx = x[3 * i + d] + dt * v[3 * i + d];
            x[3 * i + d] = xx - box[d] * round(xx / box[d]);
        }
    }
}

/* VV_NVT2_STOCH vverlet.f90:263-296 (sigma 1): f gains the random force;
 * returns mv2, *bad as or_fluct */
double or_vv_nvt2_stoch(int n, const simox_potential* P, const int* id, double* v, double* f, double dt,
                        double alpha, double T_given, uint64_t seed, uint64_t step, int* bad)
{
    double beta = sqrt(2.0 * alpha * T_given / dt), mv2 = 0.0;
    for (int i = 0; i < n; i++) {
        double xm = P->param[id[i] - 1].xm, t = 0.0;
        for (int d = 0; d < 3; d++) {
            double eta = or_fluct(seed, step, i, d, 1.0, bad);
            f[3 * i + d] = f[3 * i + d] + eta * beta;
            v[3 * i + d] = (v[3 * i + d] + 0.5 * dt * f[3 * i + d] / xm) / (1.0 + 0.5 * alpha * dt / xm);
            t = t + xm * (v[3 * i + d] * v[3 * i + d]);
        }
        mv2 = mv2 + t;
    }
    return mv2;
}

/* ====================================================================== */
/* Oxidation-mode host steps (main.f90:62-84)                             */
/* ====================================================================== */
/* REMOVE_RIGID_MOTION vverlet.f90:211-234 */
void or_remove_rigid_motion(int n, double* x, double* v)
{
    double sumv[3] = {0.0, 0.0, 0.0}, avg_z = 0.0;
    if (n <= 0) return;
    for (int i = 0; i < n; i++) {
        for (int d = 0; d < 3; d++) sumv[d] = sumv[d] + v[3 * i + d];
        avg_z = avg_z + x[3 * i + 2];
    }
    for (int d = 0; d < 3; d++) sumv[d] = sumv[d] / (double)n;
    avg_z = avg_z / (double)n;
    for (int i = 0; i < n; i++) {
        for (int d = 0; d < 3; d++) v[3 * i + d] = v[3 * i + d] - sumv[d];
        x[3 * i + 2] = x[3 * i + 2] - avg_z;
    }
}

/* OXIDE_CHECK util.f90:152-188; returns 1 when a new dimer is due */
int or_oxide_check(int n, const int* id, const double* x, const double* q, int n_o2, double q_crit)
{
    double m_height = 0.0, o_height = 0.0, q_max = -10.0;
    for (int i = 0; i < n; i++)
        if (id[i] == 1) m_height = fmax(x[3 * i + 2], m_height);
    for (int i = n - 1; i >= n - 2 * n_o2 && i >= 0; i--)
        if (id[i] == 4) {
            o_height = fmax(x[3 * i + 2], o_height);
            q_max = fmax(q[i], q_max);
        }
    return ((m_height + 0.0) > o_height || q_max < q_crit) ? 1 : 0;
}

/* RANDOM_POSITION_O2 util.f90:104-148 with the seeded draws of stream
 * (1 << 63 | event), counter = draw number in the reference's order.
 * Returns 0, or -1 for "=== Too many new oxygens ===" / no room. */
int or_random_position_o2(int n_o, double z_new, double Lx, double Ly, uint64_t seed, uint64_t event,
                          double* xx)
{
    const double L0 = 2.0;
    int n_o2 = n_o / 2;
    if (n_o2 <= 0) return 0;
    double Rcut = sqrt(Lx * Ly / (double)n_o2) * 0.5;
    if (Rcut < L0) return -1;
    double Rcut2 = Rcut * Rcut;
    uint64_t a = (1ULL << 63) | event, k = 0;
    double* cx = (double*)calloc((size_t)n_o2 * 3, sizeof(double));
    if (!cx) return -1;
    cx[0] = (or_rng_uniform(seed, a, k++) - 0.5) * Lx;
    cx[1] = (or_rng_uniform(seed, a, k++) - 0.5) * Ly;
    for (int i = 1; i < n_o2; i++) {
        int placed = 0;
        for (int t = 0; t < 100000 && !placed; t++) {
            cx[3 * i] = (or_rng_uniform(seed, a, k++) - 0.5) * Lx;
            cx[3 * i + 1] = (or_rng_uniform(seed, a, k++) - 0.5) * Ly;
            placed = 1;
            for (int j = 0; j < i; j++) {
                double dx = cx[3 * i] - cx[3 * j], dy = cx[3 * i + 1] - cx[3 * j + 1];
                double r2 = dx * dx + dy * dy;
                if (r2 < Rcut2) placed = 0;
            }
        }
        if (!placed) { free(cx); return -1; }
    }
    for (int i = 0; i < n_o2; i++) cx[3 * i + 2] = z_new;
    for (int i = 0; i < n_o2; i++) {
        double phi = or_rng_uniform(seed, a, k++) * M_PI * 2.0;
        double theta = or_rng_uniform(seed, a, k++) * M_PI;
        double d[3] = {L0 * sin(theta) * cos(phi), L0 * sin(theta) * cos(phi), L0 * cos(theta)};
        for (int c = 0; c < 3; c++) {
            xx[3 * (2 * i) + c] = d[c] + cx[3 * i + c];
            xx[3 * (2 * i + 1) + c] = -d[c] + cx[3 * i + c];
        }
    }
    free(cx);
    return 0;
}
