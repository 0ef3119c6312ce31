/*
 * mopac_oracle.c -- CPU FP64 restatement of MOPAC's PM7 sp-basis SCF path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle the CUDA product is
 * checked against.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it.  The product
 * library (mopac_gpu_b200) never links or calls it.
 *
 * It restates, in plain C, the reference's algorithms for the elements the
 * benchmark workloads use (H, C, O under PM7; sp basis, no d shells):
 *   parameters     models/parameters_for_PM7_C.F90 (H :24, C :91, O :127,
 *                  v_par7 :1392-1395, alpb/xfac :1405-1483), symmetrised as in
 *                  models/switch.F90:647-651
 *   derived params models/calpar.F90 (dd, qq, am, ad, aq, eisol) and
 *                  integrals/mndod.F90:25-59 (inid: po, ddp)
 *   overlaps       integrals/h1elec.F90, diat.F90 (diat, diat2), set.F90
 *                  (set, aintgs, bintgs), coe.F90
 *   2-e integrals  integrals/rotate.F90 -> mndod.F90 rotatd :1096, rotmat
 *                  :1382, reppd :426, reppd2 :846 (sp part), spcore :1683,
 *                  tx :1870, w2mat :1992, wstore :2027, elenuc :2367,
 *                  to_point :3462 (l_feather is on for PM7, readmo.F90:783)
 *   core-core      integrals/ccrep.F90 (PM7 branch)
 *   H and W        integrals/hcore.F90 (loop order and W layout)
 *   Fock build     SCF/fock2.F90 (sp branches), integrals/jab.F90, kab.F90,
 *                  SCF/fock1.F90
 *   energy         integrals/helect.F90
 *   extrapolation  SCF/cnvg.F90
 *   guess          moldat.F90:731-760 (pdiag)
 *   heats          interface/mopac_api_initialize.F90:340-350 (atheat),
 *                  corrections/H_bond_correction_PM6_DH_Dispersion.F90
 *                  (PM7 dispersion), bond counting after
 *                  corrections/set_up_dentate.F90:36-80
 * Summation orders of fock2/jab/kab/fock1/helect are kept term by term; the
 * file is compiled with -ffp-contract=off so no FMA is introduced.
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define A0 0.529177210903
#define EV 27.211386245988
#define FPC9 23.060547830619029
#define TRUNC1 7.0
#define TRUNC2 0.22

/* ------------------------------------------------------------------ */
/* Element parameters (PM7).  Index by atomic number; only 1, 6, 8.    */
/* ------------------------------------------------------------------ */
typedef struct {
  int natorb, ios, iop, npq;
  double tore, uss, upp, betas, betap, zs, zp, gss, gsp, gpp, gp2, hsp;
  double g1, g2, g3; /* first PM7 Gaussian (guess1/2/3(:,1)) */
  double eheat;
  /* derived */
  double dd, qq, am, ad, aq, eisol;
  double po1, po2, po3, po7, po9, ddp2, ddp3;
} elem_t;

static elem_t E[9];
static double XFAC[9][9], ALPB[9][9];
static const double PAR1 = 8.947612, PAR2 = 6.024265, PAR3 = -0.012037, PAR4 = 0.701333;
static int params_ready = 0;

static void set_elem(int z, int natorb, int ios, int iop, int npq, double tore,
                     double uss, double upp, double betas, double betap,
                     double zs, double zp, double gss, double gsp, double gpp,
                     double gp2, double hsp, double g1, double g2, double g3,
                     double eheat) {
  elem_t *e = &E[z];
  memset(e, 0, sizeof(*e));
  e->natorb = natorb; e->ios = ios; e->iop = iop; e->npq = npq; e->tore = tore;
  e->uss = uss; e->upp = upp; e->betas = betas; e->betap = betap;
  e->zs = zs; e->zp = zp; e->gss = gss; e->gsp = gsp; e->gpp = gpp;
  e->gp2 = gp2; e->hsp = hsp; e->g1 = g1; e->g2 = g2; e->g3 = g3;
  e->eheat = eheat;
}

/* calpar.F90:49-150 for one sp element (qn = principal quantum number). */
static void calpar_sp(int z) {
  elem_t *e = &E[z];
  const double p4 = 16.0; /* p = 2, p4 = p**4 */
  if (z == 1) {
    /* calpar.F90:152-158: hydrogen overrides */
    e->eisol = e->uss;
    e->am = e->gss / EV;
    e->ad = e->am;
    e->aq = e->am;
    return;
  }
  double gssc = (double)(e->ios - 1 > 0 ? e->ios - 1 : 0);
  int k = e->iop;
  double gspc = (double)(e->ios * k);
  int l = k < 6 - k ? k : 6 - k;
  double gp2c = (double)((k * (k - 1)) / 2) + 0.5 * (double)(l * (l - 1)) / 2.0;
  double gppc = -0.5 * (double)(l * (l - 1)) / 2.0;
  double hspc = -(double)k * (double)e->ios * 0.5;
  e->zp = fmax(0.3, e->zp);
  double hpp = 0.5 * (e->gpp - e->gp2);
  hpp = fmax(0.1, hpp);
  e->hsp = fmax(1.0e-7, e->hsp);
  e->eisol = e->uss * e->ios + e->upp * e->iop + e->gss * gssc + e->gpp * gppc +
             e->gsp * gspc + e->gp2 * gp2c + e->hsp * hspc;
  double qn = (double)e->npq;
  e->dd = (2.0 * qn + 1) * pow(4.0 * e->zs * e->zp, qn + 0.5) /
          pow(e->zs + e->zp, 2.0 * qn + 2) / sqrt(3.0);
  e->qq = sqrt((4.0 * qn * qn + 6.0 * qn + 2.0) / 20.0) / e->zp;
  /* secant solve for ad (calpar.F90:116-126) */
  double gdd1 = pow(e->hsp / (EV * e->dd * e->dd), 1.0 / 3.0);
  double d1 = gdd1, d2 = gdd1 + 0.04;
  for (int j = 0; j < 5; ++j) {
    double df = d2 - d1;
    double hsp1 = 0.5 * d1 - 0.5 / sqrt(4.0 * e->dd * e->dd + 1.0 / (d1 * d1));
    double hsp2 = 0.5 * d2 - 0.5 / sqrt(4.0 * e->dd * e->dd + 1.0 / (d2 * d2));
    if (fabs(hsp2 - hsp1) < 1.0e-25) break;
    double d3 = d1 + df * (e->hsp / EV - hsp1) / (hsp2 - hsp1);
    d1 = d2;
    d2 = d3;
  }
  double gqq = pow(p4 * hpp / (EV * 48.0 * pow(e->qq, 4)), 0.2);
  double q1 = gqq, q2 = gqq + 0.04;
  for (int j = 0; j < 5; ++j) {
    double qf = q2 - q1;
    double hpp1 = 0.25 * q1 - 0.5 / sqrt(4.0 * e->qq * e->qq + 1.0 / (q1 * q1)) +
                  0.25 / sqrt(8.0 * e->qq * e->qq + 1.0 / (q1 * q1));
    double hpp2 = 0.25 * q2 - 0.5 / sqrt(4.0 * e->qq * e->qq + 1.0 / (q2 * q2)) +
                  0.25 / sqrt(8.0 * e->qq * e->qq + 1.0 / (q2 * q2));
    if (fabs(hpp2 - hpp1) < 1.0e-25) break;
    double q3 = q1 + qf * (hpp / EV - hpp1) / (hpp2 - hpp1);
    q1 = q2;
    q2 = q3;
  }
  e->am = e->gss / EV;
  e->ad = d2;
  e->aq = q2;
}

/* inid (mndod.F90:25-59): multipole additive terms. */
static void inid_sp(int z) {
  elem_t *e = &E[z];
  e->po1 = 0.5 / e->am;
  e->po2 = e->ad > 1.0e-5 ? 0.5 / e->ad : 0.0;
  e->po3 = e->aq > 1.0e-5 ? 0.5 / e->aq : 0.0;
  e->po7 = e->po1;
  e->ddp2 = e->dd;
  e->ddp3 = e->qq * sqrt(2.0);
  e->po9 = e->po1; /* pocord is zero for H, C, O in PM7 */
  if (z == 1) { e->po2 = 0.0; e->po3 = 0.0; }
}

static void init_params(void) {
  if (params_ready) return;
  memset(E, 0, sizeof(E));
  /*           Z  norb ios iop npq tore   uss          upp          betas        betap       zs        zp        gss        gsp        gpp        gp2       hsp       gues1      gues2     gues3     eheat */
  set_elem(1, 1, 1, 0, 1, 1.0, -11.070112, 0.0, -8.389745, 0.0, 1.260237, 0.0, 14.149656, 0.0, 0.0, 0.0, 0.0, 0.177854, 1.428710, 0.991324, 52.102);
  set_elem(6, 4, 2, 2, 2, 4.0, -51.372620, -40.135421, -14.414930, -7.893717, 1.942244, 1.708723, 12.347323, 11.932801, 10.452226, 9.385498, 0.802634, 0.045888, 5.037055, 1.588715, 170.890);
  set_elem(8, 4, 2, 4, 2, 6.0, -96.087736, -71.087738, -67.776339, -20.267981, 5.972309, 2.349017, 14.955121, 16.088521, 12.403337, 10.499706, 5.028656, -0.016243, 1.871970, 1.844360, 59.559);
  const int zs_[3] = {1, 6, 8};
  for (int i = 0; i < 3; ++i) { calpar_sp(zs_[i]); inid_sp(zs_[i]); }
  memset(XFAC, 0, sizeof(XFAC));
  memset(ALPB, 0, sizeof(ALPB));
  ALPB[1][1] = 4.051163; XFAC[1][1] = 2.845627;
  ALPB[6][1] = 1.038716; XFAC[6][1] = 0.204582;
  ALPB[6][6] = 2.655746; XFAC[6][6] = 0.937818;
  ALPB[8][1] = 1.508030; XFAC[8][1] = 0.160602;
  ALPB[8][6] = 2.850931; XFAC[8][6] = 0.826848;
  ALPB[8][8] = 2.457135; XFAC[8][8] = 0.356439;
  for (int i = 1; i <= 8; ++i)
    for (int j = 1; j < i; ++j) { XFAC[j][i] = XFAC[i][j]; ALPB[j][i] = ALPB[i][j]; }
  params_ready = 1;
}

static int supported(int z) { return z == 1 || z == 6 || z == 8; }

/* ------------------------------------------------------------------ */
/* Overlap integrals: diat2 / set / aintgs / bintgs / coe / diat      */
/* ------------------------------------------------------------------ */
static const double FACT[18] = {1.0, 1.0, 2.0, 6.0, 24.0, 120.0, 720.0, 5040.0, 40320.0,
                                362880.0, 3628800.0, 39916800.0, 479001600.0,
                                6227020800.0, 87178291200.0, 1307674368000.0,
                                20922789888000.0, 355687428096000.0};

typedef struct { double a[16], b[16], sa, sb; int isp, ips; } ovl_t;

static double ipow(double x, int m) { /* x**m with integer m */
  double r = 1.0;
  for (int i = 0; i < m; ++i) r *= x;
  return r;
}

static void aintgs(ovl_t *o, double x, int k) {
  double c = exp(-x);
  o->a[1] = c / x;
  for (int i = 1; i <= k; ++i) o->a[i + 1] = (o->a[i] * i + c) / x;
}

static void bintgs(ovl_t *o, double x, int k) {
  double absx = fabs(x);
  int last = 0, mode = 0; /* 0: recursion, 1: series, 2: tiny */
  if (absx > 3.0) mode = 0;
  else if (absx > 2.0) { if (k <= 10) mode = 0; else { last = 15; mode = 1; } }
  else if (absx > 1.0) { if (k <= 7) mode = 0; else { last = 12; mode = 1; } }
  else if (absx > 0.5) { if (k <= 5) mode = 0; else { last = 7; mode = 1; } }
  else if (absx <= 1.0e-6) mode = 2;
  else { last = 6; mode = 1; }
  if (mode == 0) {
    double expx = exp(x), expmx = 1.0 / expx;
    o->b[1] = (expx - expmx) / x;
    for (int i = 1; i <= k; ++i)
      o->b[i + 1] = (i * o->b[i] + ((i & 1) ? -1.0 : 1.0) * expx - expmx) / x;
  } else if (mode == 1) {
    for (int i = 0; i <= k; ++i) {
      double y = 0.0;
      for (int m = 0; m <= last; ++m) {
        double xf = 1.0;
        if (m != 0) xf = FACT[m];
        y = y + ipow(-x, m) * (double)(2 * ((m + i + 1) % 2)) / (xf * (double)(m + i + 1));
      }
      o->b[i + 1] = y;
    }
  } else {
    for (int i = 0; i <= k; ++i) o->b[i + 1] = (double)(2 * ((i + 1) % 2)) / (i + 1.0);
  }
}

static void set_ovl(ovl_t *o, double s1, double s2, int na, int nb, double rab, int ii) {
  if (na <= nb) { o->isp = 1; o->ips = 2; o->sa = s1; o->sb = s2; }
  else { o->isp = 2; o->ips = 1; o->sa = s2; o->sb = s1; }
  int j = ii + 2;
  if (ii > 3) j = j - 1;
  double alpha = 0.5 * rab * (o->sa + o->sb);
  double beta = 0.5 * rab * (o->sb - o->sa);
  aintgs(o, alpha, j - 1);
  bintgs(o, beta, j - 1);
}

/* diat2 (diat.F90:211-): s[la][lb][m], 1-based la/lb/m in 1..3 */
static void diat2(int na, double esa, double epa, double r12, int nb, double esb,
                  double epb, double s[4][4][4]) {
  static const int inmb[18] = {0, 1, 0, 2, 2, 3, 4, 5, 6, 7, 0, 8, 8, 8, 9, 10, 11, 12};
  static const int iii[79] = {0, 1, 2, 4, 2, 4, 4, 2, 4, 4, 4, 2, 4, 4, 4, 4, 2, 4, 4, 4, 4, 4,
                              2, 4, 4, 4, 4, 4, 4, 3, 5, 5, 5, 5, 5, 5, 6, 3, 5, 5, 5, 5, 5, 5, 6, 6,
                              3, 5, 5, 5, 5, 5, 5, 6, 6, 6, 3, 5, 5, 5, 5, 5, 5, 6, 6, 6, 6, 3, 5,
                              5, 5, 5, 5, 5, 6, 6, 6, 6, 6};
  int jmax = inmb[na] > inmb[nb] ? inmb[na] : inmb[nb];
  int jmin = inmb[na] < inmb[nb] ? inmb[na] : inmb[nb];
  int nbond = (jmax * (jmax - 1)) / 2 + jmin;
  int ii = iii[nbond];
  memset(s, 0, sizeof(double) * 64);
  double rab = r12 / A0;
  ovl_t o;
  const double *a = o.a, *b = o.b;
  if (ii == 2) {
    set_ovl(&o, esa, esb, na, nb, rab, ii);
    double rab4 = ipow(rab, 4) * 0.125;
    double w = sqrt(ipow(o.sa, 3) * ipow(o.sb, 5)) * rab4;
    double t = sqrt(1.0 / 3.0);
    s[1][1][1] = w * t * (a[4] * b[1] - b[4] * a[1] + a[3] * b[2] - b[3] * a[2]);
    if (na > 1) set_ovl(&o, epa, esb, na, nb, rab, ii);
    if (nb > 1) set_ovl(&o, esa, epb, na, nb, rab, ii);
    w = sqrt(ipow(o.sa, 3) * ipow(o.sb, 5)) * rab4;
    s[o.isp][o.ips][1] = w * (a[3] * b[1] - b[3] * a[1] + a[4] * b[2] - b[4] * a[2]);
  } else if (ii == 4) {
    set_ovl(&o, esa, esb, na, nb, rab, ii);
    double rab4 = ipow(rab, 5) * 0.0625;
    double w = sqrt(ipow(o.sa * o.sb, 5)) * rab4;
    s[1][1][1] = w * (a[5] * b[1] + b[5] * a[1] - 2.0 * a[3] * b[3]) / 3.0;
    set_ovl(&o, esa, epb, na, nb, rab, ii);
    if (na > nb) set_ovl(&o, epa, esb, na, nb, rab, ii);
    w = sqrt(ipow(o.sa * o.sb, 5)) * rab4;
    double rt3 = 1.0 / sqrt(3.0);
    double d = a[4] * (b[1] - b[3]) - a[2] * (b[3] - b[5]);
    double e = b[4] * (a[1] - a[3]) - b[2] * (a[3] - a[5]);
    s[o.isp][o.ips][1] = w * rt3 * (d + e);
    set_ovl(&o, epa, esb, na, nb, rab, ii);
    if (na > nb) set_ovl(&o, esa, epb, na, nb, rab, ii);
    w = sqrt(ipow(o.sa * o.sb, 5)) * rab4;
    d = a[4] * (b[1] - b[3]) - a[2] * (b[3] - b[5]);
    e = b[4] * (a[1] - a[3]) - b[2] * (a[3] - a[5]);
    s[o.ips][o.isp][1] = w * rt3 * (d - e);
    set_ovl(&o, epa, epb, na, nb, rab, ii);
    w = sqrt(ipow(o.sa * o.sb, 5)) * rab4;
    s[2][2][1] = -w * (b[3] * (a[5] + a[1]) - a[3] * (b[5] + b[1]));
    s[2][2][2] = 0.5 * w * (a[5] * (b[1] - b[3]) - b[5] * (a[1] - a[3]) - a[3] * b[1] + b[3] * a[1]);
  } else { /* ii == 1: s-s between first-row atoms */
    set_ovl(&o, esa, esb, na, nb, rab, ii);
    s[1][1][1] = 0.25 * sqrt(ipow(o.sa * o.sb * rab * rab, 3)) * (a[3] * b[1] - b[3] * a[1]);
  }
}

/* diat (diat.F90:16-) for sp atoms: di[i][j], 1-based orbital indices
 * (1 = s, 2 = px, 3 = py, 4 = pz).  xj = coord(j) - coord(i). */
static void diat(int ni, int nj, const double xj[3], double di[5][5], double cutof1) {
  memset(di, 0, sizeof(double) * 25);
  double x2 = xj[0], y2 = xj[1], z2 = xj[2];
  double rr = x2 * x2 + y2 * y2 + z2 * z2;
  if (rr >= cutof1) return;
  /* coe (coe.F90): direction cosines of the pair axis */
  double xy = x2 * x2 + y2 * y2;
  double r = sqrt(xy + z2 * z2);
  xy = sqrt(xy);
  double ca, cb, sa, sb;
  if (xy >= 1.0e-10) { ca = x2 / xy; cb = z2 / r; sa = y2 / xy; sb = xy / r; }
  else if (z2 < 0.0) { ca = -1.0; cb = -1.0; sa = 0.0; sb = 0.0; }
  else if (z2 == 0.0) { ca = 0.0; cb = 0.0; sa = 0.0; sb = 0.0; }
  else { ca = 1.0; cb = 1.0; sa = 0.0; sb = 0.0; }
  /* c[L][slot][m], L 1..2, slot 1..5, m 1..5 */
  double c[3][6][6];
  memset(c, 0, sizeof(c));
  c[1][3][3] = 1.0;
  int nij = E[ni].natorb > E[nj].natorb ? E[ni].natorb : E[nj].natorb;
  if (nij >= 2) {
    c[2][4][4] = ca * cb;  c[2][4][3] = ca * sb;  c[2][4][2] = -sa;
    c[2][3][4] = -sb;      c[2][3][3] = cb;       c[2][3][2] = 0.0;
    c[2][2][4] = sa * cb;  c[2][2][3] = sa * sb;  c[2][2][2] = ca;
  }
  if (r < 0.001) return;
  int ia = E[ni].npq + 1 < 3 ? E[ni].npq + 1 : 3;
  int ib = E[nj].npq + 1 < 3 ? E[nj].npq + 1 : 3;
  double s[4][4][4];
  diat2(ni, E[ni].zs, E[ni].zp, r, nj, E[nj].zs, E[nj].zp, s);
  /* ival(L, slot) -> orbital index (1-based), 0 = none */
  static const int ival[3][6] = {{0, 0, 0, 0, 0, 0}, {0, 1, 1, 1, 1, 0}, {0, 0, 3, 4, 2, 0}};
  if (ia > 2) ia = 2; /* sp only: the d slot carries no orbital */
  if (ib > 2) ib = 2;
  for (int i = 1; i <= ia; ++i) {
    int kmin = 4 - i, kmax = 2 + i;
    for (int j = 1; j <= ib; ++j) {
      double aa, bb;
      if (j == 2) { aa = -1.0; bb = 1.0; }
      else { aa = 1.0; bb = (j == 3) ? -1.0 : 1.0; }
      int lmin = 4 - j, lmax = 2 + j;
      for (int k = kmin; k <= kmax; ++k)
        for (int l = lmin; l <= lmax; ++l) {
          int ii = ival[i][k], jj = ival[j][l];
          if (ii == 0 || jj == 0) continue;
          di[ii][jj] = s[i][j][1] * (c[i][k][3] * c[j][l][3]) * aa +
                       s[i][j][2] * (c[i][k][4] * c[j][l][4] + c[i][k][2] * c[j][l][2]) * bb +
                       s[i][j][3] * (c[i][k][5] * c[j][l][5] + c[i][k][1] * c[j][l][1]);
        }
    }
  }
}

/* h1elec.F90: resonance integrals <i|H|j> = S(i,j) * (beta_i + beta_j)/2 */
static void h1elec(int ni, int nj, const double *xi, const double *xj, double di[5][5], double cutof1) {
  double rab = (xi[0] - xj[0]) * (xi[0] - xj[0]) + (xi[1] - xj[1]) * (xi[1] - xj[1]) +
               (xi[2] - xj[2]) * (xi[2] - xj[2]);
  if (rab > 1.0e4) { memset(di, 0, sizeof(double) * 25); return; }
  double xjuc[3] = {xj[0] - xi[0], xj[1] - xi[1], xj[2] - xi[2]};
  diat(ni, nj, xjuc, di, cutof1);
  double bi[5], bj[5];
  bi[1] = E[ni].betas * 0.5; bi[2] = bi[3] = bi[4] = E[ni].betap * 0.5;
  bj[1] = E[nj].betas * 0.5; bj[2] = bj[3] = bj[4] = E[nj].betap * 0.5;
  for (int j = 1; j <= E[nj].natorb; ++j)
    for (int i = 1; i <= E[ni].natorb; ++i) di[i][j] = di[i][j] * (bi[i] + bj[j]);
}

/* ------------------------------------------------------------------ */
/* Two-centre integrals: rotmat / reppd / spcore / tx / rotatd         */
/* ------------------------------------------------------------------ */
static void to_point(double r, double *point, double *cst) {
  *point = EV * A0 / r;
  if (r < TRUNC1) *cst = 1.0 - exp(-(r - TRUNC1) * (r - TRUNC1) * TRUNC2);
  else *cst = 0.0;
}

/* reppd (mndod.F90:426-843), sp part, l_feather on. */
static void reppd(int ni, int nj, double rij, double ri[23], double *gab) {
  static const int nri[23] = {0, 1, -1, 1, 1, -1, 1, 1, -1, -1, -1, 1, 1, -1, -1, -1, 1, 1, 1, 1, 1, 1, 1};
  const double td = 2.0, pp = 0.5;
  double ev1 = EV / 2, ev2 = ev1 / 2, ev3 = ev2 / 2, ev4 = ev3 / 2;
  for (int i = 0; i < 23; ++i) ri[i] = 0.0;
  double r = rij / A0;
  int si = E[ni].natorb >= 3, sj = E[nj].natorb >= 3;
  double aee = E[ni].po9 + E[nj].po9;
  aee = aee * aee;
  *gab = EV / sqrt(r * r + aee);
  aee = pp / E[ni].am + pp / E[nj].am;
  aee = aee * aee;
  double arg[73], sqr[73];
  if (!si && !sj) {
    ri[1] = EV / sqrt(r * r + aee);
  } else if (si && !sj) {
    double da = E[ni].dd, qa = E[ni].qq * td;
    double ade = pp / E[ni].ad + pp / E[nj].am; ade = ade * ade;
    double aqe = pp / E[ni].aq + pp / E[nj].am; aqe = aqe * aqe;
    double rsq = r * r, xxx;
    arg[1] = rsq + aee;
    xxx = r + da; arg[2] = xxx * xxx + ade;
    xxx = r - da; arg[3] = xxx * xxx + ade;
    xxx = r + qa; arg[4] = xxx * xxx + aqe;
    xxx = r - qa; arg[5] = xxx * xxx + aqe;
    arg[6] = rsq + aqe;
    arg[7] = arg[6] + qa * qa;
    for (int i = 1; i <= 7; ++i) sqr[i] = sqrt(arg[i]);
    double ee = EV / sqr[1];
    ri[1] = ee;
    ri[2] = ev1 / sqr[2] - ev1 / sqr[3];
    ri[3] = ee + ev2 / sqr[4] + ev2 / sqr[5] - ev1 / sqr[6];
    ri[4] = ee + ev1 / sqr[7] - ev1 / sqr[6];
  } else if (!si && sj) {
    double db = E[nj].dd, qb = E[nj].qq * td;
    double aed = pp / E[ni].am + pp / E[nj].ad; aed = aed * aed;
    double aeq = pp / E[ni].am + pp / E[nj].aq; aeq = aeq * aeq;
    double rsq = r * r, xxx;
    arg[1] = rsq + aee;
    xxx = r - db; arg[2] = xxx * xxx + aed;
    xxx = r + db; arg[3] = xxx * xxx + aed;
    xxx = r - qb; arg[4] = xxx * xxx + aeq;
    xxx = r + qb; arg[5] = xxx * xxx + aeq;
    arg[6] = rsq + aeq;
    arg[7] = arg[6] + qb * qb;
    for (int i = 1; i <= 7; ++i) sqr[i] = sqrt(arg[i]);
    double ee = EV / sqr[1];
    ri[1] = ee;
    ri[5] = ev1 / sqr[2] - ev1 / sqr[3];
    ri[11] = ee + ev2 / sqr[4] + ev2 / sqr[5] - ev1 / sqr[6];
    ri[12] = ee + ev1 / sqr[7] - ev1 / sqr[6];
  } else {
    double da = E[ni].dd, db = E[nj].dd, qa = E[ni].qq * td, qb = E[nj].qq * td;
    double ade = pp / E[ni].ad + pp / E[nj].am; ade *= ade;
    double aqe = pp / E[ni].aq + pp / E[nj].am; aqe *= aqe;
    double aed = pp / E[ni].am + pp / E[nj].ad; aed *= aed;
    double aeq = pp / E[ni].am + pp / E[nj].aq; aeq *= aeq;
    double axx = pp / E[ni].ad + pp / E[nj].ad; axx *= axx;
    double adq = pp / E[ni].ad + pp / E[nj].aq; adq *= adq;
    double aqd = pp / E[ni].aq + pp / E[nj].ad; aqd *= aqd;
    double aqq = pp / E[ni].aq + pp / E[nj].aq; aqq *= aqq;
    double rsq = r * r, xxx, yyy, zzz, www;
    arg[1] = rsq + aee;
    xxx = r + da; arg[2] = xxx * xxx + ade;
    xxx = r - da; arg[3] = xxx * xxx + ade;
    xxx = r - qa; arg[4] = xxx * xxx + aqe;
    xxx = r + qa; arg[5] = xxx * xxx + aqe;
    arg[6] = rsq + aqe;
    arg[7] = arg[6] + qa * qa;
    xxx = r - db; arg[8] = xxx * xxx + aed;
    xxx = r + db; arg[9] = xxx * xxx + aed;
    xxx = r - qb; arg[10] = xxx * xxx + aeq;
    xxx = r + qb; arg[11] = xxx * xxx + aeq;
    arg[12] = rsq + aeq;
    arg[13] = arg[12] + qb * qb;
    xxx = da - db; arg[14] = rsq + axx + xxx * xxx;
    xxx = da + db; arg[15] = rsq + axx + xxx * xxx;
    xxx = r + da - db; arg[16] = xxx * xxx + axx;
    xxx = r - da + db; arg[17] = xxx * xxx + axx;
    xxx = r - da - db; arg[18] = xxx * xxx + axx;
    xxx = r + da + db; arg[19] = xxx * xxx + axx;
    xxx = r + da; arg[20] = xxx * xxx + adq;
    arg[21] = arg[20] + qb * qb;
    xxx = r - da; arg[22] = xxx * xxx + adq;
    arg[23] = arg[22] + qb * qb;
    xxx = r - db; arg[24] = xxx * xxx + aqd;
    arg[25] = arg[24] + qa * qa;
    xxx = r + db; arg[26] = xxx * xxx + aqd;
    arg[27] = arg[26] + qa * qa;
    xxx = r + da - qb; arg[28] = xxx * xxx + adq;
    xxx = r - da - qb; arg[29] = xxx * xxx + adq;
    xxx = r + da + qb; arg[30] = xxx * xxx + adq;
    xxx = r - da + qb; arg[31] = xxx * xxx + adq;
    xxx = r + qa - db; arg[32] = xxx * xxx + aqd;
    xxx = r + qa + db; arg[33] = xxx * xxx + aqd;
    xxx = r - qa - db; arg[34] = xxx * xxx + aqd;
    xxx = r - qa + db; arg[35] = xxx * xxx + aqd;
    arg[36] = rsq + aqq;
    xxx = qa - qb; arg[37] = arg[36] + xxx * xxx;
    xxx = qa + qb; arg[38] = arg[36] + xxx * xxx;
    arg[39] = arg[36] + qa * qa;
    arg[40] = arg[36] + qb * qb;
    arg[41] = arg[39] + qb * qb;
    xxx = r - qb; arg[42] = xxx * xxx + aqq;
    arg[43] = arg[42] + qa * qa;
    xxx = r + qb; arg[44] = xxx * xxx + aqq;
    arg[45] = arg[44] + qa * qa;
    xxx = r + qa; arg[46] = xxx * xxx + aqq;
    arg[47] = arg[46] + qb * qb;
    xxx = r - qa; arg[48] = xxx * xxx + aqq;
    arg[49] = arg[48] + qb * qb;
    xxx = r + qa - qb; arg[50] = xxx * xxx + aqq;
    xxx = r + qa + qb; arg[51] = xxx * xxx + aqq;
    xxx = r - qa - qb; arg[52] = xxx * xxx + aqq;
    xxx = r - qa + qb; arg[53] = xxx * xxx + aqq;
    qa = E[ni].qq;
    qb = E[nj].qq;
    xxx = da - qb; xxx = xxx * xxx;
    yyy = r - qb; yyy = yyy * yyy;
    zzz = da + qb; zzz = zzz * zzz;
    www = r + qb; www = www * www;
    arg[54] = xxx + yyy + adq;
    arg[55] = xxx + www + adq;
    arg[56] = zzz + yyy + adq;
    arg[57] = zzz + www + adq;
    xxx = qa - db; xxx = xxx * xxx;
    yyy = qa + db; yyy = yyy * yyy;
    zzz = r + qa; zzz = zzz * zzz;
    www = r - qa; www = www * www;
    arg[58] = zzz + xxx + aqd;
    arg[59] = www + xxx + aqd;
    arg[60] = zzz + yyy + aqd;
    arg[61] = www + yyy + aqd;
    xxx = qa - qb; xxx = xxx * xxx;
    arg[62] = arg[36] + td * xxx;
    yyy = qa + qb; yyy = yyy * yyy;
    arg[63] = arg[36] + td * yyy;
    arg[64] = arg[36] + td * (qa * qa + qb * qb);
    zzz = r + qa - qb; zzz = zzz * zzz;
    arg[65] = zzz + xxx + aqq;
    arg[66] = zzz + yyy + aqq;
    zzz = r + qa + qb; zzz = zzz * zzz;
    arg[67] = zzz + xxx + aqq;
    arg[68] = zzz + yyy + aqq;
    zzz = r - qa - qb; zzz = zzz * zzz;
    arg[69] = zzz + xxx + aqq;
    arg[70] = zzz + yyy + aqq;
    zzz = r - qa + qb; zzz = zzz * zzz;
    arg[71] = zzz + xxx + aqq;
    arg[72] = zzz + yyy + aqq;
    for (int i = 1; i <= 72; ++i) sqr[i] = sqrt(arg[i]);
    double ee = EV / sqr[1];
    double dze = (-ev1 / sqr[2]) + ev1 / sqr[3];
    double qzze = ev2 / sqr[4] + ev2 / sqr[5] - ev1 / sqr[6];
    double qxxe = ev1 / sqr[7] - ev1 / sqr[6];
    double edz = (-ev1 / sqr[8]) + ev1 / sqr[9];
    double eqzz = ev2 / sqr[10] + ev2 / sqr[11] - ev1 / sqr[12];
    double eqxx = ev1 / sqr[13] - ev1 / sqr[12];
    double dxdx = ev1 / sqr[14] - ev1 / sqr[15];
    double dzdz = ev2 / sqr[16] + ev2 / sqr[17] - ev2 / sqr[18] - ev2 / sqr[19];
    double dzqxx = ev2 / sqr[20] - ev2 / sqr[21] - ev2 / sqr[22] + ev2 / sqr[23];
    double qxxdz = ev2 / sqr[24] - ev2 / sqr[25] - ev2 / sqr[26] + ev2 / sqr[27];
    double dzqzz = (-ev3 / sqr[28]) + ev3 / sqr[29] - ev3 / sqr[30] + ev3 / sqr[31] - ev2 / sqr[22] + ev2 / sqr[20];
    double qzzdz = (-ev3 / sqr[32]) + ev3 / sqr[33] - ev3 / sqr[34] + ev3 / sqr[35] + ev2 / sqr[24] - ev2 / sqr[26];
    double qxxqxx = ev3 / sqr[37] + ev3 / sqr[38] - ev2 / sqr[39] - ev2 / sqr[40] + ev2 / sqr[36];
    double qxxqyy = ev2 / sqr[41] - ev2 / sqr[39] - ev2 / sqr[40] + ev2 / sqr[36];
    double qxxqzz = ev3 / sqr[43] + ev3 / sqr[45] - ev3 / sqr[42] - ev3 / sqr[44] - ev2 / sqr[39] + ev2 / sqr[36];
    double qzzqxx = ev3 / sqr[47] + ev3 / sqr[49] - ev3 / sqr[46] - ev3 / sqr[48] - ev2 / sqr[40] + ev2 / sqr[36];
    double qzzqzz = ev4 / sqr[50] + ev4 / sqr[51] + ev4 / sqr[52] + ev4 / sqr[53] - ev3 / sqr[48] - ev3 / sqr[46] -
                    ev3 / sqr[42] - ev3 / sqr[44] + ev2 / sqr[36];
    double dxqxz = (-ev2 / sqr[54]) + ev2 / sqr[55] + ev2 / sqr[56] - ev2 / sqr[57];
    double qxzdx = (-ev2 / sqr[58]) + ev2 / sqr[59] + ev2 / sqr[60] - ev2 / sqr[61];
    double qxzqxz = ev3 / sqr[65] - ev3 / sqr[67] - ev3 / sqr[69] + ev3 / sqr[71] - ev3 / sqr[66] + ev3 / sqr[68] +
                    ev3 / sqr[70] - ev3 / sqr[72];
    ri[1] = ee;
    ri[2] = -dze;
    ri[3] = ee + qzze;
    ri[4] = ee + qxxe;
    ri[5] = -edz;
    ri[6] = dzdz;
    ri[7] = dxdx;
    ri[8] = (-edz) - qzzdz;
    ri[9] = (-edz) - qxxdz;
    ri[10] = -qxzdx;
    ri[11] = ee + eqzz;
    ri[12] = ee + eqxx;
    ri[13] = (-dze) - dzqzz;
    ri[14] = (-dze) - dzqxx;
    ri[15] = -dxqxz;
    ri[16] = ee + eqzz + qzze + qzzqzz;
    ri[17] = ee + eqzz + qxxe + qxxqzz;
    ri[18] = ee + eqxx + qzze + qzzqxx;
    ri[19] = ee + eqxx + qxxe + qxxqxx;
    ri[20] = qxzqxz;
    ri[21] = ee + eqxx + qxxe + qxxqyy;
    ri[22] = pp * (qxxqxx - qxxqyy);
  }
  /* l_feather: smooth switch to point charges (reppd :801-823) */
  double point, cst;
  to_point(rij, &point, &cst);
  static const int coul[23] = {0, 1, 0, 1, 1, 0, 0, 0, 0, 0, 0, 1, 1, 0, 0, 0, 1, 1, 1, 1, 0, 1, 0};
  for (int i = 1; i <= 22; ++i) {
    if (coul[i]) ri[i] = ri[i] * cst + (1.0 - cst) * point;
    else ri[i] = ri[i] * cst;
  }
  *gab = *gab * cst + (1.0 - cst) * point;
  for (int i = 1; i <= 22; ++i) ri[i] = ri[i] * nri[i];
}

/* spcore (mndod.F90:1683-1774): electron-core attraction in local frame. */
static void spcore(int ni, int nj, double r, double core[11][3]) {
  static const double pxy[8] = {0, 1.0, -0.5, -0.5, 0.5, 0.25, 0.25, 0.5};
  memset(core, 0, sizeof(double) * 33);
  double r2 = r * r;
  double aci = E[ni].po9, acj = E[nj].po9;
  double ssi = (aci + E[nj].po1) * (aci + E[nj].po1);
  double ssj = (acj + E[ni].po1) * (acj + E[ni].po1);
  core[1][1] = -E[nj].tore * EV / sqrt(r2 + ssj);
  core[1][2] = -E[ni].tore * EV / sqrt(r2 + ssi);
  if (ni >= 3 || nj >= 3) {
    if (ni >= 3) {
      double ppj = (acj + E[ni].po7) * (acj + E[ni].po7);
      double da = E[ni].ddp2, qa = E[ni].ddp3 / sqrt(2.0);
      double twoqa = qa + qa;
      double adj = (E[ni].po2 + acj) * (E[ni].po2 + acj);
      double aqj = (E[ni].po3 + acj) * (E[ni].po3 + acj);
      double xj[8];
      xj[1] = r2 + ppj;
      xj[2] = r2 + aqj;
      xj[3] = (r + da) * (r + da) + adj;
      xj[4] = (r - da) * (r - da) + adj;
      xj[5] = (r - twoqa) * (r - twoqa) + aqj;
      xj[6] = (r + twoqa) * (r + twoqa) + aqj;
      xj[7] = r2 + twoqa * twoqa + aqj;
      for (int i = 1; i <= 7; ++i) xj[i] = pxy[i] / sqrt(xj[i]);
      double aj2 = (xj[3] + xj[4]) * EV;
      double aj3 = (xj[1] + xj[2] + xj[5] + xj[6]) * EV;
      double aj4 = (xj[1] + xj[2] + xj[7]) * EV;
      core[2][1] = -E[nj].tore * aj2;
      core[3][1] = -E[nj].tore * aj3;
      core[4][1] = -E[nj].tore * aj4;
    }
    if (nj >= 3) {
      double ppi = (aci + E[nj].po7) * (aci + E[nj].po7);
      double db = E[nj].ddp2, qb = E[nj].ddp3 / sqrt(2.0);
      double adi = (E[nj].po2 + aci) * (E[nj].po2 + aci);
      double aqi = (E[nj].po3 + aci) * (E[nj].po3 + aci);
      double twoqb = qb + qb;
      double xi[8];
      xi[1] = r2 + ppi;
      xi[2] = r2 + aqi;
      xi[3] = (r + db) * (r + db) + adi;
      xi[4] = (r - db) * (r - db) + adi;
      xi[5] = (r - twoqb) * (r - twoqb) + aqi;
      xi[6] = (r + twoqb) * (r + twoqb) + aqi;
      xi[7] = r2 + twoqb * twoqb + aqi;
      for (int i = 1; i <= 7; ++i) xi[i] = pxy[i] / sqrt(xi[i]);
      double ai2 = -(xi[3] + xi[4]) * EV;
      double ai3 = (xi[1] + xi[2] + xi[5] + xi[6]) * EV;
      double ai4 = (xi[1] + xi[2] + xi[7]) * EV;
      core[2][2] = -E[ni].tore * ai2;
      core[3][2] = -E[ni].tore * ai3;
      core[4][2] = -E[ni].tore * ai4;
    }
  }
}

/* indexd / indx pair numbering (mndod.F90 fordd :2533-2541) */
static int indexd_(int i, int j) { if (i < j) { int t = i; i = j; j = t; } return -(j * (j - 1)) / 2 + i + 9 * (j - 1); }
static int indx_(int i, int j) { if (i < j) { int t = i; i = j; j = t; } return (i * (i - 1)) / 2 + j; }

/* ind2 SP-SP entries (fordd :2547-2580) and reppd2's ipos map. */
static int ind2_sp(int ij, int kl) {
  static const int tab[][3] = {{1, 1, 1},   {1, 2, 2},   {1, 10, 3},  {1, 18, 4},  {1, 25, 5},
                               {2, 1, 6},   {2, 2, 7},   {2, 10, 8},  {2, 18, 9},  {2, 25, 10},
                               {10, 1, 11}, {10, 2, 12}, {10, 10, 13}, {10, 18, 14}, {10, 25, 15},
                               {3, 3, 16},  {3, 11, 17}, {11, 3, 18}, {11, 11, 19}, {18, 1, 20},
                               {18, 2, 21}, {18, 10, 22}, {18, 18, 23}, {18, 25, 24}, {4, 4, 25},
                               {4, 12, 26}, {12, 4, 27}, {12, 12, 28}, {19, 19, 29}, {25, 1, 30},
                               {25, 2, 31}, {25, 10, 32}, {25, 18, 33}, {25, 25, 34}};
  for (unsigned t = 0; t < sizeof(tab) / sizeof(tab[0]); ++t)
    if (tab[t][0] == ij && tab[t][1] == kl) return tab[t][2];
  return 0;
}
static const int IPOS[35] = {0, 1, 5, 11, 12, 12, 2, 6, 13, 14, 14, 3, 8, 16, 18, 18, 7, 15,
                             10, 20, 4, 9, 17, 19, 21, 7, 15, 10, 20, 22, 4, 9, 17, 21, 19};
static const int MET[11] = {0, 1, 2, 3, 2, 3, 3, 2, 3, 3, 3};

/* rotation products (rotmat :1382-1567, sp part) */
typedef struct { double p[4][4]; double pp[7][4][4]; } rot_t;

static double rotmat(const double *ci, const double *cj, rot_t *R) {
  const double small = 1.0e-7;
  double x11 = cj[0] - ci[0], x22 = cj[1] - ci[1], x33 = cj[2] - ci[2];
  double b = x11 * x11 + x22 * x22;
  double r = sqrt(b + x33 * x33);
  double sqb = sqrt(b);
  double sb = sqb / r, ca, sa, cb;
  if (sb > small) { ca = x11 / sqb; sa = x22 / sqb; cb = x33 / r; }
  else {
    sa = 0.0; sb = 0.0;
    if (x33 < 0.0) { ca = -1.0; cb = -1.0; }
    else if (x33 > 0.0) { ca = 1.0; cb = 1.0; }
    else { ca = 0.0; cb = 0.0; }
  }
  double (*p)[4] = R->p;
  p[1][1] = ca * sb; p[2][1] = ca * cb; p[3][1] = -sa;
  p[1][2] = sa * sb; p[2][2] = sa * cb; p[3][2] = ca;
  p[1][3] = cb;      p[2][3] = -sb;     p[3][3] = 0.0;
  for (int k = 1; k <= 3; ++k) {
    R->pp[1][k][k] = p[k][1] * p[k][1];
    R->pp[2][k][k] = p[k][2] * p[k][2];
    R->pp[3][k][k] = p[k][3] * p[k][3];
    R->pp[4][k][k] = p[k][1] * p[k][2];
    R->pp[5][k][k] = p[k][1] * p[k][3];
    R->pp[6][k][k] = p[k][2] * p[k][3];
    for (int l = 1; l < k; ++l) {
      R->pp[1][k][l] = 2.0 * p[k][1] * p[l][1];
      R->pp[2][k][l] = 2.0 * p[k][2] * p[l][2];
      R->pp[3][k][l] = 2.0 * p[k][3] * p[l][3];
      R->pp[4][k][l] = p[k][1] * p[l][2] + p[k][2] * p[l][1];
      R->pp[5][k][l] = p[k][1] * p[l][3] + p[k][3] * p[l][1];
      R->pp[6][k][l] = p[k][2] * p[l][3] + p[k][3] * p[l][2];
    }
  }
  return r;
}

/* ccrep.F90, PM7 branch. r in Bohr on entry. Returns core-core repulsion. */
static double ccrep(int ni, int nj, double r, double gab) {
  r = r * A0;
  double enuc = E[ni].tore * E[nj].tore * gab;
  double fff = XFAC[ni][nj];
  double enuclr, scale, abond;
  if (fabs(fff) < 1.0e-5) { /* PM7: average the diagonal pair parameters */
    XFAC[ni][nj] = 0.5 * (XFAC[ni][ni] + XFAC[nj][nj]);
    ALPB[ni][nj] = 0.5 * (ALPB[ni][ni] + ALPB[nj][nj]);
    fff = XFAC[ni][nj];
  }
  if (fabs(fff) > 1.0e-5) {
    abond = ALPB[ni][nj];
    if (abond < 1.0e-6) abond = 1.2;
    /* the reference writes 0.0003 as a default-kind (single precision) literal */
    scale = 1.0 + 2.0 * fff * exp(-abond * (r + (double)0.0003f * ipow(r, 6)));
    int i = ni > nj ? ni : nj, j = ni < nj ? ni : nj;
    if (j == 1) {
      if (i == 6 || i == 7) scale = 1.0 + 2.0 * fff * exp(-abond * r * r);
      else if (i == 8) scale = 1.0 + 2.0 * fff * exp(-abond * r * r) - PAR3 * exp(-PAR4 * r * 2);
    } else if (j == 6 && i == 6) {
      scale = scale + PAR1 * exp(-PAR2 * r);
    }
    enuclr = enuc * scale;
  } else {
    abond = 0.0;
    scale = 10.0 * exp(-2.18 * r);
    enuclr = fabs(scale * enuc) + enuc;
  }
  scale = 0.0;
  double ax = E[ni].g2 * (r - E[ni].g3) * (r - E[ni].g3);
  if (ax < 25.0) scale = scale + E[ni].tore * E[nj].tore / r * E[ni].g1 * exp(-ax);
  ax = E[nj].g2 * (r - E[nj].g3) * (r - E[nj].g3);
  if (ax < 25.0) scale = scale + E[ni].tore * E[nj].tore / r * E[nj].g1 * exp(-ax);
  enuclr = enuclr + scale;
  ax = r / (pow((double)ni, 0.3333) + pow((double)nj, 0.3333));
  if (ax < 3.0) {
    scale = 1.0e-8 / ipow(ax, 12);
    enuclr = enuclr + (scale < 1.0e5 ? scale : 1.0e5);
  }
  return enuclr;
}

/* rotate -> rotatd for an sp pair.  w: limij*limkl block in reference layout
 * (kl fastest); e1b/e2a: packed local blocks; returns enuc. */
static double rotate_pair(int ni, int nj, const double *xi, const double *xj, double *w,
                          double *e1b, double *e2a) {
  double xd[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
  double rij2 = xd[0] * xd[0] + xd[1] * xd[1] + xd[2] * xd[2];
  int ii = E[ni].natorb, kk = E[nj].natorb;
  int limij = indx_(ii, ii), limkl = indx_(kk, kk);
  if (rij2 < 0.00002) {
    memset(w, 0, sizeof(double) * limij * limkl);
    memset(e1b, 0, sizeof(double) * 10);
    memset(e2a, 0, sizeof(double) * 10);
    return 0.0;
  }
  rot_t R;
  double r = rotmat(xi, xj, &R);
  double ri[23], gab;
  reppd(ni, nj, r, ri, &gab);
  double rij = r;
  double rb = r / A0;
  double core[11][3];
  spcore(ni, nj, rb, core);
  double point, cst;
  to_point(rij, &point, &cst);
  point = -(EV / rb) * E[nj].tore;
  core[1][1] = core[1][1] * cst + (1.0 - cst) * point;
  core[2][1] = core[2][1] * cst;
  core[3][1] = core[3][1] * cst + (1.0 - cst) * point;
  core[4][1] = core[4][1] * cst + (1.0 - cst) * point;
  point = -(EV / rb) * E[ni].tore;
  core[1][2] = core[1][2] * cst + (1.0 - cst) * point;
  core[2][2] = core[2][2] * cst;
  core[3][2] = core[3][2] * cst + (1.0 - cst) * point;
  core[4][2] = core[4][2] * cst + (1.0 - cst) * point;
  double rep[35];
  for (int i = 1; i <= 34; ++i) rep[i] = ri[IPOS[i]];
  /* tx: v(ij_local_A, kl_mol_B) */
  double v[26][11];
  memset(v, 0, sizeof(v));
  for (int i1 = 1; i1 <= ii; ++i1)
    for (int j1 = 1; j1 <= i1; ++j1) {
      int ij = indexd_(i1, j1);
      for (int k1 = 1; k1 <= kk; ++k1)
        for (int l1 = 1; l1 <= k1; ++l1) {
          int kl = indexd_(k1, l1);
          int nd = ind2_sp(ij, kl);
          if (nd == 0) continue;
          double wrepp = rep[nd];
          int mm = MET[indx_(k1, l1)];
          if (mm == 1) v[ij][1] = wrepp;
          else if (mm == 2) {
            int k = k1 - 1;
            v[ij][2] = v[ij][2] + R.p[k][1] * wrepp;
            v[ij][4] = v[ij][4] + R.p[k][2] * wrepp;
            v[ij][7] = v[ij][7] + R.p[k][3] * wrepp;
          } else {
            int k = k1 - 1, l = l1 - 1;
            v[ij][3] = v[ij][3] + R.pp[1][k][l] * wrepp;
            v[ij][6] = v[ij][6] + R.pp[2][k][l] * wrepp;
            v[ij][10] = v[ij][10] + R.pp[3][k][l] * wrepp;
            v[ij][5] = v[ij][5] + R.pp[4][k][l] * wrepp;
            v[ij][8] = v[ij][8] + R.pp[5][k][l] * wrepp;
            v[ij][9] = v[ij][9] + R.pp[6][k][l] * wrepp;
          }
        }
    }
  /* rotatd main loop: rotate atom A's side into the molecular frame */
  double ww[100];
  memset(ww, 0, sizeof(ww));
#define INDW(a, b) ((indx_((a), (b)) - 1) * limkl + kl - 1)
  for (int i1 = 1; i1 <= ii; ++i1)
    for (int j1 = 1; j1 <= i1; ++j1) {
      int ij = indexd_(i1, j1);
      int mm = MET[indx_(i1, j1)];
      for (int k = 1; k <= kk; ++k)
        for (int l = 1; l <= k; ++l) {
          int kl = indx_(k, l);
          double wrepp = v[ij][kl];
          if (wrepp == 0.0) continue; /* logv */
          if (mm == 1) ww[INDW(1, 1)] = wrepp;
          else if (mm == 2) {
            for (int i = 1; i <= 3; ++i) ww[INDW(i + 1, 1)] += R.p[i1 - 1][i] * wrepp;
          } else {
            for (int i = 1; i <= 3; ++i) {
              double cc = R.pp[i][i1 - 1][j1 - 1];
              ww[INDW(i + 1, i + 1)] += cc * wrepp;
              for (int j = 1; j < i; ++j) {
                cc = R.pp[1 + i + j][i1 - 1][j1 - 1];
                ww[INDW(i + 1, j + 1)] += cc * wrepp;
              }
            }
          }
        }
    }
#undef INDW
  memcpy(w, ww, sizeof(double) * limij * limkl);
  double enuc = ccrep(ni, nj, rb, gab);
  /* elenuc (mndod.F90:2367): electron-nuclear attraction blocks */
  static const int indpp[4][4] = {{0, 0, 0, 0}, {0, 1, 4, 5}, {0, 4, 2, 6}, {0, 5, 6, 3}};
  for (int n = 1; n <= 2; ++n) {
    int lim = n == 1 ? ii : kk;
    double *out = n == 1 ? e1b : e2a;
    int m = 0;
    for (int i = 1; i <= lim; ++i) {
      int ind1 = i - 1;
      for (int j = 1; j <= i; ++j) {
        int ind2 = j - 1;
        double h;
        if (ind1 == 0) h = core[1][n];
        else if (ind2 == 0) h = R.p[1][ind1] * core[2][n];
        else {
          int ipp = indpp[ind1][ind2];
          h = core[3][n] * R.pp[ipp][1][1] + core[4][n] * (R.pp[ipp][2][2] + R.pp[ipp][3][3]);
        }
        out[m++] = 0.0 + h;
      }
    }
  }
  return enuc;
}

/* wstore (mndod.F90:2027): one-centre block, ilim x ilim, column-major. */
static void wstore(int ni, double *w) {
  int ilim = indx_(E[ni].natorb, E[ni].natorb);
  for (int i = 0; i < ilim * ilim; ++i) w[i] = 0.0;
#define WS(a, b) w[((a) - 1) + ilim * ((b) - 1)]
  WS(1, 1) = E[ni].gss;
  if (E[ni].natorb > 2) {
    int ip = 1, ipx = ip + 2, ipy = ip + 5, ipz = ip + 9;
    double gsp = E[ni].gsp, gpp = E[ni].gpp, gp2 = E[ni].gp2, hsp = E[ni].hsp;
    WS(ipx, ip) = gsp; WS(ipy, ip) = gsp; WS(ipz, ip) = gsp;
    WS(ip, ipx) = gsp; WS(ip, ipy) = gsp; WS(ip, ipz) = gsp;
    WS(ipx, ipx) = gpp; WS(ipy, ipy) = gpp; WS(ipz, ipz) = gpp;
    WS(ipy, ipx) = gp2; WS(ipz, ipx) = gp2; WS(ipz, ipy) = gp2;
    WS(ipx, ipy) = gp2; WS(ipx, ipz) = gp2; WS(ipy, ipz) = gp2;
    WS(ip + 1, ip + 1) = hsp; WS(ip + 3, ip + 3) = hsp; WS(ip + 6, ip + 6) = hsp;
    WS(ip + 4, ip + 4) = 0.5 * (gpp - gp2);
    WS(ip + 7, ip + 7) = 0.5 * (gpp - gp2);
    WS(ip + 8, ip + 8) = 0.5 * (gpp - gp2);
  }
#undef WS
}

/* ------------------------------------------------------------------ */
/* Public API (ctypes)                                                 */
/* ------------------------------------------------------------------ */
int orc_supported(int z) { return supported(z); }

/* Orbital layout: nfirst/nlast are 1-based like the reference. Returns norbs
 * or -1 for an unsupported element. */
int orc_layout(int numat, const int *nat, int *nfirst, int *nlast) {
  init_params();
  int ia = 1;
  for (int i = 0; i < numat; ++i) {
    if (!supported(nat[i])) return -1;
    nfirst[i] = ia;
    nlast[i] = ia + E[nat[i]].natorb - 1;
    ia = nlast[i] + 1;
  }
  return ia - 1;
}

long long orc_n2elec(int numat, const int *nat) {
  init_params();
  long long n = 0;
  for (int i = 0; i < numat; ++i) {
    int li = indx_(E[nat[i]].natorb, E[nat[i]].natorb);
    for (int j = 0; j < i; ++j) n += (long long)li * indx_(E[nat[j]].natorb, E[nat[j]].natorb);
    n += (long long)li * li;
  }
  return n;
}

double orc_param(int z, const char *name) {
  init_params();
  if (!supported(z)) return 0.0;
  elem_t *e = &E[z];
  if (!strcmp(name, "dd")) return e->dd;
  if (!strcmp(name, "qq")) return e->qq;
  if (!strcmp(name, "am")) return e->am;
  if (!strcmp(name, "ad")) return e->ad;
  if (!strcmp(name, "aq")) return e->aq;
  if (!strcmp(name, "eisol")) return e->eisol;
  if (!strcmp(name, "tore")) return e->tore;
  return 0.0;
}

/* hcore.F90:150-297 (no field, no COSMO, id = 0).  h: mpack, w: n2elec. */
void orc_hcore(int numat, const int *nat, const double *coord, double *h, double *w,
               double *enuclr_out) {
  init_params();
  int nfirst[numat > 0 ? numat : 1], nlast[numat > 0 ? numat : 1];
  int norbs = orc_layout(numat, nat, nfirst, nlast);
  long long mpack = (long long)norbs * (norbs + 1) / 2;
  for (long long i = 0; i < mpack; ++i) h[i] = 0.0;
  double enuclr = 0.0;
  const double cutof1 = 225.0;
  long long kr = 0;
  for (int i = 0; i < numat; ++i) {
    int ia = nfirst[i], ib = nlast[i], ni = nat[i];
    for (int i1 = ia; i1 <= ib; ++i1) { /* diagonal: uspd */
      long long i2 = (long long)i1 * (i1 - 1) / 2 + i1;
      h[i2 - 1] = (i1 == ia) ? E[ni].uss : E[ni].upp;
    }
    const double *xi = coord + 3 * i;
    for (int j = 0; j < i; ++j) {
      int ja = nfirst[j], jb = nlast[j], nj = nat[j];
      const double *xj = coord + 3 * j;
      double di[5][5];
      h1elec(ni, nj, xi, xj, di, cutof1);
      int i2 = 0;
      for (int i1 = ia; i1 <= ib; ++i1) {
        long long ii = (long long)i1 * (i1 - 1) / 2 + ja - 1;
        ++i2;
        int jj = i1 < jb ? i1 : jb;
        for (int c = 1; c <= jj - ja + 1; ++c) h[ii + c - 1] = h[ii + c - 1] + di[i2][c];
      }
      double e1b[10], e2a[10];
      double enuc = rotate_pair(ni, nj, xi, xj, w + kr, e1b, e2a);
      kr += (long long)indx_(E[ni].natorb, E[ni].natorb) * indx_(E[nj].natorb, E[nj].natorb);
      enuclr = enuclr + enuc;
      i2 = 0;
      for (int i1 = ia; i1 <= ib; ++i1) {
        long long ii = (long long)i1 * (i1 - 1) / 2 + ia - 1;
        for (int c = 1; c <= i1 - ia + 1; ++c) h[ii + c - 1] = h[ii + c - 1] + e1b[i2 + c - 1] * 1.0;
        i2 += i1 - ia + 1;
      }
      i2 = 0;
      for (int i1 = ja; i1 <= jb; ++i1) {
        long long ii = (long long)i1 * (i1 - 1) / 2 + ja - 1;
        for (int c = 1; c <= i1 - ja + 1; ++c) h[ii + c - 1] = h[ii + c - 1] + e2a[i2 + c - 1] * 1.0;
        i2 += i1 - ja + 1;
      }
    }
    wstore(ni, w + kr);
    int il = indx_(E[ni].natorb, E[ni].natorb);
    kr += (long long)il * il;
  }
  *enuclr_out = enuclr;
}

/* fock1.F90: one-centre terms for atom ia..ib (1-based orbitals). */
static void fock1(double *f, const double *ptot, const double *pa, const double *w, int ia, int ib) {
  int ilim = ((ib - ia + 1) * (ib - ia + 2)) / 2;
#define WF(a, b) w[((a) - 1) + ilim * ((b) - 1)]
  for (int i = ia; i <= ib; ++i) {
    int iw = i - ia + 1;
    for (int j = ia; j <= i; ++j) {
      int jw = j - ia + 1;
      long long ij = (long long)i * (i - 1) / 2 + j;
      int ijw = (iw * (iw - 1)) / 2 + jw;
      double sum = 0.0;
      for (int k = ia; k <= ib; ++k) {
        int kw = k - ia + 1;
        for (int l = ia; l <= ib; ++l) {
          int lw = l - ia + 1;
          int ip = k > l ? k : l, jp = k < l ? k : l;
          long long ijp = (long long)ip * (ip - 1) / 2 + jp;
          int im = kw > lw ? kw : lw, jm = kw < lw ? kw : lw;
          int klw = (im * (im - 1)) / 2 + jm;
          im = kw > jw ? kw : jw; jm = kw < jw ? kw : jw;
          int ikw = (im * (im - 1)) / 2 + jm;
          im = lw > iw ? lw : iw; jm = lw < iw ? lw : iw;
          int jlw = (im * (im - 1)) / 2 + jm;
          sum = sum + ptot[ijp - 1] * WF(ijw, klw) - pa[ijp - 1] * WF(ikw, jlw);
        }
      }
      f[ij - 1] = f[ij - 1] + sum;
    }
  }
#undef WF
}

#define IF_(i) (((long long)(i) * ((i) - 1)) / 2)
/* fock2.F90:111-369 (sp branches, mode 2).  All arrays packed lower, 0-based
 * storage, 1-based orbital numbering in nfirst/nlast.  f is updated in place. */
void orc_fock2(int numat, const int *nfirst, const int *nlast, double *f, const double *ptot,
               const double *p, const double *w) {
  /* pair-index helpers for jab/kab term orders */
  static const int pidx[16] = {1, 2, 4, 7, 2, 3, 5, 8, 4, 5, 6, 9, 7, 8, 9, 10};
  long long kk = 0;
  for (int ii = 0; ii < numat; ++ii) {
    int ia = nfirst[ii], ib = nlast[ii];
    for (int jj = 0; jj < ii; ++jj) {
      int ja = nfirst[jj], jb = nlast[jj];
      const double *wk = w + kk;
      if (ib - ia >= 3 && jb - ja >= 3) {
        /* jab: Coulomb between two heavy atoms */
        double pja[16], pjb[16];
        for (int a = 0; a < 4; ++a)
          for (int b = 0; b < 4; ++b) {
            int r = ia + a, c = ia + b;
            int mx = r > c ? r : c, mn = r < c ? r : c;
            pja[a * 4 + b] = ptot[IF_(mx) + mn - 1];
            r = ja + a; c = ja + b;
            mx = r > c ? r : c; mn = r < c ? r : c;
            pjb[a * 4 + b] = ptot[IF_(mx) + mn - 1];
          }
        double suma[10], sumb[10];
        for (int q = 0; q < 10; ++q) {
          double sa = pja[0] * wk[(pidx[0] - 1) * 10 + q];
          for (int m = 1; m < 16; ++m) sa = sa + pja[m] * wk[(pidx[m] - 1) * 10 + q];
          suma[q] = sa;
          double sb = pjb[0] * wk[q * 10 + pidx[0] - 1];
          for (int m = 1; m < 16; ++m) sb = sb + pjb[m] * wk[q * 10 + pidx[m] - 1];
          sumb[q] = sb;
        }
        int i = 0;
        for (int i5 = 1; i5 <= 4; ++i5) {
          int iia = ia + i5 - 1, ija = ja + i5 - 1;
          long long ioff = IF_(iia) + ia - 1, joff = IF_(ija) + ja - 1;
          for (int i6 = 1; i6 <= i5; ++i6) {
            ++ioff; ++joff;
            f[ioff - 1] = f[ioff - 1] + sumb[i];
            f[joff - 1] = f[joff - 1] + suma[i];
            ++i;
          }
        }
        /* kab: exchange, off-diagonal block */
        double pk[16];
        for (int a = 0; a < 4; ++a)
          for (int b = 0; b < 4; ++b) pk[a * 4 + b] = p[IF_(ia + a) + ja + b - 1];
        for (int mu = 1; mu <= 4; ++mu)
          for (int nu = 1; nu <= 4; ++nu) {
            double s = 0.0;
            int first = 1;
            for (int lam = 1; lam <= 4; ++lam)
              for (int sig = 1; sig <= 4; ++sig) {
                double t = pk[(lam - 1) * 4 + sig - 1] * wk[(indx_(mu, lam) - 1) * 10 + indx_(nu, sig) - 1];
                if (first) { s = t; first = 0; } else s = s + t;
              }
            long long idx = IF_(ia + mu - 1) + ja + nu - 1;
            f[idx - 1] = f[idx - 1] - s;
          }
        kk += 100;
      } else if (ib - ia >= 3 && ja == jb) {
        double sumdia = 0.0, sumoff = 0.0;
        long long ll = IF_(ja) + ja;
        int k = 0;
        for (int i = 0; i <= 3; ++i) {
          long long j1 = IF_(ia + i) + ia - 1;
          if (i > 0) {
            for (int j = 1; j <= i; ++j) {
              f[j + j1 - 1] = f[j + j1 - 1] + ptot[ll - 1] * wk[j + k - 1];
              sumoff = sumoff + ptot[j + j1 - 1] * wk[j + k - 1];
            }
            k = i + k;
            j1 = i + j1;
          }
          j1 = j1 + 1;
          k = k + 1;
          f[j1 - 1] = f[j1 - 1] + ptot[ll - 1] * wk[k - 1];
          sumdia = sumdia + ptot[j1 - 1] * wk[k - 1];
        }
        f[ll - 1] = f[ll - 1] + sumoff * 2.0 + sumdia;
        for (int i = ia; i <= ib; ++i) {
          long long i1 = IF_(i) + ja;
          double sum = 0.0;
          for (int j = 1; j <= ib - ia + 1; ++j)
            sum = sum + p[IF_(j - 1 + ia) + ja - 1] * wk[indx_(i - ia + 1, j) - 1];
          f[i1 - 1] = f[i1 - 1] - sum;
        }
        kk += 10;
      } else if (jb - ja >= 3 && ia == ib) {
        double sumdia = 0.0, sumoff = 0.0;
        long long ll = IF_(ia) + ia;
        int k = 0;
        for (int i = 0; i <= 3; ++i) {
          long long j1 = IF_(ja + i) + ja - 1;
          if (i > 0) {
            for (int j = 1; j <= i; ++j) {
              f[j + j1 - 1] = f[j + j1 - 1] + ptot[ll - 1] * wk[j + k - 1];
              sumoff = sumoff + ptot[j + j1 - 1] * wk[j + k - 1];
            }
            k = i + k;
            j1 = i + j1;
          }
          j1 = j1 + 1;
          k = k + 1;
          f[j1 - 1] = f[j1 - 1] + ptot[ll - 1] * wk[k - 1];
          sumdia = sumdia + ptot[j1 - 1] * wk[k - 1];
        }
        f[ll - 1] = f[ll - 1] + sumoff * 2.0 + sumdia;
        long long k0 = IF_(ia) + ja;
        for (int i = 0; i < 4; ++i) {
          double sum = 0.0;
          for (int l = 1; l <= 4; ++l) sum = sum + p[l - 1 + k0 - 1] * wk[indx_(i + 1, l) - 1];
          f[k0 + i - 1] = f[k0 + i - 1] - sum;
        }
        kk += 10;
      } else if (jb == ja && ia == ib) {
        long long i1 = IF_(ia) + ia, j1 = IF_(ja) + ja, ij = i1 + ja - ia;
        f[i1 - 1] = f[i1 - 1] + ptot[j1 - 1] * wk[0];
        f[j1 - 1] = f[j1 - 1] + ptot[i1 - 1] * wk[0];
        f[ij - 1] = f[ij - 1] - p[ij - 1] * wk[0];
        kk += 1;
      }
    }
    int ilim = ((ib - ia + 1) * (ib - ia + 2)) / 2;
    fock1(f, ptot, p, w + kk, ia, ib);
    kk += (long long)ilim * ilim;
  }
}

/* helect.F90 */
double orc_helect(int n, const double *p, const double *h, const double *f) {
  double ed = 0.0, ee = 0.0;
  long long k = 0;
  int nn = n + 1;
  for (int i = 2; i <= nn; ++i) {
    k = k + 1;
    int jj = i - 1;
    ed = ed + p[k - 1] * (h[k - 1] + f[k - 1]);
    if (i == nn) continue;
    if (jj > 0) {
      double s = 0.0;
      for (int q = 1; q <= jj; ++q) s = s + p[k + q - 1] * (h[k + q - 1] + f[k + q - 1]);
      ee = ee + s;
      k = jj + k;
    }
  }
  ee = ee + 0.5 * ed;
  return ee;
}

/* cnvg.F90 (RHF: rhfuhf = 2). pnew is the fresh density (overwritten by the
 * extrapolated one), p the previous density, p1 the diagonal two steps back. */
void orc_cnvg(int norbs, double *pnew, double *p, double *p1, int niter, double *pl_out) {
  const double rhfuhf = 2.0;
  double pl = 0.0, faca = 0.0, facb = 0.0, fac = 0.0;
  double damp = 1.0e10;
  if (niter > 3) damp = 0.05;
  int extrap = (niter % 3) != 0;
  double sum1 = 0.0;
  long long k = 0;
  for (int i = 1; i <= norbs; ++i) {
    k = k + i;
    double a = pnew[k - 1];
    sum1 = sum1 + a;
    double sa = fabs(a - p[k - 1]);
    if (sa > pl) pl = sa;
    if (!extrap) {
      faca = faca + sa * sa;
      double t = a - 2.0 * p[k - 1] + p1[i - 1];
      facb = facb + t * t;
    }
    p1[i - 1] = p[k - 1];
    p[k - 1] = a;
  }
  if (facb > 1.0e-10 && faca < (100.0 * facb)) fac = sqrt(faca / facb);
  long long ie = 0;
  double sum2 = 0.0;
  for (int i = 1; i <= norbs; ++i) {
    int ii = i - 1;
    for (int j = 1; j <= ii; ++j) {
      ie = ie + 1;
      double a = pnew[ie - 1];
      p[ie - 1] = a + fac * (a - p[ie - 1]);
      pnew[ie - 1] = p[ie - 1];
    }
    ie = ie + 1;
    if (fabs(p[ie - 1] - p1[i - 1]) > damp)
      p[ie - 1] = p1[i - 1] + copysign(damp, p[ie - 1] - p1[i - 1]);
    else
      p[ie - 1] = p[ie - 1] + fac * (p[ie - 1] - p1[i - 1]);
    double t = p[ie - 1] > 0.0 ? p[ie - 1] : 0.0;
    p[ie - 1] = t < rhfuhf ? t : rhfuhf;
    sum2 = sum2 + p[ie - 1];
    pnew[ie - 1] = p[ie - 1];
  }
  double sum0 = sum1;
  for (;;) {
    double sum;
    if (sum2 > 1.0e-3) sum = sum1 / sum2;
    else sum = 0.0;
    sum1 = sum0;
    if (sum2 < 1.0e-3 || fabs(sum - 1.0) < 1.0e-5) break;
    sum2 = 0.0;
    for (int i = 1; i <= norbs; ++i) {
      long long j = IF_(i) + i;
      p[j - 1] = p[j - 1] * sum + 1.0e-20;
      p[j - 1] = p[j - 1] > 0.0 ? p[j - 1] : 0.0;
      if (p[j - 1] > rhfuhf) {
        p[j - 1] = rhfuhf;
        sum1 = sum1 - rhfuhf;
      } else {
        sum2 = sum2 + p[j - 1];
      }
      pnew[j - 1] = p[j - 1];
    }
  }
  *pl_out = pl;
}

/* moldat.F90:731-760 diagonal guess, neutral molecule (kharge = 0). */
void orc_pdiag(int numat, const int *nat, double *pdiag) {
  init_params();
  int l = 0;
  for (int i = 0; i < numat; ++i) {
    int z = nat[i];
    if (E[z].natorb == 1) pdiag[l++] = E[z].tore;
    else for (int q = 0; q < 4; ++q) pdiag[l++] = E[z].tore * 0.25;
  }
}

/* atheat: sum(eheat) - sum(eisol)*fpc_9 (C-C triple-bond term is zero for
 * H/C/O molecules without sp carbon pairs). */
double orc_atheat(int numat, const int *nat) {
  init_params();
  double atheat = 0.0, eat = 0.0;
  for (int i = 0; i < numat; ++i) atheat = atheat + E[nat[i]].eheat;
  for (int i = 0; i < numat; ++i) eat = eat + E[nat[i]].eisol;
  return atheat - eat * FPC9;
}

/* Bond count used by the PM7 dispersion term: set_up_dentate.F90:36-80 uses
 * covalent radii with element-pair safety factors.  Radii here are the
 * covalent radii for H, C, O. */
static void count_bonds(int numat, const int *nat, const double *coord, int *nb) {
  for (int i = 0; i < numat; ++i) nb[i] = 0;
  for (int i = 0; i < numat; ++i)
    for (int j = 0; j < i; ++j) {
      double rad[9] = {0, 0.37, 0, 0, 0, 0, 0.77, 0, 0.73};
      int il = nat[i] < nat[j] ? nat[i] : nat[j], iu = nat[i] > nat[j] ? nat[i] : nat[j];
      double safety = 1.1;
      if (il == 1 && iu == 6) safety = 1.25;
      if (il == 6 && iu < 8) safety = 1.2;
      double dx = coord[3 * i] - coord[3 * j], dy = coord[3 * i + 1] - coord[3 * j + 1],
             dz = coord[3 * i + 2] - coord[3 * j + 2];
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      if (r < safety * (rad[nat[i]] + rad[nat[j]])) { nb[i]++; nb[j]++; }
    }
}

/* PM6_DH_Disp for PM7 (H_bond_correction_PM6_DH_Dispersion.F90:49-260), id=0. */
double orc_disp_pm7(int numat, const int *nat, const double *coord) {
  double Cc[9] = {0, 0.16, 0.084, 0, 0, 5.79, 1.65, 1.11, 0.70};
  double Rr[9] = {0, 156.0, 140.0, 0, 0, 180.0, 170.0, 155.0, 152.0};
  double Nn[9] = {0, 0.80, 1.42, 0, 0, 2.16, 2.50, 2.82, 3.15};
  const double alpha = 15.450118, s = 1.226593, cscale = 2.286419;
  int *nb = (int *)malloc(sizeof(int) * (numat > 0 ? numat : 1));
  count_bonds(numat, nat, coord, nb);
  double E_disp = 0.0;
  for (int i = 0; i < numat; ++i) {
    int ni = nat[i];
    for (int j = i + 1; j < numat; ++j) {
      int nj = nat[j];
      double C6i = ni == 6 ? (nb[i] == 4 ? 0.95 : 1.65) : Cc[ni];
      double C6j = nj == 6 ? (nb[j] == 4 ? 0.95 : 1.65) : Cc[nj];
      double C6 = 2.0 * pow(C6i * C6i * C6j * C6j * Nn[ni] * Nn[nj], 1.0 / 3.0) /
                  (pow(C6i * Nn[nj] * Nn[nj], 1.0 / 3.0) + pow(C6j * Nn[ni] * Nn[ni], 1.0 / 3.0));
      double R0 = (Rr[ni] * Rr[ni] * Rr[ni] + Rr[nj] * Rr[nj] * Rr[nj]) / (Rr[ni] * Rr[ni] + Rr[nj] * Rr[nj]) /
                  1000.0 * 2.0;
      double dx = coord[3 * i] - coord[3 * j], dy = coord[3 * i + 1] - coord[3 * j + 1],
             dz = coord[3 * i + 2] - coord[3 * j + 2];
      double rab = dx * dx + dy * dy + dz * dz;
      if (rab < 100.0 * 100.0) {
        double Rij = sqrt(rab) * 0.1;
        double damp = 1.0 / (1.0 + exp(-alpha * (Rij / (s * R0) - 1.0)));
        E_disp = E_disp - C6 / ipow(Rij, 6) * damp / (1000.0 * 4.184);
      }
    }
  }
  free(nb);
  return E_disp * cscale;
}

double orc_const(const char *name) {
  if (!strcmp(name, "fpc_9")) return FPC9;
  if (!strcmp(name, "ev")) return EV;
  if (!strcmp(name, "a0")) return A0;
  return 0.0;
}

/* ======================================================================
 * MOZYME sparse pair-block storage and the kernels on it.
 * ====================================================================== */

/* fillij (MOZYME/fillij.F90:20-230), first call, molecular (id = 0), full
 * nijbo table (lijbo): for atom i in order, the blocks of its partners j < i
 * with r^2 < cutof2 (iorbs(i) x iorbs(j), atom i's orbitals outer), then its
 * own lower triangle.  nijbo (numat x numat, row-major here, symmetric) gets
 * the 0-based block offset, -2 for cutof2 <= r^2 < cutof1 and -1 beyond.
 * Returns mpack. */
long long orc_mz_layout(int numat, const int *iorbs, const double *coord, double cutof1, double cutof2,
                        long long *nijbo) {
    long long mpack = 0;
    for (int i = 0; i < numat; ++i) {
        const int io = iorbs[i];
        const double x1 = coord[3 * i], x2 = coord[3 * i + 1], x3 = coord[3 * i + 2];
        for (int j = 0; j < i; ++j) {
            const int jo = iorbs[j];
            const double dx = x1 - coord[3 * j], dy = x2 - coord[3 * j + 1], dz = x3 - coord[3 * j + 2];
            const double r = dx * dx + dy * dy + dz * dz;
            long long v;
            if (r < cutof2) {
                v = mpack;
                mpack += (long long)io * jo;
            } else if (r < cutof1) {
                v = -2;
            } else {
                v = -1;
            }
            nijbo[(long long)i * numat + j] = v;
            nijbo[(long long)j * numat + i] = v;
        }
        nijbo[(long long)i * numat + i] = mpack;
        mpack += (long long)io * (io + 1) / 2;
    }
    return mpack;
}

/* density_for_MOZYME (MOZYME/density_for_MOZYME.F90:16-342), lijbo branch,
 * CPU arithmetic.  LMO i (0-based) covers the ncf[i] atoms icocc[nncf[i] ..]
 * (1-based atom numbers), its coefficients start at cocc[ncocc[i]] in the
 * order of that atom list, iorbs[atom] per atom. */
void orc_mz_density(int numat, const int *iorbs, const long long *nijbo, int nclose, const int *ncf,
                    const int *nncf, const int *icocc, const int *ncocc, const double *cocc, int mode,
                    long long mpack, const double *partp, double *p) {
    if (mode == 0) {
        for (long long l = 0; l < mpack; ++l) p[l] = 0.0;
    } else if (mode == -1) {
        for (long long l = 0; l < mpack; ++l) p[l] = -0.5 * partp[l];
    } else {
        for (long long l = 0; l < mpack; ++l) p[l] = 0.5 * partp[l];
    }
    for (int i = 0; i < nclose; ++i) {
        const int loop = ncocc[i];
        int ja = 0;
        for (int jj = nncf[i]; jj < nncf[i] + ncf[i]; ++jj) {
            const int j = icocc[jj] - 1;
            const int nj = iorbs[j];
            int ka = loop;
            for (int kk = nncf[i]; kk < nncf[i] + ncf[i]; ++kk) {
                const int k = icocc[kk] - 1;
                const long long base = nijbo[(long long)j * numat + k];
                if (j == k) {
                    long long l = base;
                    for (int j1 = 0; j1 < nj; ++j1) {
                        const double sum = cocc[ja + j1 + loop];
                        for (int k1 = 0; k1 <= j1; ++k1) {
                            p[l] = p[l] + cocc[ka + k1] * sum;
                            ++l;
                        }
                    }
                } else if (j > k && base >= 0) {
                    long long l = base;
                    for (int j1 = 0; j1 < nj; ++j1) {
                        const double sum = cocc[ja + j1 + loop];
                        for (int k1 = 0; k1 < iorbs[k]; ++k1) {
                            p[l] = p[l] + cocc[ka + k1] * sum;
                            ++l;
                        }
                    }
                }
                ka += iorbs[k];
            }
            ja += nj;
        }
    }
    double spinfa;
    if (mode == 0 || mode == 1) spinfa = 2.0;
    else if (mode == -1) spinfa = -2.0;
    else spinfa = 1.0;
    if (fabs(spinfa - 1.0) > 1.0e-10)
        for (long long l = 0; l < mpack; ++l) p[l] = spinfa * p[l];
}

/* helecz (MOZYME/helecz.F90:16-52) */
double orc_mz_helecz(int numat, const int *iorbs, const long long *nijbo, const double *p, const double *h,
                     const double *f) {
    double ed = 0.0, ee = 0.0;
    for (int i = 0; i < numat; ++i) {
        for (int j = 0; j < i; ++j) {
            const long long k = nijbo[(long long)i * numat + j];
            if (k >= 0) {
                const long long l = k + (long long)iorbs[i] * iorbs[j];
                for (long long m = k; m < l; ++m) ee = ee + p[m] * (h[m] + f[m]);
            }
        }
        long long k = nijbo[(long long)i * numat + i];
        for (int l1 = 0; l1 < iorbs[i]; ++l1) {
            for (int l2 = 0; l2 < l1; ++l2) {
                ee = ee + p[k] * (h[k] + f[k]);
                ++k;
            }
            ed = ed + p[k] * (h[k] + f[k]);
            ++k;
        }
    }
    return ee + 0.5 * ed;
}

/* cnvgz (MOZYME/cnvgz.F90:16-85); idiag is 1-based like the reference's. */
void orc_mz_cnvgz(int norbs, long long mpack, double *pnew, double *p, double *p1, double *p2, double *p3,
                  int niter, const long long *idiag, int use3, double *pmax_out) {
    for (int i = 0; i < norbs; ++i) {
        const long long j = idiag[i] - 1;
        p3[i] = pnew[j];
        p2[i] = p[j];
    }
    double pmax = 0.0;
    for (long long i = 0; i < mpack; ++i) {
        const double sa = fabs(pnew[i] - p[i]);
        pmax = pmax > sa ? pmax : sa;
    }
    if (use3) {
        if (niter % 3 == 0) {
            double faca = 0.0, facb = 0.0;
            for (int i = 0; i < norbs; ++i) {
                const double sa = fabs(p3[i] - p2[i]);
                faca = faca + sa * sa;
                const double t = p3[i] - 2.0 * p2[i] + p1[i];
                facb = facb + t * t;
            }
            if (facb > 0.0 && faca < 100.0 * facb) {
                const double fac = sqrt(faca / facb);
                for (long long i = 0; i < mpack; ++i) pnew[i] = pnew[i] + fac * (pnew[i] - p[i]);
            }
        }
        if (niter > 3) {
            const double damp = 0.05;
            if (pmax > damp) {
                for (int i = 0; i < norbs; ++i) {
                    const long long j = idiag[i] - 1;
                    if (fabs(p3[i] - p2[i]) > damp) {
                        pnew[j] = p2[i] + copysign(damp, p3[i] - p2[i]);
                        const double v = pnew[j] > 0.0 ? pnew[j] : 0.0;
                        pnew[j] = v < 2.0 ? v : 2.0;
                    }
                }
            }
        }
    }
    for (int i = 0; i < norbs; ++i) p1[i] = p2[i];
    for (long long i = 0; i < mpack; ++i) p[i] = pnew[i];
    *pmax_out = pmax;
}

/* Offsets of the dense W blocks (hcore's sequential layout): pair (i, j),
 * j < i, at woff[i*numat + j], the one-centre block of i at woff[i*numat + i]. */
static void dense_w_offsets(int numat, const int *iorbs, long long *woff) {
    long long kk = 0;
    for (int i = 0; i < numat; ++i) {
        for (int j = 0; j < i; ++j) {
            woff[(long long)i * numat + j] = kk;
            const int a = iorbs[i] >= 3, b = iorbs[j] >= 3;
            kk += (a && b) ? 100 : ((a || b) ? 10 : 1);
        }
        woff[(long long)i * numat + i] = kk;
        const int il = iorbs[i] * (iorbs[i] + 1) / 2;
        kk += (long long)il * il;
    }
}

/* fz2n (MOZYME/fock2z.F90:669-1293), mode 0 (the whole F), direct and
 * semi-direct (the defaults), molecular, s/p atoms, no COSMO.  f holds H on
 * entry and F on exit, in the pair-block storage of nijbo.  The integrals of
 * a stored pair are the pair's block of the dense W (the reference computes
 * them on the fly with the same rotate), the one-centre blocks are the
 * atoms' blocks of the dense W.  Pairs outside cutof2 get the point-charge
 * monopole, and those inside cutof1 also the dipole terms; all one-centre
 * terms come after the pair loop, as in the direct path. */
void orc_mz_fock(int numat, const int *nat, const double *coord, const int *iorbs, const long long *nijbo,
                 const double *w, const double *ptot, double *f, double *qe_out) {
    static const int pidx[16] = {1, 2, 4, 7, 2, 3, 5, 8, 4, 5, 6, 9, 7, 8, 9, 10};
    long long *woff = (long long *)malloc(sizeof(long long) * (size_t)numat * numat);
    double *qe = (double *)malloc(sizeof(double) * numat);
    double *pt2 = (double *)malloc(sizeof(double) * 16 * (size_t)numat);
    dense_w_offsets(numat, iorbs, woff);
#define NB_(i, j) nijbo[(long long)(i) * numat + (j)]
    for (int i = 0; i < numat; ++i) {  /* chrge_for_MOZYME */
        long long ii = NB_(i, i);
        double sum = 0.0;
        for (int j = 1; j <= iorbs[i]; ++j) {
            ii += j;
            sum = sum + ptot[ii - 1];
        }
        qe[i] = sum;
        const long long b = NB_(i, i);
        int m = 0;
        for (int j = 1; j <= iorbs[i]; ++j)
            for (int k = 1; k <= iorbs[i]; ++k) {
                const int jk = j < k ? j : k, kj = j + k - jk;
                pt2[16 * i + m] = ptot[b + (kj * (kj - 1)) / 2 + jk - 1];
                ++m;
            }
    }
    double w2 = 0.0, w3 = 0.0, w4 = 0.0, w5 = 0.0, w6 = 0.0, w7 = 0.0;
    for (int ii = 0; ii < numat; ++ii) {
        const int iab = iorbs[ii];
        if (iab == 0) continue;
        for (int jj = 0; jj < ii; ++jj) {
            const int jba = iorbs[jj];
            const long long off = NB_(ii, jj);
            if (off >= 0) {
                const double *wk = w + woff[(long long)ii * numat + jj];
                if (iab >= 3 && jba >= 3) {
                    /* jab_for_MOZYME(1, 1, ptot2(ii), ptot2(jj), w, F(ii ii), F(jj jj)) */
                    double suma[10], sumb[10];
                    for (int i = 0; i < 10; ++i) { suma[i] = 0.0; sumb[i] = 0.0; }
                    for (int j = 0; j < 16; ++j)
                        for (int i = 0; i < 10; ++i) {
                            suma[i] = suma[i] + pt2[16 * ii + j] * wk[(pidx[j] - 1) * 10 + i];
                            sumb[i] = sumb[i] + pt2[16 * jj + j] * wk[i * 10 + pidx[j] - 1];
                        }
                    const long long fi = NB_(ii, ii), fj = NB_(jj, jj);
                    int i = 0;
                    for (int i5 = 1; i5 <= 4; ++i5) {
                        long long ioff = (i5 * (i5 - 1)) / 2, joff = ioff;
                        for (int i6 = 1; i6 <= i5; ++i6) {
                            ++ioff; ++joff;
                            f[fi + ioff - 1] = f[fi + ioff - 1] + sumb[i];
                            f[fj + joff - 1] = f[fj + joff - 1] + suma[i];
                            ++i;
                        }
                    }
                    /* kab_for_MOZYME(0, 0, ptot(l), w, f(l)) */
                    double sum[16];
                    for (int j = 0; j < 16; ++j) {
                        const int mu = j / 4 + 1, nu = j % 4 + 1;
                        sum[j] = 0.0;
                        for (int i2 = 0; i2 < 16; ++i2) {
                            const int lam = i2 / 4 + 1, sig = i2 % 4 + 1;
                            sum[j] = sum[j] + ptot[off + i2] * wk[(indx_(mu, lam) - 1) * 10 + indx_(nu, sig) - 1];
                        }
                    }
                    for (int i2 = 0; i2 < 16; ++i2) f[off + i2] = f[off + i2] - sum[i2] * 0.5;
                } else if (iab >= 3 && jba == 1) {
                    double sumdia = 0.0, sumoff = 0.0;
                    const long long lj = NB_(jj, jj) + 1;
                    long long li = NB_(ii, ii);
                    int k = 0;
                    for (int i = 1; i <= 4; ++i) {
                        for (int j = 1; j <= i - 1; ++j) {
                            ++li; ++k;
                            f[li - 1] = f[li - 1] + ptot[lj - 1] * wk[k - 1];
                            sumoff = sumoff + ptot[li - 1] * wk[k - 1];
                        }
                        ++li; ++k;
                        f[li - 1] = f[li - 1] + ptot[lj - 1] * wk[k - 1];
                        sumdia = sumdia + ptot[li - 1] * wk[k - 1];
                    }
                    f[lj - 1] = f[lj - 1] + sumoff * 2.0 + sumdia;
                    k = 0;
                    for (int i = 1; i <= 4; ++i) {
                        double s = 0.0;
                        for (int j = 1; j <= 4; ++j) {
                            ++k;
                            s = s + ptot[off + j - 1] * wk[pidx[k - 1] - 1];
                        }
                        f[off + i - 1] = f[off + i - 1] - s * 0.5;
                    }
                } else if (jba >= 3 && iab == 1) {
                    double sumdia = 0.0, sumoff = 0.0;
                    long long lj = NB_(jj, jj);
                    const long long li = NB_(ii, ii) + 1;
                    int k = 0;
                    for (int i = 1; i <= 4; ++i) {
                        for (int j = 1; j <= i - 1; ++j) {
                            ++k; ++lj;
                            f[lj - 1] = f[lj - 1] + ptot[li - 1] * wk[k - 1];
                            sumoff = sumoff + ptot[lj - 1] * wk[k - 1];
                        }
                        ++lj; ++k;
                        f[lj - 1] = f[lj - 1] + ptot[li - 1] * wk[k - 1];
                        sumdia = sumdia + ptot[lj - 1] * wk[k - 1];
                    }
                    f[li - 1] = f[li - 1] + sumoff * 2.0 + sumdia;
                    k = 0;
                    for (int i = 1; i <= 4; ++i) {
                        double s = 0.0;
                        for (int j = 1; j <= 4; ++j) {
                            ++k;
                            s = s + ptot[off + j - 1] * wk[pidx[k - 1] - 1];
                        }
                        f[off + i - 1] = f[off + i - 1] - s * 0.5;
                    }
                } else if (iab == 1 && jba == 1) {
                    const long long lii = NB_(ii, ii) + 1, lij = off + 1, ljj = NB_(jj, jj) + 1;
                    f[lii - 1] = f[lii - 1] + ptot[ljj - 1] * wk[0];
                    f[ljj - 1] = f[ljj - 1] + ptot[lii - 1] * wk[0];
                    f[lij - 1] = f[lij - 1] - ptot[lij - 1] * wk[0] * 0.5;
                }
            } else {
                long long i1 = NB_(ii, ii), j1 = NB_(jj, jj);
                double dx = coord[3 * ii] - coord[3 * jj];
                double dy = coord[3 * ii + 1] - coord[3 * jj + 1];
                double dz = coord[3 * ii + 2] - coord[3 * jj + 2];
                const double r2 = dx * dx + dy * dy + dz * dz;
                const int ni = nat[ii], nj = nat[jj];
                const double aee = 0.5 / E[ni].am + 0.5 / E[nj].am;
                double point, cst;
                const double rij = sqrt(r2);
                to_point(rij, &point, &cst);
                double w1 = EV / sqrt(r2 / (A0 * A0) + aee * aee);
                w1 = w1 * cst + (1.0 - cst) * point;
                for (int i = 1; i <= iab; ++i) {
                    i1 += i;
                    f[i1 - 1] = f[i1 - 1] + qe[jj] * w1;
                }
                for (int j = 1; j <= jba; ++j) {
                    j1 += j;
                    f[j1 - 1] = f[j1 - 1] + qe[ii] * w1;
                }
                i1 = NB_(ii, ii);
                j1 = NB_(jj, jj);
                if (off == -2) {
                    const double r = sqrt(r2);
                    dx = dx / r; dy = dy / r; dz = dz / r;
                    if (fabs(dz) > 0.99999999) dz = copysign(1.0, dz);
                    if (iab > 1) {
                        const double da = E[ni].dd, ade = 0.5 / E[ni].ad + 0.5 / E[nj].am;
                        const double rp = sqrt((r / A0 + da) * (r / A0 + da) + ade * ade);
                        const double rm = sqrt((r / A0 - da) * (r / A0 - da) + ade * ade);
                        double ri2 = EV * (0.5 / rp - 0.5 / rm);
                        to_point(r, &point, &cst);
                        ri2 = ri2 * cst;
                        w5 = ri2 * dx; w6 = ri2 * dy; w7 = ri2 * dz;
                    }
                    if (jba > 1) {
                        const double da = E[nj].dd, ade = 0.5 / E[ni].am + 0.5 / E[nj].ad;
                        const double rp = sqrt((r / A0 + da) * (r / A0 + da) + ade * ade);
                        const double rm = sqrt((r / A0 - da) * (r / A0 - da) + ade * ade);
                        double ri5 = -EV * (0.5 / rp - 0.5 / rm);
                        to_point(r, &point, &cst);
                        ri5 = ri5 * cst;
                        w2 = ri5 * dx; w3 = ri5 * dy; w4 = ri5 * dz;
                    }
#define FA(x) f[(x) - 1]
#define PA(x) ptot[(x) - 1]
                    if (iab > 1 && jba > 1) {
                        FA(j1 + 2) = FA(j1 + 2) + qe[ii] * w2;
                        FA(j1 + 4) = FA(j1 + 4) + qe[ii] * w3;
                        FA(j1 + 7) = FA(j1 + 7) + qe[ii] * w4;
                        FA(i1 + 2) = FA(i1 + 2) + qe[jj] * w5;
                        FA(i1 + 4) = FA(i1 + 4) + qe[jj] * w6;
                        FA(i1 + 7) = FA(i1 + 7) + qe[jj] * w7;
                        const int dg[4] = {1, 3, 6, 10};
                        for (int q = 0; q < 4; ++q) FA(j1 + dg[q]) = FA(j1 + dg[q]) + PA(i1 + 2) * w5 * 2;
                        for (int q = 0; q < 4; ++q) FA(j1 + dg[q]) = FA(j1 + dg[q]) + PA(i1 + 4) * w6 * 2;
                        for (int q = 0; q < 4; ++q) FA(j1 + dg[q]) = FA(j1 + dg[q]) + PA(i1 + 7) * w7 * 2;
                        for (int q = 0; q < 4; ++q) FA(i1 + dg[q]) = FA(i1 + dg[q]) + PA(j1 + 2) * w2 * 2;
                        for (int q = 0; q < 4; ++q) FA(i1 + dg[q]) = FA(i1 + dg[q]) + PA(j1 + 4) * w3 * 2;
                        for (int q = 0; q < 4; ++q) FA(i1 + dg[q]) = FA(i1 + dg[q]) + PA(j1 + 7) * w4 * 2;
                    } else if (iab > 1) {
                        FA(i1 + 2) = FA(i1 + 2) + qe[jj] * w5;
                        FA(i1 + 4) = FA(i1 + 4) + qe[jj] * w6;
                        FA(i1 + 7) = FA(i1 + 7) + qe[jj] * w7;
                        FA(j1 + 1) = FA(j1 + 1) + PA(i1 + 2) * w5 * 2;
                        FA(j1 + 1) = FA(j1 + 1) + PA(i1 + 4) * w6 * 2;
                        FA(j1 + 1) = FA(j1 + 1) + PA(i1 + 7) * w7 * 2;
                    } else if (jba > 1) {
                        FA(j1 + 2) = FA(j1 + 2) + qe[ii] * w2;
                        FA(j1 + 4) = FA(j1 + 4) + qe[ii] * w3;
                        FA(j1 + 7) = FA(j1 + 7) + qe[ii] * w4;
                        FA(i1 + 1) = FA(i1 + 1) + PA(j1 + 2) * w2 * 2;
                        FA(i1 + 1) = FA(i1 + 1) + PA(j1 + 4) * w3 * 2;
                        FA(i1 + 1) = FA(i1 + 1) + PA(j1 + 7) * w4 * 2;
                    }
#undef FA
#undef PA
                }
            }
        }
    }
    /* fock1_for_MOZYME for every atom, after the pairs (direct path) */
    for (int ii = 0; ii < numat; ++ii) {
        const int iab = iorbs[ii];
        if (iab == 0) continue;
        const int ilim = iab * (iab + 1) / 2;
        const double *wo = w + woff[(long long)ii * numat + ii];
        const long long base = NB_(ii, ii);
#define WF(a, b) wo[((a) - 1) + ilim * ((b) - 1)]
        for (int i = 1; i <= iab; ++i)
            for (int j = 1; j <= i; ++j) {
                const int ij = (i * (i - 1)) / 2 + j, ijw = ij;
                double sum = 0.0;
                for (int k = 1; k <= iab; ++k)
                    for (int l = 1; l <= iab; ++l) {
                        const int ip = k > l ? k : l, jp = k < l ? k : l;
                        const int ijp = (ip * (ip - 1)) / 2 + jp;
                        const int klw = ijp;
                        int im = k > j ? k : j, jm = k < j ? k : j;
                        const int ikw = (im * (im - 1)) / 2 + jm;
                        im = l > i ? l : i; jm = l < i ? l : i;
                        const int jlw = (im * (im - 1)) / 2 + jm;
                        sum = sum + ptot[base + ijp - 1] * WF(ijw, klw) - 0.5 * ptot[base + ijp - 1] * WF(ikw, jlw);
                    }
                f[base + ij - 1] = f[base + ij - 1] + sum;
            }
#undef WF
    }
#undef NB_
    if (qe_out)
        for (int i = 0; i < numat; ++i) qe_out[i] = qe[i];
    free(woff);
    free(qe);
    free(pt2);
}

/* diagg1 (MOZYME/diagg1.F90:16-503), lijbo path, s/p atoms.  LMO arrays as in
 * MOZYME_C with 0-based starts (nncf, ncocc, nnce, ncvir) and 1-based atom
 * numbers (icocc, icvir); first[a] is the 0-based first orbital of atom a.
 * st[0..3] = fref, safety, oldlim, tiny of the previous call (in/out); the
 * interaction list (ifmo as pairs of 1-based LMO numbers, fmo) and nfmo are
 * in/out like the reference's saved arrays; *nij: capacity in, count out.
 * eigv (virtual LMO energies) out; eigs (occupied) out when recomputed.
 * Returns sumt. */
double orc_mz_diagg1(int numat, const int *iorbs, const int *first, int norbs, const long long *nijbo,
                     const double *fao, const double *p, int nocc, const int *ncf, const int *nncf, const int *icocc,
                     const int *ncocc, const double *cocc, int nvir, const int *nce, const int *nnce,
                     const int *icvir, const int *ncvir, const double *cvir, int idiagg, double *st, int *nfmo,
                     int *ifmo, double *fmo, long long *nij_io, double *eigv, double *eigs, int *eigs_done) {
#define NB_(i, j) nijbo[(long long)(i) * numat + (j)]
    double fref = st[0], safety = st[1], oldlim = st[2], tiny = st[3];
    const long long nij = *nij_io;
    int ncocc_tot = 0;
    for (int j = 0; j < nocc; ++j) ncocc_tot = nncf[j] + ncf[j] > ncocc_tot ? nncf[j] + ncf[j] : ncocc_tot;
    double *aocc = (double *)calloc((size_t)ncocc_tot + 1, sizeof(double));
    double *avir = (double *)calloc((size_t)numat, sizeof(double));
    double *aov = (double *)calloc((size_t)numat, sizeof(double));
    double *ws = (double *)calloc((size_t)norbs, sizeof(double));
    char *latoms = (char *)calloc((size_t)numat, 1);
    for (int j = 0; j < nocc; ++j) {
        const int loopj = ncocc[j];
        int kl = 0;
        for (int kk = nncf[j]; kk < nncf[j] + ncf[j]; ++kk) {
            const int k1 = icocc[kk] - 1;
            double sum = 0.0;
            for (int k = 0; k < iorbs[k1]; ++k) {
                ++kl;
                sum = sum + cocc[kl + loopj - 1] * cocc[kl + loopj - 1];
            }
            aocc[kk] = sum;
        }
    }
    const double cutlim = 1.0e-8;
    double cutoff = cutlim > tiny * 10.0 * cutlim ? cutlim : tiny * 10.0 * cutlim;
    const double flim = 3.0 < fref * 0.5 ? 3.0 : fref * 0.5;
    fref = 0.0;
    if (idiagg <= 5) cutoff = cutlim;
    double sumt = 0.0;
    long long ijc = 0;
    tiny = 0.0;
    for (int i = 0; i < nvir; ++i) {
        const int loopi = ncvir[i];
        for (int a = 0; a < numat; ++a) latoms[a] = 0;
        int l = 0;
        for (int j = nnce[i]; j < nnce[i] + nce[i]; ++j) {
            const int j1 = icvir[j] - 1;
            double sum = 0.0;
            for (int k = l + 1; k <= l + iorbs[j1]; ++k) sum = sum + cvir[k + loopi - 1] * cvir[k + loopi - 1];
            l += iorbs[j1];
            avir[j1] = sum;
            latoms[j1] = 1;
        }
        for (int jj = nnce[i]; jj < nnce[i] + nce[i]; ++jj) {
            const int j1 = icvir[jj] - 1;
            for (int jx = 1; jx <= iorbs[j1]; ++jx) ws[first[j1] + jx - 1] = 0.0;
            int kl = loopi;
            for (int kk = nnce[i]; kk < nnce[i] + nce[i]; ++kk) {
                const int k1 = icvir[kk] - 1;
                const long long kj = NB_(k1, j1);
                if (kj >= 0 && avir[k1] * p[kj] > cutoff) {
                    if (iorbs[k1] == 1 && iorbs[j1] == 1) {
                        ws[first[j1]] = ws[first[j1]] + fao[kj] * cvir[kl];
                    } else if (k1 > j1) {
                        long long ii = kj;
                        for (int i4 = 1; i4 <= iorbs[k1]; ++i4)
                            for (int jx = 1; jx <= iorbs[j1]; ++jx) {
                                ++ii;
                                ws[first[j1] + jx - 1] = ws[first[j1] + jx - 1] + fao[ii - 1] * cvir[kl + i4 - 1];
                            }
                    } else if (k1 < j1) {
                        long long ii = kj;
                        for (int jx = 1; jx <= iorbs[j1]; ++jx)
                            for (int i4 = 1; i4 <= iorbs[k1]; ++i4) {
                                ++ii;
                                ws[first[j1] + jx - 1] = ws[first[j1] + jx - 1] + fao[ii - 1] * cvir[kl + i4 - 1];
                            }
                    } else {
                        for (int jx = 1; jx <= iorbs[j1]; ++jx)
                            for (int i4 = 1; i4 <= iorbs[j1]; ++i4) {
                                const long long ii = i4 > jx ? kj + (i4 * (i4 - 1)) / 2 + jx : kj + (jx * (jx - 1)) / 2 + i4;
                                ws[first[j1] + jx - 1] = ws[first[j1] + jx - 1] + fao[ii - 1] * cvir[kl + i4 - 1];
                            }
                    }
                }
                kl += iorbs[k1];
            }
        }
        for (int j = 0; j < numat; ++j) {
            if (latoms[j]) {
                double sum = 0.0;
                for (int k = first[j]; k < first[j] + iorbs[j]; ++k) sum = sum + ws[k] * ws[k];
                aov[j] = sum;
            } else {
                aov[j] = 0.0;
            }
        }
        {
            double sum = 0.0;
            int kl = loopi;
            for (int kk = nnce[i]; kk < nnce[i] + nce[i]; ++kk) {
                const int k1 = icvir[kk] - 1;
                if (aov[k1] * avir[k1] > cutoff) {
                    for (int k = first[k1]; k < first[k1] + iorbs[k1]; ++k) {
                        ++kl;
                        sum = sum + ws[k] * cvir[kl - 1];
                    }
                } else {
                    kl += iorbs[k1];
                }
            }
            eigv[i] = sum;
        }
        if (idiagg <= 5 || idiagg % 2 == 0) {
            int nf = 0;
            const int i1 = icvir[nnce[i]] - 1;
            const int i2 = nce[i] > 1 ? icvir[nnce[i] + 1] - 1 : i1;
            for (int j = 0; j < nocc; ++j) {
                if (ijc == nij) continue;
                const int j1 = icocc[nncf[j]] - 1;
                const int j2 = ncf[j] > 1 ? icocc[nncf[j] + 1] - 1 : j1;
                const long long a11 = NB_(i1, j1), a12 = NB_(i1, j2), a21 = NB_(i2, j1), a22 = NB_(i2, j2);
                if (a11 >= 0 || a12 >= 0 || a21 >= 0 || a22 >= 0) {
                    double sum = 0.0;
                    if (a11 >= 0) sum = fabs(fao[a11]);
                    if (a12 >= 0) sum = sum + fabs(fao[a12]);
                    if (a21 >= 0) sum = sum + fabs(fao[a21]);
                    if (a22 >= 0) sum = sum + fabs(fao[a22]);
                    if (sum >= flim) {
                        const int loopj = ncocc[j];
                        int lij = 0, kl = 0;
                        sum = 0.0;
                        for (int kk = nncf[j]; kk < nncf[j] + ncf[j]; ++kk) {
                            const int k1 = icocc[kk] - 1;
                            if (aocc[kk] * aov[k1] < cutoff || !latoms[k1]) {
                                kl += iorbs[k1];
                            } else {
                                lij = 1;
                                for (int k = first[k1]; k < first[k1] + iorbs[k1]; ++k) {
                                    ++kl;
                                    sum = sum + ws[k] * cocc[kl + loopj - 1];
                                }
                            }
                        }
                        sumt = sumt + fabs(sum);
                        tiny = tiny > fabs(sum) ? tiny : fabs(sum);
                        if (lij && fabs(sum) > oldlim) {
                            ++nf;
                            ifmo[2 * ijc] = i + 1;
                            ifmo[2 * ijc + 1] = j + 1;
                            fmo[ijc] = sum;
                            ++ijc;
                        }
                    }
                }
            }
            nfmo[i] = nf;
        } else {
            const long long ij0 = ijc;
            for (int jj = 1; jj <= nfmo[i]; ++jj) {
                if (ijc == nij) break;
                const int j = ifmo[2 * (ij0 + jj - 1) + 1] - 1;
                const int loopj = ncocc[j];
                double sum = 0.0;
                int kl = 0;
                for (int kk = nncf[j]; kk < nncf[j] + ncf[j]; ++kk) {
                    const int k1 = icocc[kk] - 1;
                    if (aov[k1] * aocc[kk] < cutoff || !latoms[k1]) {
                        kl += iorbs[k1];
                    } else {
                        for (int k = first[k1]; k < first[k1] + iorbs[k1]; ++k) {
                            ++kl;
                            sum = sum + ws[k] * cocc[kl + loopj - 1];
                        }
                    }
                }
                sumt = sumt + fabs(sum);
                tiny = tiny > fabs(sum) ? tiny : fabs(sum);
                fmo[ijc] = sum;
                ++ijc;
            }
        }
    }
    if (ijc == nij) safety = safety * 2.0;
    else safety = safety * 0.5 > 1.0 ? safety * 0.5 : 1.0;
    *nij_io = ijc;
    *eigs_done = 0;
    if (idiagg > 2 && idiagg % 4 != 0) {
        const double t2 = tiny * tiny;  /* tiny**4 as gfortran expands it: (t t)(t t) */
        fref = t2 * t2;
    } else {
        for (int i = 0; i < nocc; ++i) {
            const int loopi = ncocc[i];
            int l = 0;
            for (int j = nncf[i]; j < nncf[i] + ncf[i]; ++j) {
                const int j1 = icocc[j] - 1;
                double sum = 0.0;
                for (int k = l + 1; k <= l + iorbs[j1]; ++k) sum = sum + cocc[k + loopi - 1] * cocc[k + loopi - 1];
                l += iorbs[j1];
                avir[j1] = sum;
            }
            double sum = 0.0;
            int jl = loopi;
            for (int j = nncf[i]; j < nncf[i] + ncf[i]; ++j) {
                const int j1 = icocc[j] - 1;
                int kl = loopi;
                for (int k = nncf[i]; k < nncf[i] + ncf[i]; ++k) {
                    const int k1 = icocc[k] - 1;
                    const long long k1j1 = NB_(k1, j1);
                    if (k1j1 >= 0 && avir[k1] * p[k1j1] * aocc[k] >= cutoff) {
                        for (int jx = 1; jx <= iorbs[j1]; ++jx) {
                            double sum1 = 0.0;
                            if (k1 > j1) {
                                for (int i4 = 1; i4 <= iorbs[k1]; ++i4)
                                    sum1 = sum1 + fao[k1j1 + (long long)(i4 - 1) * iorbs[j1] + jx - 1] * cocc[kl + i4 - 1];
                            } else if (k1 < j1) {
                                for (int i4 = 1; i4 <= iorbs[k1]; ++i4)
                                    sum1 = sum1 + fao[k1j1 + (long long)(jx - 1) * iorbs[k1] + i4 - 1] * cocc[kl + i4 - 1];
                            } else {
                                for (int j4 = 1; j4 <= jx; ++j4)
                                    sum1 = sum1 + fao[k1j1 + (jx * (jx - 1)) / 2 + j4 - 1] * cocc[kl + j4 - 1];
                                for (int i4 = jx + 1; i4 <= iorbs[k1]; ++i4)
                                    sum1 = sum1 + fao[k1j1 + (i4 * (i4 - 1)) / 2 + jx - 1] * cocc[kl + i4 - 1];
                            }
                            sum = sum + cocc[jl + jx - 1] * sum1;
                        }
                    }
                    kl += iorbs[k1];
                }
                jl += iorbs[j1];
            }
            eigs[i] = sum;
        }
        oldlim = tiny * safety * 1.0e-3;
        const double t2 = tiny * tiny;
        fref = t2 * t2;
        *eigs_done = 1;
    }
    st[0] = fref;
    st[1] = safety;
    st[2] = oldlim;
    st[3] = tiny;
    free(aocc); free(avir); free(aov); free(ws); free(latoms);
#undef NB_
    return sumt;
}

/* diagg2 (MOZYME/diagg2.F90:16-359): the 2x2 rotations of the interaction
 * list in order, growing an LMO by an atom whose new coefficients exceed
 * thresh and rejecting (restoring both LMOs) a rotation that would overflow
 * their space.  LMO arrays 0-based starts as in orc_mz_diagg1; nncf/ncocc
 * (nnce/ncvir) of LMO k+1 bound LMO k's space, icocc_dim/cocc_dim
 * (icvir_dim/cvir_dim) the last one's.  ctl[0..4] = const (damping), shift,
 * thresh, tiny (diagg1's, in: scaled here as the reference does), bigeps;
 * nrejct[2] saved between calls.  eigs: occupied LMO energies, eigv: virtual.
 * Returns sumb (sum of |beta|). */
double orc_mz_diagg2(int numat, const int *iorbs, int norbs, int nocc, int *ncf, const int *nncf, int *icocc,
                     const int *ncocc, double *cocc, long long icocc_dim, long long cocc_dim, int nvir, int *nce,
                     const int *nnce, int *icvir, const int *ncvir, double *cvir, long long icvir_dim,
                     long long cvir_dim, const int *ifmo, const double *fmo, long long nij, const double *eigs,
                     const double *eigv, int idiagg, const double *ctl, int *nrejct, long long *nrej_out) {
    const double cst = ctl[0], shift = ctl[1], thresh = ctl[2], bigeps = ctl[4];
    double tiny = ctl[3], biglim;
    const int retry = (nrejct[0] == nrejct[1] && nrejct[0] != 0 && nrejct[0] < 20);
    if (idiagg % 5 == 0 || idiagg <= 5) {
        tiny = -1.0;
        biglim = -1.0;
    } else {
        tiny = 0.01 * tiny;
        biglim = bigeps;
    }
    int *iused = (int *)malloc(sizeof(int) * numat);
    char *latoms = (char *)calloc(numat, 1);
    double *storei = (double *)malloc(sizeof(double) * norbs);
    double *storej = (double *)malloc(sizeof(double) * norbs);
    for (int a = 0; a < numat; ++a) iused[a] = -1;
    double sumb = 0.0;
    long long nrej = 0;
    for (long long ij = 0; ij < nij; ++ij) {
        const int i = ifmo[2 * ij] - 1, j = ifmo[2 * ij + 1] - 1;
        if (!(fabs(fmo[ij]) >= tiny)) continue;
        const double c = fmo[ij] * cst;
        const double d = eigs[j] - eigv[i] - shift;
        if (!(fabs(c / d) >= biglim)) continue;
        const int ncfj = ncf[j], ncei = nce[i];
        const long long jlr = ncocc[j] + 1;  /* 1-based, as the reference */
        long long jur, jncf;
        if (j != nocc - 1) { jur = ncocc[j + 1]; jncf = nncf[j + 1]; } else { jur = cocc_dim; jncf = icocc_dim; }
        jur = jlr + norbs - 1 < jur ? jlr + norbs - 1 : jur;
        const long long ilr = ncvir[i] + 1;
        long long iur, incv;
        if (i != nvir - 1) { iur = ncvir[i + 1]; incv = nnce[i + 1]; } else { iur = cvir_dim; incv = icvir_dim; }
        iur = ilr + norbs - 1 < iur ? ilr + norbs - 1 : iur;
        for (long long k = jlr, l = 0; k <= jur; ++k, ++l) storej[l] = cocc[k - 1];
        for (long long k = ilr, l = 0; k <= iur; ++k, ++l) storei[l] = cvir[k - 1];
        const double e = copysign(sqrt(4.0 * c * c + d * d), d);
        double alpha = sqrt(0.5 * (1.0 + d / e));
        for (;;) {
            const double beta = -copysign(sqrt(1.0 - alpha * alpha), c);
            sumb = sumb + fabs(beta);
            int mlf = 0, rejected = 0;
            for (int lf = nncf[j]; lf < nncf[j] + ncf[j]; ++lf) {
                const int ii = icocc[lf] - 1;
                iused[ii] = mlf;
                mlf += iorbs[ii];
            }
            const long long loopi = ncvir[i], loopj = ncocc[j];
            long long mle = 0;
            for (int le = nnce[i]; le < nnce[i] + nce[i] && !rejected; ++le) {
                const int mie = icvir[le] - 1;
                latoms[mie] = 1;
                long long mlff = iused[mie] + loopj;
                if (iused[mie] >= 0) {
                    for (long long mlee = mle + 1 + loopi; mlee <= mle + iorbs[mie] + loopi; ++mlee) {
                        ++mlff;
                        const double a = cocc[mlff - 1], b = cvir[mlee - 1];
                        cocc[mlff - 1] = alpha * a + beta * b;
                        cvir[mlee - 1] = alpha * b - beta * a;
                    }
                } else {
                    double sum = 0.0;
                    for (long long mlee = mle + 1 + loopi; mlee <= mle + iorbs[mie] + loopi; ++mlee) {
                        const double t = beta * cvir[mlee - 1];
                        sum = sum + t * t;
                    }
                    if (sum > thresh) {
                        if (nncf[j] + ncf[j] >= jncf || mlf + iorbs[mie] + loopj > jur) { rejected = 1; break; }
                        ncf[j] = ncf[j] + 1;
                        icocc[nncf[j] + ncf[j] - 1] = mie + 1;
                        iused[mie] = mlf;
                        mlf += iorbs[mie];
                        mlff = iused[mie] + loopj;
                        for (long long mlee = mle + 1 + loopi; mlee <= mle + iorbs[mie] + loopi; ++mlee) {
                            ++mlff;
                            cocc[mlff - 1] = beta * cvir[mlee - 1];
                            cvir[mlee - 1] = alpha * cvir[mlee - 1];
                        }
                    }
                }
                mle += iorbs[mie];
            }
            if (!rejected) {
                for (int lf = nncf[j]; lf < nncf[j] + ncf[j]; ++lf) {
                    const int ii = icocc[lf] - 1;
                    if (latoms[ii]) continue;
                    double sum = 0.0;
                    for (long long mlff = iused[ii] + loopj + 1; mlff <= iused[ii] + loopj + iorbs[ii]; ++mlff) {
                        const double t = beta * cocc[mlff - 1];
                        sum = sum + t * t;
                    }
                    if (sum > thresh) {
                        if (nnce[i] + nce[i] >= incv || mle + iorbs[ii] + loopi > iur) { rejected = 1; break; }
                        nce[i] = nce[i] + 1;
                        icvir[nnce[i] + nce[i] - 1] = ii + 1;
                        latoms[ii] = 1;
                        long long mlff = iused[ii] + loopj;
                        for (long long mlee = mle + 1 + loopi; mlee <= mle + iorbs[ii] + loopi; ++mlee) {
                            ++mlff;
                            cvir[mlee - 1] = -beta * cocc[mlff - 1];
                            cocc[mlff - 1] = alpha * cocc[mlff - 1];
                        }
                        mle += iorbs[ii];
                    }
                }
            }
            if (!rejected) break;
            /* label 1000 */
            ++nrej;
            for (long long k = jlr, l = 0; k <= jur; ++k, ++l) cocc[k - 1] = storej[l];
            for (long long k = ilr, l = 0; k <= iur; ++k, ++l) cvir[k - 1] = storei[l];
            ncf[j] = ncfj;
            nce[i] = ncei;
            for (int k = 0; k < numat; ++k) { iused[k] = -1; latoms[k] = 0; }
            if (retry) {
                alpha = 0.5 * (alpha + 1.0);
            } else {
                goto next_ij;
            }
        }
        for (int le = nnce[i]; le < nnce[i] + nce[i]; ++le) latoms[icvir[le] - 1] = 0;
        for (int lf = nncf[j]; lf < nncf[j] + ncf[j]; ++lf) iused[icocc[lf] - 1] = -1;
    next_ij:;
    }
    nrejct[1] = nrejct[0];
    nrejct[0] = (int)nrej;
    *nrej_out = nrej;
    free(iused); free(latoms); free(storei); free(storej);
    return sumb;
}

/* ------------------------------------------------------------------ */
/* hcore_for_MOZYME (MOZYME/hcore_for_MOZYME.F90), molecular (id = 0),   */
/* mode 0, no field: H and W on fillij's pair-block storage.             */
/* ------------------------------------------------------------------ */
/* outer1 (MOZYME/outer1.F90, mode 0): pairs beyond cutof1, a feathered
 * point charge; e1b/e2a: packed local diagonal (10 for sp). */
static double outer1_pair(int ni, int nj, const double *ci, const double *cj, double *e1b, double *e2a) {
  double rij = sqrt((ci[0] - cj[0]) * (ci[0] - cj[0]) + (ci[1] - cj[1]) * (ci[1] - cj[1]) +
                    (ci[2] - cj[2]) * (ci[2] - cj[2]));
  double r = rij / A0;
  double aee = 0.5 / E[ni].am + 0.5 / E[nj].am;
  aee = aee * aee;
  double ww = EV / sqrt(r * r + aee);
  double point, cst;
  to_point(rij, &point, &cst);              /* l_feather: PM7 */
  ww = ww * cst + (1.0 - cst) * point;
  for (int k = 0; k < 10; ++k) { e1b[k] = 0.0; e2a[k] = 0.0; }
  static const int dg[4] = {0, 2, 5, 9};
  for (int k = 0; k < 4; ++k) {
    e1b[dg[k]] = -ww * E[nj].tore;
    e2a[dg[k]] = -ww * E[ni].tore;
  }
  return E[ni].tore * E[nj].tore * ww;
}

/* outer2 (MOZYME/outer2.F90, mode 0): pairs between cutof2 and cutof1,
 * monopole and dipole terms from reppd along the unit vector j -> i. */
static double outer2_pair(int ni, int nj, const double *ci, const double *cj, double *e1b, double *e2a) {
  double x[3] = {ci[0] - cj[0], ci[1] - cj[1], ci[2] - cj[2]};
  double rij = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  double ri[23], gab;
  reppd(ni, nj, rij, ri, &gab);
  double a = 1.0 / rij;
  x[0] *= a; x[1] *= a; x[2] *= a;
  if (fabs(x[2]) > 0.99999999) x[2] = x[2] >= 0.0 ? 1.0 : -1.0;
  int si = E[ni].natorb > 1, sj = E[nj].natorb > 1;
  double w1 = ri[1];
  for (int k = 0; k < 10; ++k) { e1b[k] = 0.0; e2a[k] = 0.0; }
  e1b[0] = -w1 * E[nj].tore;
  e2a[0] = -w1 * E[ni].tore;
  if (sj) {
    double w2 = -ri[5] * x[0], w3 = -ri[5] * x[1], w4 = -ri[5] * x[2];
    e2a[1] = -w2 * E[ni].tore; e2a[2] = -w1 * E[ni].tore; e2a[3] = -w3 * E[ni].tore;
    e2a[5] = -w1 * E[ni].tore; e2a[6] = -w4 * E[ni].tore; e2a[9] = -w1 * E[ni].tore;
  }
  if (si) {
    double w5 = -ri[2] * x[0], w6 = -ri[2] * x[1], w7 = -ri[2] * x[2];
    e1b[1] = -w5 * E[nj].tore; e1b[2] = -w1 * E[nj].tore; e1b[3] = -w6 * E[nj].tore;
    e1b[5] = -w1 * E[nj].tore; e1b[6] = -w7 * E[nj].tore; e1b[9] = -w1 * E[nj].tore;
  }
  return E[ni].tore * E[nj].tore * w1;
}

/* H on the pair blocks (mpack from orc_mz_layout, nijbo from it too), W of
 * the stored pairs in the dense W's order (pairs at or beyond cutof2 left
 * out; the Fock build treats them through the coordinates), enuclr over all
 * pairs.  Returns the number of W values written. */
long long orc_mz_hcore(int numat, const int *nat, const double *coord, const long long *nijbo, double *h,
                       double *w, double *enuclr_out) {
  init_params();
  double enuclr = 0.0;
  const double cutof1 = 225.0;  /* h1elec's overlap cutoff, as the dense hcore */
  long long kr = 0, mp = 0;
  for (int i = 0; i < numat; ++i) {
    long long o = nijbo[(long long)i * numat + i] + E[nat[i]].natorb * (E[nat[i]].natorb + 1) / 2;
    if (o > mp) mp = o;
  }
  for (long long q = 0; q < mp; ++q) h[q] = 0.0;
  for (int i = 0; i < numat; ++i) {
    const int ni = nat[i], io = E[ni].natorb;
    const long long di = nijbo[(long long)i * numat + i];
    for (int a = 0; a < io; ++a) h[di + (long long)a * (a + 1) / 2 + a] = a == 0 ? E[ni].uss : E[ni].upp;
    const double *xi = coord + 3 * i;
    for (int j = 0; j < i; ++j) {
      const int nj = nat[j], jo = E[nj].natorb;
      const double *xj = coord + 3 * j;
      const long long bo = nijbo[(long long)i * numat + j];
      double e1b[10], e2a[10], enuc;
      if (bo >= 0) {
        double dm[5][5];
        h1elec(ni, nj, xi, xj, dm, cutof1);
        for (int a = 0; a < io; ++a)
          for (int b = 0; b < jo; ++b) h[bo + (long long)a * jo + b] = h[bo + (long long)a * jo + b] + dm[a + 1][b + 1];
        enuc = rotate_pair(ni, nj, xi, xj, w + kr, e1b, e2a);
        kr += (long long)indx_(io, io) * indx_(jo, jo);
      } else if (bo == -2) {
        enuc = outer2_pair(ni, nj, xi, xj, e1b, e2a);
      } else {
        enuc = outer1_pair(ni, nj, xi, xj, e1b, e2a);
      }
      enuclr = enuclr + enuc;
      const long long dj = nijbo[(long long)j * numat + j];
      for (int m = 0; m < indx_(io, io); ++m) h[di + m] = h[di + m] + e1b[m] * 1.0;
      for (int m = 0; m < indx_(jo, jo); ++m) h[dj + m] = h[dj + m] + e2a[m] * 1.0;
    }
    wstore(ni, w + kr);
    const int il = indx_(io, io);
    kr += (long long)il * il;
  }
  *enuclr_out = enuclr;
  return kr;
}

/* diag_for_GPU.F90:151-206 (CPU branch): the ordered 2x2 rotation sweep over
 * the columns of c (n x n, column-major), occupied i outer and virtual j
 * inner.  fmo is nvirt x nocc column-major, eig holds the orbital energies.
 * A pair is skipped when |x| < tiny or |x/d| < bigeps.  Every row of c sees
 * the same rotations in the same order and rows never mix, so the rows are
 * split over POSIX threads without changing any result.  Returns the number
 * of rotations applied. */
typedef struct {
  int n, r0, r1;
  long long cnt;
  const double *al, *be;
  const int *idx;
  double *c;
} RotJob;

static void *rot_rows(void *arg) {
  RotJob *j = (RotJob *)arg;
  for (int b0 = j->r0; b0 < j->r1; b0 += 8) {
    int b1 = b0 + 8 < j->r1 ? b0 + 8 : j->r1;
    for (long long q = 0; q < j->cnt; ++q) {
      double a = j->al[q], b = j->be[q];
      double *ci = j->c + (long long)j->idx[2 * q] * j->n, *cj = j->c + (long long)j->idx[2 * q + 1] * j->n;
      for (int r = b0; r < b1; ++r) {
        double x = ci[r], y = cj[r];
        ci[r] = a * x + b * y;
        cj[r] = a * y - b * x;
      }
    }
  }
  return NULL;
}

long long orc_rot_sweep(int n, int nocc, const double *fmo, const double *eig, double *c, double bigeps,
                        double tiny) {
  const int nvirt = n - nocc;
  if (nocc <= 0 || nvirt <= 0) return 0;
  const long long kv = (long long)nocc * nvirt;
  double *al = (double *)malloc(sizeof(double) * (size_t)kv);
  double *be = (double *)malloc(sizeof(double) * (size_t)kv);
  int *idx = (int *)malloc(sizeof(int) * 2 * (size_t)kv);
  long long cnt = 0;
  for (int i = 0; i < nocc; ++i)
    for (int jv = 0; jv < nvirt; ++jv) {
      double x = fmo[jv + (long long)nvirt * i];
      if (fabs(x) < tiny) continue;
      double d = eig[i] - eig[nocc + jv];
      if (fabs(x / d) < bigeps) continue;
      double e = copysign(sqrt(4.0 * x * x + d * d), d);
      double a = sqrt(0.5 * (1.0 + d / e));
      al[cnt] = a;
      be[cnt] = -copysign(sqrt(1.0 - a * a), x);
      idx[2 * cnt] = i;
      idx[2 * cnt + 1] = nocc + jv;
      ++cnt;
    }
  int nt = (int)sysconf(_SC_NPROCESSORS_ONLN);
  const char *env = getenv("OMP_NUM_THREADS");
  if (env && atoi(env) > 0) nt = atoi(env);
  if (nt < 1) nt = 1;
  if (nt > 64) nt = 64;
  if (nt > (n + 7) / 8) nt = (n + 7) / 8;
  pthread_t th[64];
  RotJob jobs[64];
  int chunk = ((n + nt - 1) / nt + 7) / 8 * 8;
  int started = 0;
  for (int t = 0; t < nt; ++t) {
    int r0 = t * chunk, r1 = r0 + chunk < n ? r0 + chunk : n;
    if (r0 >= r1) break;
    RotJob jb = {n, r0, r1, cnt, al, be, idx, c};
    jobs[t] = jb;
    if (t == 0) continue;
    if (pthread_create(&th[t], NULL, rot_rows, &jobs[t]) != 0) { rot_rows(&jobs[t]); th[t] = 0; }
    started = t;
  }
  rot_rows(&jobs[0]);
  for (int t = 1; t <= started; ++t)
    if (th[t]) pthread_join(th[t], NULL);
  free(al);
  free(be);
  free(idx);
  return cnt;
}
