// PM7 parameters for the elements this build supports (H, C, O), restated from
// models/parameters_for_PM7_C.F90 (H :24-32, C :91-109, O :127-145,
// v_par7 :1392-1395, alpb/xfac :1405-1483) and the derived multipole
// quantities of models/calpar.F90:49-158 and integrals/mndod.F90:25-59 (inid).
// The derived values are computed once on the host by pm7_derive().
#pragma once
#include <math.h>
#include <string.h>

#define PM7_A0 0.529177210903
#define PM7_EV 27.211386245988
#define PM7_FPC9 23.060547830619029

typedef struct {
  int z, natorb, ios, iop, npq;
  double tore, uss, upp, betas, betap, zs, zp, gss, gsp, gpp, gp2, hsp;
  double g1, g2, g3, eheat;
  double dd, qq, am, ad, aq, eisol, po1, po2, po3, po7, po9, ddp2, ddp3;
} Pm7Elem;

typedef struct {
  Pm7Elem el[9];        // indexed by atomic number, only 1, 6, 8 filled
  double xfac[9][9], alpb[9][9];
  double par1, par2, par3, par4;
} Pm7Params;

static inline void pm7_set(Pm7Elem* e, int z, int natorb, int ios, int iop, int npq, double tore, double uss,
                           double upp, double betas, double betap, double zs, double zp, double gss, double gsp,
                           double gpp, double gp2, double hsp, double g1, double g2, double g3, double eheat) {
  memset(e, 0, sizeof(*e));
  e->z = z; e->natorb = natorb; e->ios = ios; e->iop = iop; e->npq = npq; e->tore = tore;
  e->uss = uss; e->upp = upp; e->betas = betas; e->betap = betap; e->zs = zs; e->zp = zp;
  e->gss = gss; e->gsp = gsp; e->gpp = gpp; e->gp2 = gp2; e->hsp = hsp;
  e->g1 = g1; e->g2 = g2; e->g3 = g3; e->eheat = eheat;
}

// calpar (sp elements) + inid.
static inline void pm7_derive(Pm7Elem* e) {
  if (e->z == 1) {
    e->eisol = e->uss;
    e->am = e->gss / PM7_EV;
    e->ad = e->am;
    e->aq = e->am;
  } else {
    const double gssc = (double)(e->ios - 1 > 0 ? e->ios - 1 : 0);
    const int k = e->iop;
    const double gspc = (double)(e->ios * k);
    const int l = k < 6 - k ? k : 6 - k;
    const double gp2c = (double)((k * (k - 1)) / 2) + 0.5 * (double)(l * (l - 1)) / 2.0;
    const double gppc = -0.5 * (double)(l * (l - 1)) / 2.0;
    const double hspc = -(double)k * (double)e->ios * 0.5;
    e->zp = fmax(0.3, e->zp);
    double hpp = fmax(0.1, 0.5 * (e->gpp - e->gp2));
    e->hsp = fmax(1.0e-7, e->hsp);
    e->eisol = e->uss * e->ios + e->upp * e->iop + e->gss * gssc + e->gpp * gppc + e->gsp * gspc +
               e->gp2 * gp2c + e->hsp * hspc;
    const double qn = (double)e->npq;
    e->dd = (2.0 * qn + 1) * pow(4.0 * e->zs * e->zp, qn + 0.5) / pow(e->zs + e->zp, 2.0 * qn + 2) / sqrt(3.0);
    e->qq = sqrt((4.0 * qn * qn + 6.0 * qn + 2.0) / 20.0) / e->zp;
    double d1 = pow(e->hsp / (PM7_EV * e->dd * e->dd), 1.0 / 3.0), d2 = d1 + 0.04;
    for (int j = 0; j < 5; ++j) {
      const double df = d2 - d1;
      const double h1 = 0.5 * d1 - 0.5 / sqrt(4.0 * e->dd * e->dd + 1.0 / (d1 * d1));
      const double h2 = 0.5 * d2 - 0.5 / sqrt(4.0 * e->dd * e->dd + 1.0 / (d2 * d2));
      if (fabs(h2 - h1) < 1.0e-25) break;
      const double d3 = d1 + df * (e->hsp / PM7_EV - h1) / (h2 - h1);
      d1 = d2;
      d2 = d3;
    }
    double q1 = pow(16.0 * hpp / (PM7_EV * 48.0 * pow(e->qq, 4)), 0.2), q2 = q1 + 0.04;
    for (int j = 0; j < 5; ++j) {
      const double qf = q2 - q1;
      const double h1 = 0.25 * q1 - 0.5 / sqrt(4.0 * e->qq * e->qq + 1.0 / (q1 * q1)) +
                        0.25 / sqrt(8.0 * e->qq * e->qq + 1.0 / (q1 * q1));
      const double h2 = 0.25 * q2 - 0.5 / sqrt(4.0 * e->qq * e->qq + 1.0 / (q2 * q2)) +
                        0.25 / sqrt(8.0 * e->qq * e->qq + 1.0 / (q2 * q2));
      if (fabs(h2 - h1) < 1.0e-25) break;
      const double q3 = q1 + qf * (hpp / PM7_EV - h1) / (h2 - h1);
      q1 = q2;
      q2 = q3;
    }
    e->am = e->gss / PM7_EV;
    e->ad = d2;
    e->aq = q2;
  }
  e->po1 = 0.5 / e->am;
  e->po2 = (e->z != 1 && e->ad > 1.0e-5) ? 0.5 / e->ad : 0.0;
  e->po3 = (e->z != 1 && e->aq > 1.0e-5) ? 0.5 / e->aq : 0.0;
  e->po7 = e->po1;
  e->ddp2 = e->dd;
  e->ddp3 = e->qq * sqrt(2.0);
  e->po9 = e->po1;  // pocord is zero for H, C, O under PM7
}

static inline void pm7_init(Pm7Params* P) {
  memset(P, 0, sizeof(*P));
  pm7_set(&P->el[1], 1, 1, 1, 0, 1, 1.0, -11.070112, 0.0, -8.389745, 0.0, 1.260237, 0.0, 14.149656, 0.0, 0.0, 0.0,
          0.0, 0.177854, 1.428710, 0.991324, 52.102);
  pm7_set(&P->el[6], 6, 4, 2, 2, 2, 4.0, -51.372620, -40.135421, -14.414930, -7.893717, 1.942244, 1.708723,
          12.347323, 11.932801, 10.452226, 9.385498, 0.802634, 0.045888, 5.037055, 1.588715, 170.890);
  pm7_set(&P->el[8], 8, 4, 2, 4, 2, 6.0, -96.087736, -71.087738, -67.776339, -20.267981, 5.972309, 2.349017,
          14.955121, 16.088521, 12.403337, 10.499706, 5.028656, -0.016243, 1.871970, 1.844360, 59.559);
  pm7_derive(&P->el[1]);
  pm7_derive(&P->el[6]);
  pm7_derive(&P->el[8]);
  P->alpb[1][1] = 4.051163; P->xfac[1][1] = 2.845627;
  P->alpb[6][1] = 1.038716; P->xfac[6][1] = 0.204582;
  P->alpb[6][6] = 2.655746; P->xfac[6][6] = 0.937818;
  P->alpb[8][1] = 1.508030; P->xfac[8][1] = 0.160602;
  P->alpb[8][6] = 2.850931; P->xfac[8][6] = 0.826848;
  P->alpb[8][8] = 2.457135; P->xfac[8][8] = 0.356439;
  for (int i = 1; i <= 8; ++i)
    for (int j = 1; j < i; ++j) { P->xfac[j][i] = P->xfac[i][j]; P->alpb[j][i] = P->alpb[i][j]; }
  P->par1 = 8.947612; P->par2 = 6.024265; P->par3 = -0.012037; P->par4 = 0.701333;
}

static inline int pm7_supported(int z) { return z == 1 || z == 6 || z == 8; }
