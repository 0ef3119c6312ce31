// One-electron matrix H, two-electron integrals W and core-core repulsion on
// the GPU for sp atoms under PM7 -- the step before the SCF path
// (integrals/hcore.F90:150-297 with rotate -> rotatd, reppd, spcore, elenuc,
// ccrep, h1elec -> diat/diat2/set/coe, wstore; integrals/mndod.F90).
//
//   hcore_pairs  one thread per atom pair (i > j): the W block in the
//                reference layout (i's pair index outer, j's inner), the
//                resonance block H(i-orbitals, j-orbitals) and the pair's
//                core-core energy.
//   hcore_diag   one thread per atom A: A's diagonal H block, accumulating
//                U_ss/U_pp and the electron-core terms of every partner in
//                the reference's order (partners below A, then above A), and
//                the one-centre W block (wstore).
//   enuc_sum     fixed-order reduction of the pair energies.
#include <algorithm>

#include "mb_common.cuh"
#include "pm7_params.h"

namespace {

struct DevParams {
  Pm7Elem el[9];
  double xfac[9][9], alpb[9][9];
  double par1, par2, par3, par4;
};
__constant__ DevParams c_P;

__constant__ double c_fact[18] = {1.0, 1.0, 2.0, 6.0, 24.0, 120.0, 720.0, 5040.0, 40320.0, 362880.0,
                                  3628800.0, 39916800.0, 479001600.0, 6227020800.0, 87178291200.0,
                                  1307674368000.0, 20922789888000.0, 355687428096000.0};

__device__ __forceinline__ double ipow(double x, int m) {
  double r = 1.0;
  for (int i = 0; i < m; ++i) r *= x;
  return r;
}
__device__ __forceinline__ int indx_(int i, int j) { return i > j ? (i * (i - 1)) / 2 + j : (j * (j - 1)) / 2 + i; }

// ------------------------------------------------------------ overlaps
struct Ovl { double a[8], b[8], sa, sb; int isp, ips; };

__device__ void aintgs(Ovl& o, double x, int k) {
  const double c = exp(-x);
  o.a[1] = c / x;
  for (int i = 1; i <= k; ++i) o.a[i + 1] = (o.a[i] * i + c) / x;
}

__device__ void bintgs(Ovl& o, double x, int k) {
  const double ax = fabs(x);
  int last = 0, mode = 0;
  if (ax > 3.0) mode = 0;
  else if (ax > 2.0) { if (k <= 10) mode = 0; else { last = 15; mode = 1; } }
  else if (ax > 1.0) { if (k <= 7) mode = 0; else { last = 12; mode = 1; } }
  else if (ax > 0.5) { if (k <= 5) mode = 0; else { last = 7; mode = 1; } }
  else if (ax <= 1.0e-6) mode = 2;
  else { last = 6; mode = 1; }
  if (mode == 0) {
    const double expx = exp(x), expmx = 1.0 / expx;
    o.b[1] = (expx - expmx) / x;
    for (int i = 1; i <= k; ++i) o.b[i + 1] = (i * o.b[i] + ((i & 1) ? -1.0 : 1.0) * expx - expmx) / x;
  } else if (mode == 1) {
    for (int i = 0; i <= k; ++i) {
      double y = 0.0;
      for (int m = 0; m <= last; ++m) {
        const double xf = m != 0 ? c_fact[m] : 1.0;
        y = y + ipow(-x, m) * (double)(2 * ((m + i + 1) % 2)) / (xf * (double)(m + i + 1));
      }
      o.b[i + 1] = y;
    }
  } else {
    for (int i = 0; i <= k; ++i) o.b[i + 1] = (double)(2 * ((i + 1) % 2)) / (i + 1.0);
  }
}

__device__ void set_ovl(Ovl& o, double s1, double s2, int na, int nb, double rab, int ii) {
  if (na <= nb) { o.isp = 1; o.ips = 2; o.sa = s1; o.sb = s2; }
  else { o.isp = 2; o.ips = 1; o.sa = s2; o.sb = s1; }
  int j = ii + 2;
  if (ii > 3) j = j - 1;
  aintgs(o, 0.5 * rab * (o.sa + o.sb), j - 1);
  bintgs(o, 0.5 * rab * (o.sb - o.sa), j - 1);
}

// s[la][lb][m] (1-based) for first-row sp atoms (diat2 cases 1, 2, 4)
__device__ void diat2(int na, double esa, double epa, double r12, int nb, double esb, double epb,
                      double s[3][3][3]) {
  for (int x = 0; x < 27; ++x) (&s[0][0][0])[x] = 0.0;
  const int ina = na == 1 ? 1 : (na == 6 ? 4 : 6), inb = nb == 1 ? 1 : (nb == 6 ? 4 : 6);
  const int jmax = ina > inb ? ina : inb, jmin = ina < inb ? ina : inb;
  const int ii = jmax == 1 ? 1 : (jmin == 1 ? 2 : 4);
  const double rab = r12 / PM7_A0;
  Ovl o;
  const double* a = o.a;
  const double* b = o.b;
  if (ii == 2) {
    set_ovl(o, esa, esb, na, nb, rab, ii);
    const double rab4 = ipow(rab, 4) * 0.125;
    double w = sqrt(ipow(o.sa, 3) * ipow(o.sb, 5)) * rab4;
    s[1][1][1] = w * sqrt(1.0 / 3.0) * (a[4] * b[1] - b[4] * a[1] + a[3] * b[2] - b[3] * a[2]);
    if (na > 1) set_ovl(o, epa, esb, na, nb, rab, ii);
    if (nb > 1) set_ovl(o, esa, epb, na, nb, rab, ii);
    w = sqrt(ipow(o.sa, 3) * ipow(o.sb, 5)) * rab4;
    s[o.isp][o.ips][1] = w * (a[3] * b[1] - b[3] * a[1] + a[4] * b[2] - b[4] * a[2]);
  } else if (ii == 4) {
    set_ovl(o, esa, esb, na, nb, rab, ii);
    const double rab4 = ipow(rab, 5) * 0.0625;
    double w = sqrt(ipow(o.sa * o.sb, 5)) * rab4;
    s[1][1][1] = w * (a[5] * b[1] + b[5] * a[1] - 2.0 * a[3] * b[3]) / 3.0;
    set_ovl(o, esa, epb, na, nb, rab, ii);
    if (na > nb) set_ovl(o, epa, esb, na, nb, rab, ii);
    w = sqrt(ipow(o.sa * o.sb, 5)) * rab4;
    const double rt3 = 1.0 / sqrt(3.0);
    double d = a[4] * (b[1] - b[3]) - a[2] * (b[3] - b[5]);
    double e = b[4] * (a[1] - a[3]) - b[2] * (a[3] - a[5]);
    s[o.isp][o.ips][1] = w * rt3 * (d + e);
    set_ovl(o, epa, esb, na, nb, rab, ii);
    if (na > nb) set_ovl(o, esa, epb, na, nb, rab, ii);
    w = sqrt(ipow(o.sa * o.sb, 5)) * rab4;
    d = a[4] * (b[1] - b[3]) - a[2] * (b[3] - b[5]);
    e = b[4] * (a[1] - a[3]) - b[2] * (a[3] - a[5]);
    s[o.ips][o.isp][1] = w * rt3 * (d - e);
    set_ovl(o, epa, epb, na, nb, rab, ii);
    w = sqrt(ipow(o.sa * o.sb, 5)) * rab4;
    s[2][2][1] = -w * (b[3] * (a[5] + a[1]) - a[3] * (b[5] + b[1]));
    s[2][2][2] = 0.5 * w * (a[5] * (b[1] - b[3]) - b[5] * (a[1] - a[3]) - a[3] * b[1] + b[3] * a[1]);
  } else {
    set_ovl(o, esa, esb, na, nb, rab, ii);
    s[1][1][1] = 0.25 * sqrt(ipow(o.sa * o.sb * rab * rab, 3)) * (a[3] * b[1] - b[3] * a[1]);
  }
}

// Resonance block di[i][j] (1-based orbitals: s, px, py, pz) of atom i with
// atom j at xj - xi.
__device__ void h1elec(int ni, int nj, const double* xi, const double* xj, double di[5][5]) {
  for (int x = 0; x < 25; ++x) (&di[0][0])[x] = 0.0;
  const double x2 = xj[0] - xi[0], y2 = xj[1] - xi[1], z2 = xj[2] - xi[2];
  const double rr = x2 * x2 + y2 * y2 + z2 * z2;
  if (rr > 1.0e4 || rr >= 225.0) return;  // cutofs (h1elec) and cutof1 (diat)
  double xy = x2 * x2 + y2 * y2;
  const double r = sqrt(xy + z2 * z2);
  xy = sqrt(xy);
  double ca, cb, sa, sb;
  if (xy >= 1.0e-10) { ca = x2 / xy; cb = z2 / r; sa = y2 / xy; sb = xy / r; }
  else if (z2 < 0.0) { ca = -1.0; cb = -1.0; sa = 0.0; sb = 0.0; }
  else if (z2 == 0.0) { ca = 0.0; cb = 0.0; sa = 0.0; sb = 0.0; }
  else { ca = 1.0; cb = 1.0; sa = 0.0; sb = 0.0; }
  if (r < 0.001) return;
  // c[L][slot][m] for L = s (1), p (2); slot -> orbital: s 3->1; p 2->py, 3->pz, 4->px
  double c[3][5][5];
  for (int x = 0; x < 75; ++x) (&c[0][0][0])[x] = 0.0;
  c[1][3][3] = 1.0;
  const int nij = c_P.el[ni].natorb > c_P.el[nj].natorb ? c_P.el[ni].natorb : c_P.el[nj].natorb;
  if (nij >= 2) {
    c[2][4][4] = ca * cb; c[2][4][3] = ca * sb; c[2][4][2] = -sa;
    c[2][3][4] = -sb;     c[2][3][3] = cb;      c[2][3][2] = 0.0;
    c[2][2][4] = sa * cb; c[2][2][3] = sa * sb; c[2][2][2] = ca;
  }
  double s[3][3][3];
  diat2(ni, c_P.el[ni].zs, c_P.el[ni].zp, r, nj, c_P.el[nj].zs, c_P.el[nj].zp, s);
  const int orb[3][5] = {{0, 0, 0, 0, 0}, {0, 0, 0, 1, 0}, {0, 0, 3, 4, 2}};
  for (int i = 1; i <= 2; ++i) {
    const int kmin = 4 - i, kmax = 2 + i;
    for (int j = 1; j <= 2; ++j) {
      const double aa = j == 2 ? -1.0 : 1.0, bb = 1.0;
      const int lmin = 4 - j, lmax = 2 + j;
      for (int k = kmin; k <= kmax; ++k)
        for (int l = lmin; l <= lmax; ++l) {
          const int ii = orb[i][k], jj = orb[j][l];
          if (ii == 0 || jj == 0) continue;
          di[ii][jj] = s[i][j][1] * (c[i][k][3] * c[j][l][3]) * aa +
                       s[i][j][2] * (c[i][k][4] * c[j][l][4] + c[i][k][2] * c[j][l][2]) * bb +
                       s[i][j][3] * (0.0 + 0.0);
        }
    }
  }
  double bi[5], bj[5];
  bi[1] = c_P.el[ni].betas * 0.5; bi[2] = bi[3] = bi[4] = c_P.el[ni].betap * 0.5;
  bj[1] = c_P.el[nj].betas * 0.5; bj[2] = bj[3] = bj[4] = c_P.el[nj].betap * 0.5;
  for (int j = 1; j <= c_P.el[nj].natorb; ++j)
    for (int i = 1; i <= c_P.el[ni].natorb; ++i) di[i][j] = di[i][j] * (bi[i] + bj[j]);
}

// ------------------------------------------------------- local integrals
__device__ __forceinline__ void to_point(double r, double* point, double* cst) {
  *point = PM7_EV * PM7_A0 / r;
  *cst = (r < 7.0) ? 1.0 - exp(-(r - 7.0) * (r - 7.0) * 0.22) : 0.0;
}

// 22 local-frame repulsion integrals (reppd, l_feather) and G_AB.
__device__ void reppd(int ni, int nj, double rij, double ri[23], double* gab) {
  const double ev1 = PM7_EV / 2, ev2 = ev1 / 2, ev3 = ev2 / 2, ev4 = ev3 / 2, td = 2.0, pp = 0.5;
  for (int i = 0; i < 23; ++i) ri[i] = 0.0;
  const Pm7Elem& A = c_P.el[ni];
  const Pm7Elem& B = c_P.el[nj];
  const double r = rij / PM7_A0;
  const bool si = A.natorb >= 3, sj = B.natorb >= 3;
  double aee = A.po9 + B.po9;
  aee = aee * aee;
  *gab = PM7_EV / sqrt(r * r + aee);
  aee = pp / A.am + pp / B.am;
  aee = aee * aee;
  if (!si && !sj) {
    ri[1] = PM7_EV / sqrt(r * r + aee);
  } else if (si && !sj) {
    const double da = A.dd, qa = A.qq * td;
    double ade = pp / A.ad + pp / B.am; ade *= ade;
    double aqe = pp / A.aq + pp / B.am; aqe *= aqe;
    const double rsq = r * r;
    const double s1 = sqrt(rsq + aee), s2 = sqrt((r + da) * (r + da) + ade), s3 = sqrt((r - da) * (r - da) + ade),
                 s4 = sqrt((r + qa) * (r + qa) + aqe), s5 = sqrt((r - qa) * (r - qa) + aqe), a6 = rsq + aqe,
                 s6 = sqrt(a6), s7 = sqrt(a6 + qa * qa);
    const double ee = PM7_EV / s1;
    ri[1] = ee;
    ri[2] = ev1 / s2 - ev1 / s3;
    ri[3] = ee + ev2 / s4 + ev2 / s5 - ev1 / s6;
    ri[4] = ee + ev1 / s7 - ev1 / s6;
  } else if (!si && sj) {
    const double db = B.dd, qb = B.qq * td;
    double aed = pp / A.am + pp / B.ad; aed *= aed;
    double aeq = pp / A.am + pp / B.aq; aeq *= aeq;
    const double rsq = r * r;
    const double s1 = sqrt(rsq + aee), s2 = sqrt((r - db) * (r - db) + aed), s3 = sqrt((r + db) * (r + db) + aed),
                 s4 = sqrt((r - qb) * (r - qb) + aeq), s5 = sqrt((r + qb) * (r + qb) + aeq), a6 = rsq + aeq,
                 s6 = sqrt(a6), s7 = sqrt(a6 + qb * qb);
    const double ee = PM7_EV / s1;
    ri[1] = ee;
    ri[5] = ev1 / s2 - ev1 / s3;
    ri[11] = ee + ev2 / s4 + ev2 / s5 - ev1 / s6;
    ri[12] = ee + ev1 / s7 - ev1 / s6;
  } else {
    const double da = A.dd, db = B.dd;
    double qa = A.qq * td, qb = B.qq * td;
    double ade = pp / A.ad + pp / B.am; ade *= ade;
    double aqe = pp / A.aq + pp / B.am; aqe *= aqe;
    double aed = pp / A.am + pp / B.ad; aed *= aed;
    double aeq = pp / A.am + pp / B.aq; aeq *= aeq;
    double axx = pp / A.ad + pp / B.ad; axx *= axx;
    double adq = pp / A.ad + pp / B.aq; adq *= adq;
    double aqd = pp / A.aq + pp / B.ad; aqd *= aqd;
    double aqq = pp / A.aq + pp / B.aq; aqq *= aqq;
    const double rsq = r * r;
    double sq[73];
    double xxx, yyy, zzz, www;
#define SQ(i, v) sq[i] = sqrt(v)
    SQ(1, rsq + aee);
    xxx = r + da; SQ(2, xxx * xxx + ade);
    xxx = r - da; SQ(3, xxx * xxx + ade);
    xxx = r - qa; SQ(4, xxx * xxx + aqe);
    xxx = r + qa; SQ(5, xxx * xxx + aqe);
    double a6 = rsq + aqe; SQ(6, a6);
    SQ(7, a6 + qa * qa);
    xxx = r - db; SQ(8, xxx * xxx + aed);
    xxx = r + db; SQ(9, xxx * xxx + aed);
    xxx = r - qb; SQ(10, xxx * xxx + aeq);
    xxx = r + qb; SQ(11, xxx * xxx + aeq);
    double a12 = rsq + aeq; SQ(12, a12);
    SQ(13, a12 + qb * qb);
    xxx = da - db; SQ(14, rsq + axx + xxx * xxx);
    xxx = da + db; SQ(15, rsq + axx + xxx * xxx);
    xxx = r + da - db; SQ(16, xxx * xxx + axx);
    xxx = r - da + db; SQ(17, xxx * xxx + axx);
    xxx = r - da - db; SQ(18, xxx * xxx + axx);
    xxx = r + da + db; SQ(19, xxx * xxx + axx);
    xxx = r + da; double a20 = xxx * xxx + adq; SQ(20, a20);
    SQ(21, a20 + qb * qb);
    xxx = r - da; double a22 = xxx * xxx + adq; SQ(22, a22);
    SQ(23, a22 + qb * qb);
    xxx = r - db; double a24 = xxx * xxx + aqd; SQ(24, a24);
    SQ(25, a24 + qa * qa);
    xxx = r + db; double a26 = xxx * xxx + aqd; SQ(26, a26);
    SQ(27, a26 + qa * qa);
    xxx = r + da - qb; SQ(28, xxx * xxx + adq);
    xxx = r - da - qb; SQ(29, xxx * xxx + adq);
    xxx = r + da + qb; SQ(30, xxx * xxx + adq);
    xxx = r - da + qb; SQ(31, xxx * xxx + adq);
    xxx = r + qa - db; SQ(32, xxx * xxx + aqd);
    xxx = r + qa + db; SQ(33, xxx * xxx + aqd);
    xxx = r - qa - db; SQ(34, xxx * xxx + aqd);
    xxx = r - qa + db; SQ(35, xxx * xxx + aqd);
    const double a36 = rsq + aqq; SQ(36, a36);
    xxx = qa - qb; SQ(37, a36 + xxx * xxx);
    xxx = qa + qb; SQ(38, a36 + xxx * xxx);
    const double a39 = a36 + qa * qa; SQ(39, a39);
    SQ(40, a36 + qb * qb);
    SQ(41, a39 + qb * qb);
    xxx = r - qb; double a42 = xxx * xxx + aqq; SQ(42, a42);
    SQ(43, a42 + qa * qa);
    xxx = r + qb; double a44 = xxx * xxx + aqq; SQ(44, a44);
    SQ(45, a44 + qa * qa);
    xxx = r + qa; double a46 = xxx * xxx + aqq; SQ(46, a46);
    SQ(47, a46 + qb * qb);
    xxx = r - qa; double a48 = xxx * xxx + aqq; SQ(48, a48);
    SQ(49, a48 + qb * qb);
    xxx = r + qa - qb; SQ(50, xxx * xxx + aqq);
    xxx = r + qa + qb; SQ(51, xxx * xxx + aqq);
    xxx = r - qa - qb; SQ(52, xxx * xxx + aqq);
    xxx = r - qa + qb; SQ(53, xxx * xxx + aqq);
    qa = A.qq;
    qb = B.qq;
    xxx = da - qb; xxx = xxx * xxx;
    yyy = r - qb; yyy = yyy * yyy;
    zzz = da + qb; zzz = zzz * zzz;
    www = r + qb; www = www * www;
    SQ(54, xxx + yyy + adq);
    SQ(55, xxx + www + adq);
    SQ(56, zzz + yyy + adq);
    SQ(57, zzz + www + adq);
    xxx = qa - db; xxx = xxx * xxx;
    yyy = qa + db; yyy = yyy * yyy;
    zzz = r + qa; zzz = zzz * zzz;
    www = r - qa; www = www * www;
    SQ(58, zzz + xxx + aqd);
    SQ(59, www + xxx + aqd);
    SQ(60, zzz + yyy + aqd);
    SQ(61, www + yyy + aqd);
    xxx = qa - qb; xxx = xxx * xxx;
    yyy = qa + qb; yyy = yyy * yyy;
    zzz = r + qa - qb; zzz = zzz * zzz;
    SQ(65, zzz + xxx + aqq);
    SQ(66, zzz + yyy + aqq);
    zzz = r + qa + qb; zzz = zzz * zzz;
    SQ(67, zzz + xxx + aqq);
    SQ(68, zzz + yyy + aqq);
    zzz = r - qa - qb; zzz = zzz * zzz;
    SQ(69, zzz + xxx + aqq);
    SQ(70, zzz + yyy + aqq);
    zzz = r - qa + qb; zzz = zzz * zzz;
    SQ(71, zzz + xxx + aqq);
    SQ(72, zzz + yyy + aqq);
#undef SQ
    const double ee = PM7_EV / sq[1];
    const double dze = (-ev1 / sq[2]) + ev1 / sq[3];
    const double qzze = ev2 / sq[4] + ev2 / sq[5] - ev1 / sq[6];
    const double qxxe = ev1 / sq[7] - ev1 / sq[6];
    const double edz = (-ev1 / sq[8]) + ev1 / sq[9];
    const double eqzz = ev2 / sq[10] + ev2 / sq[11] - ev1 / sq[12];
    const double eqxx = ev1 / sq[13] - ev1 / sq[12];
    const double dxdx = ev1 / sq[14] - ev1 / sq[15];
    const double dzdz = ev2 / sq[16] + ev2 / sq[17] - ev2 / sq[18] - ev2 / sq[19];
    const double dzqxx = ev2 / sq[20] - ev2 / sq[21] - ev2 / sq[22] + ev2 / sq[23];
    const double qxxdz = ev2 / sq[24] - ev2 / sq[25] - ev2 / sq[26] + ev2 / sq[27];
    const double dzqzz = (-ev3 / sq[28]) + ev3 / sq[29] - ev3 / sq[30] + ev3 / sq[31] - ev2 / sq[22] + ev2 / sq[20];
    const double qzzdz = (-ev3 / sq[32]) + ev3 / sq[33] - ev3 / sq[34] + ev3 / sq[35] + ev2 / sq[24] - ev2 / sq[26];
    const double qxxqxx = ev3 / sq[37] + ev3 / sq[38] - ev2 / sq[39] - ev2 / sq[40] + ev2 / sq[36];
    const double qxxqyy = ev2 / sq[41] - ev2 / sq[39] - ev2 / sq[40] + ev2 / sq[36];
    const double qxxqzz = ev3 / sq[43] + ev3 / sq[45] - ev3 / sq[42] - ev3 / sq[44] - ev2 / sq[39] + ev2 / sq[36];
    const double qzzqxx = ev3 / sq[47] + ev3 / sq[49] - ev3 / sq[46] - ev3 / sq[48] - ev2 / sq[40] + ev2 / sq[36];
    const double qzzqzz = ev4 / sq[50] + ev4 / sq[51] + ev4 / sq[52] + ev4 / sq[53] - ev3 / sq[48] - ev3 / sq[46] -
                          ev3 / sq[42] - ev3 / sq[44] + ev2 / sq[36];
    const double dxqxz = (-ev2 / sq[54]) + ev2 / sq[55] + ev2 / sq[56] - ev2 / sq[57];
    const double qxzdx = (-ev2 / sq[58]) + ev2 / sq[59] + ev2 / sq[60] - ev2 / sq[61];
    const double qxzqxz = ev3 / sq[65] - ev3 / sq[67] - ev3 / sq[69] + ev3 / sq[71] - ev3 / sq[66] + ev3 / sq[68] +
                          ev3 / sq[70] - ev3 / sq[72];
    ri[1] = ee; ri[2] = -dze; ri[3] = ee + qzze; ri[4] = ee + qxxe; ri[5] = -edz; ri[6] = dzdz; ri[7] = dxdx;
    ri[8] = (-edz) - qzzdz; ri[9] = (-edz) - qxxdz; ri[10] = -qxzdx; ri[11] = ee + eqzz; ri[12] = ee + eqxx;
    ri[13] = (-dze) - dzqzz; ri[14] = (-dze) - dzqxx; ri[15] = -dxqxz; ri[16] = ee + eqzz + qzze + qzzqzz;
    ri[17] = ee + eqzz + qxxe + qxxqzz; ri[18] = ee + eqxx + qzze + qzzqxx; ri[19] = ee + eqxx + qxxe + qxxqxx;
    ri[20] = qxzqxz; ri[21] = ee + eqxx + qxxe + qxxqyy; ri[22] = pp * (qxxqxx - qxxqyy);
  }
  double point, cst;
  to_point(rij, &point, &cst);
  const unsigned coul = (1u << 1) | (1u << 3) | (1u << 4) | (1u << 11) | (1u << 12) | (1u << 16) | (1u << 17) |
                        (1u << 18) | (1u << 19) | (1u << 21);
  const unsigned neg = (1u << 2) | (1u << 5) | (1u << 8) | (1u << 9) | (1u << 10) | (1u << 13) | (1u << 14) |
                       (1u << 15);
  for (int i = 1; i <= 22; ++i) {
    ri[i] = ((coul >> i) & 1u) ? ri[i] * cst + (1.0 - cst) * point : ri[i] * cst;
    if ((neg >> i) & 1u) ri[i] = -ri[i];
  }
  *gab = *gab * cst + (1.0 - cst) * point;
}

// core[k][n]: electron-core attraction, local frame (spcore) with feathering.
__device__ void core_terms(int ni, int nj, double rij, double core[5][3]) {
  const Pm7Elem& A = c_P.el[ni];
  const Pm7Elem& B = c_P.el[nj];
  const double pxy[8] = {0, 1.0, -0.5, -0.5, 0.5, 0.25, 0.25, 0.5};
  for (int x = 0; x < 15; ++x) (&core[0][0])[x] = 0.0;
  const double r = rij / PM7_A0, r2 = r * r;
  const double aci = A.po9, acj = B.po9;
  const double ssi = (aci + B.po1) * (aci + B.po1), ssj = (acj + A.po1) * (acj + A.po1);
  core[1][1] = -B.tore * PM7_EV / sqrt(r2 + ssj);
  core[1][2] = -A.tore * PM7_EV / sqrt(r2 + ssi);
  if (ni >= 3) {
    const double ppj = (acj + A.po7) * (acj + A.po7), da = A.ddp2, qa = A.ddp3 / sqrt(2.0), twoqa = qa + qa;
    const double adj = (A.po2 + acj) * (A.po2 + acj), aqj = (A.po3 + acj) * (A.po3 + acj);
    double x[8];
    x[1] = r2 + ppj; x[2] = r2 + aqj; x[3] = (r + da) * (r + da) + adj; x[4] = (r - da) * (r - da) + adj;
    x[5] = (r - twoqa) * (r - twoqa) + aqj; x[6] = (r + twoqa) * (r + twoqa) + aqj; x[7] = r2 + twoqa * twoqa + aqj;
    for (int i = 1; i <= 7; ++i) x[i] = pxy[i] / sqrt(x[i]);
    core[2][1] = -B.tore * ((x[3] + x[4]) * PM7_EV);
    core[3][1] = -B.tore * ((x[1] + x[2] + x[5] + x[6]) * PM7_EV);
    core[4][1] = -B.tore * ((x[1] + x[2] + x[7]) * PM7_EV);
  }
  if (nj >= 3) {
    const double ppi = (aci + B.po7) * (aci + B.po7), db = B.ddp2, qb = B.ddp3 / sqrt(2.0), twoqb = qb + qb;
    const double adi = (B.po2 + aci) * (B.po2 + aci), aqi = (B.po3 + aci) * (B.po3 + aci);
    double x[8];
    x[1] = r2 + ppi; x[2] = r2 + aqi; x[3] = (r + db) * (r + db) + adi; x[4] = (r - db) * (r - db) + adi;
    x[5] = (r - twoqb) * (r - twoqb) + aqi; x[6] = (r + twoqb) * (r + twoqb) + aqi; x[7] = r2 + twoqb * twoqb + aqi;
    for (int i = 1; i <= 7; ++i) x[i] = pxy[i] / sqrt(x[i]);
    core[2][2] = -A.tore * (-(x[3] + x[4]) * PM7_EV);
    core[3][2] = -A.tore * ((x[1] + x[2] + x[5] + x[6]) * PM7_EV);
    core[4][2] = -A.tore * ((x[1] + x[2] + x[7]) * PM7_EV);
  }
  double point, cst;
  to_point(rij, &point, &cst);
  point = -(PM7_EV / r) * B.tore;
  core[1][1] = core[1][1] * cst + (1.0 - cst) * point;
  core[2][1] = core[2][1] * cst;
  core[3][1] = core[3][1] * cst + (1.0 - cst) * point;
  core[4][1] = core[4][1] * cst + (1.0 - cst) * point;
  point = -(PM7_EV / r) * A.tore;
  core[1][2] = core[1][2] * cst + (1.0 - cst) * point;
  core[2][2] = core[2][2] * cst;
  core[3][2] = core[3][2] * cst + (1.0 - cst) * point;
  core[4][2] = core[4][2] * cst + (1.0 - cst) * point;
}

// Rotation matrix of the pair axis (rotmat): p[k][m], k = local axis
// (sigma, pi, pi'), m = molecular x, y, z; returns the distance.
__device__ double rotmat(const double* ci, const double* cj, double p[4][4]) {
  const double x11 = cj[0] - ci[0], x22 = cj[1] - ci[1], x33 = cj[2] - ci[2];
  const double b = x11 * x11 + x22 * x22;
  const double r = sqrt(b + x33 * x33);
  const double sqb = sqrt(b);
  double sb = sqb / r, ca, sa, cb;
  if (sb > 1.0e-7) { ca = x11 / sqb; sa = x22 / sqb; cb = x33 / r; }
  else {
    sa = 0.0; sb = 0.0;
    if (x33 < 0.0) { ca = -1.0; cb = -1.0; }
    else if (x33 > 0.0) { ca = 1.0; cb = 1.0; }
    else { ca = 0.0; cb = 0.0; }
  }
  p[1][1] = ca * sb; p[2][1] = ca * cb; p[3][1] = -sa;
  p[1][2] = sa * sb; p[2][2] = sa * cb; p[3][2] = ca;
  p[1][3] = cb;      p[2][3] = -sb;     p[3][3] = 0.0;
  return r;
}

// pp(t, k, l) products of rotation rows (rotmat :1484-1501)
__device__ __forceinline__ double ppf(const double p[4][4], int t, int k, int l) {
  const int ta[7] = {0, 1, 2, 3, 1, 1, 2}, tb[7] = {0, 1, 2, 3, 2, 3, 3};
  const int a = ta[t], b = tb[t];
  if (k == l) return p[k][a] * p[k][b];
  if (t <= 3) return 2.0 * p[k][a] * p[l][a];
  return p[k][a] * p[l][b] + p[k][b] * p[l][a];
}

// The electron-core blocks e1b (atom i) / e2a (atom j), packed local order.
__device__ void elenuc(const double p[4][4], const double core[5][3], int li, int lj, double* e1b, double* e2a) {
  const int indpp[4][4] = {{0, 0, 0, 0}, {0, 1, 4, 5}, {0, 4, 2, 6}, {0, 5, 6, 3}};
  for (int nn = 1; nn <= 2; ++nn) {
    const int lim = nn == 1 ? li : lj;
    double* out = nn == 1 ? e1b : e2a;
    int m = 0;
    for (int i = 1; i <= lim; ++i)
      for (int j = 1; j <= i; ++j) {
        const int a = i - 1, b = j - 1;
        double h;
        if (a == 0) h = core[1][nn];
        else if (b == 0) h = p[1][a] * core[2][nn];
        else {
          const int t = indpp[a][b];
          h = core[3][nn] * ppf(p, t, 1, 1) + core[4][nn] * (ppf(p, t, 2, 2) + ppf(p, t, 3, 3));
        }
        out[m++] = 0.0 + h;
      }
  }
}

// ccrep (PM7): r in Bohr on entry
__device__ double ccrep(int ni, int nj, double rb, double gab) {
  const double r = rb * PM7_A0;
  const Pm7Elem& A = c_P.el[ni];
  const Pm7Elem& B = c_P.el[nj];
  const double enuc = A.tore * B.tore * gab;
  double fff = c_P.xfac[ni][nj], abond = c_P.alpb[ni][nj];
  if (fabs(fff) < 1.0e-5) {
    fff = 0.5 * (c_P.xfac[ni][ni] + c_P.xfac[nj][nj]);
    abond = 0.5 * (c_P.alpb[ni][ni] + c_P.alpb[nj][nj]);
  }
  double enuclr, scale;
  if (fabs(fff) > 1.0e-5) {
    if (abond < 1.0e-6) abond = 1.2;
    scale = 1.0 + 2.0 * fff * exp(-abond * (r + (double)0.0003f * ipow(r, 6)));
    const int i = ni > nj ? ni : nj, j = ni < nj ? ni : nj;
    if (j == 1) {
      if (i == 6 || i == 7) scale = 1.0 + 2.0 * fff * exp(-abond * r * r);
      else if (i == 8) scale = 1.0 + 2.0 * fff * exp(-abond * r * r) - c_P.par3 * exp(-c_P.par4 * r * 2);
    } else if (j == 6 && i == 6) {
      scale = scale + c_P.par1 * exp(-c_P.par2 * r);
    }
    enuclr = enuc * scale;
  } else {
    scale = 10.0 * exp(-2.18 * r);
    enuclr = fabs(scale * enuc) + enuc;
  }
  scale = 0.0;
  double ax = A.g2 * (r - A.g3) * (r - A.g3);
  if (ax < 25.0) scale = scale + A.tore * B.tore / r * A.g1 * exp(-ax);
  ax = B.g2 * (r - B.g3) * (r - B.g3);
  if (ax < 25.0) scale = scale + A.tore * B.tore / r * B.g1 * exp(-ax);
  enuclr = enuclr + scale;
  ax = r / (pow((double)ni, 0.3333) + pow((double)nj, 0.3333));
  if (ax < 3.0) {
    scale = 1.0e-8 / ipow(ax, 12);
    enuclr = enuclr + (scale < 1.0e5 ? scale : 1.0e5);
  }
  return enuclr;
}

// W block of pair (ni first, nj second) in molecular frame, reference layout.
// Local-frame pairs of each atom are numbered (indexd) 1:ss 2:ps 10:pp(sigma)
// 3:pi-s 11:pi-sigma 18:pi-pi 4:pi'-s 12:pi'-sigma 19:pi'-pi 25:pi'-pi'.
__device__ void w_block(int ni, int nj, const double p[4][4], const double ri[23], double* w) {
  const int ii = c_P.el[ni].natorb, kk = c_P.el[nj].natorb;
  const int limkl = indx_(kk, kk), limij = indx_(ii, ii);
  // rep index for (local pair on A, local pair on B): compact local ids 0..9
  // order (1,1),(2,1),(2,2),(3,1),(3,2),(3,3),(4,1),(4,2),(4,3),(4,4) -> indexd
  // 1,2,10,3,11,18,4,12,19,25
  const int repidx[10][10] = {
      // B: ss  ps  pp  pis pisg pipi pi's pi'sg pi'pi pi'pi'
      {1, 5, 11, 0, 0, 12, 0, 0, 0, 12},       // A ss
      {2, 6, 13, 0, 0, 14, 0, 0, 0, 14},       // A sigma-s
      {3, 8, 16, 0, 0, 18, 0, 0, 0, 18},       // A sigma-sigma
      {0, 0, 0, 7, 15, 0, 0, 0, 0, 0},         // A pi-s
      {0, 0, 0, 10, 20, 0, 0, 0, 0, 0},        // A pi-sigma
      {4, 9, 17, 0, 0, 19, 0, 0, 0, 21},       // A pi-pi
      {0, 0, 0, 0, 0, 0, 7, 15, 0, 0},         // A pi'-s
      {0, 0, 0, 0, 0, 0, 10, 20, 0, 0},        // A pi'-sigma
      {0, 0, 0, 0, 0, 0, 0, 0, 22, 0},         // A pi'-pi
      {4, 9, 17, 0, 0, 21, 0, 0, 0, 19}};      // A pi'-pi'
  // local pair (k1, l1) on an atom -> compact id
  // tx: v(ijA, kl_mol) for the 10 molecular pairs kl of B
  double v[10][10];
  for (int x = 0; x < 100; ++x) (&v[0][0])[x] = 0.0;
  for (int a = 0; a < (ii == 1 ? 1 : 10); ++a) {
    for (int b = 0; b < (kk == 1 ? 1 : 10); ++b) {
      const int nd = repidx[a][b];
      if (nd == 0) continue;
      const double wrepp = ri[nd];
      // b -> (k1, l1)
      int k1 = 1, l1 = 1, e = b;
      while (e >= k1) { e -= k1; ++k1; }
      l1 = e + 1;
      const int mm = (k1 == 1) ? 1 : (l1 == 1 ? 2 : 3);
      if (mm == 1) v[a][0] = wrepp;
      else if (mm == 2) {
        const int k = k1 - 1;
        v[a][1] = v[a][1] + p[k][1] * wrepp;
        v[a][3] = v[a][3] + p[k][2] * wrepp;
        v[a][6] = v[a][6] + p[k][3] * wrepp;
      } else {
        const int k = k1 - 1, l = l1 - 1;
        v[a][2] = v[a][2] + ppf(p, 1, k, l) * wrepp;
        v[a][5] = v[a][5] + ppf(p, 2, k, l) * wrepp;
        v[a][9] = v[a][9] + ppf(p, 3, k, l) * wrepp;
        v[a][4] = v[a][4] + ppf(p, 4, k, l) * wrepp;
        v[a][7] = v[a][7] + ppf(p, 5, k, l) * wrepp;
        v[a][8] = v[a][8] + ppf(p, 6, k, l) * wrepp;
      }
    }
  }
  for (int x = 0; x < limij * limkl; ++x) w[x] = 0.0;
  for (int a = 0; a < (ii == 1 ? 1 : 10); ++a) {
    int i1 = 1, j1 = 1, e = a;
    while (e >= i1) { e -= i1; ++i1; }
    j1 = e + 1;
    const int mm = (i1 == 1) ? 1 : (j1 == 1 ? 2 : 3);
    for (int kl = 1; kl <= limkl; ++kl) {
      const double wrepp = v[a][kl - 1];
      if (wrepp == 0.0) continue;
#define WI(x, y) w[(indx_((x), (y)) - 1) * limkl + kl - 1]
      if (mm == 1) WI(1, 1) = wrepp;
      else if (mm == 2) {
        for (int i = 1; i <= 3; ++i) WI(i + 1, 1) += p[i1 - 1][i] * wrepp;
      } else {
        for (int i = 1; i <= 3; ++i) {
          WI(i + 1, i + 1) += ppf(p, i, i1 - 1, j1 - 1) * wrepp;
          for (int j = 1; j < i; ++j) WI(i + 1, j + 1) += ppf(p, 1 + i + j, i1 - 1, j1 - 1) * wrepp;
        }
      }
#undef WI
    }
  }
}

// Off-diagonal H block, two-centre W block and core-core energy of pair q.
__device__ void hcore_pair_one(long long q, const int* __restrict__ nat, const double* __restrict__ coord,
                               const MbAtomsDev& at, double* __restrict__ h, double* __restrict__ w,
                               double* __restrict__ enuc_pairs) {
  {
    // pair q -> (i, j), i > j, in the reference loop order
    long long i = (long long)((sqrt(8.0 * (double)q + 1.0) + 1.0) * 0.5);
    while (i * (i - 1) / 2 > q) --i;
    while ((i + 1) * i / 2 <= q) ++i;
    const int ia = (int)i, ja = (int)(q - i * (i - 1) / 2);
    const int ni = nat[ia], nj = nat[ja];
    const double* xi = coord + 3 * ia;
    const double* xj = coord + 3 * ja;
    double di[5][5];
    h1elec(ni, nj, xi, xj, di);
    const int fi = at.first[ia], fj = at.first[ja], noi = at.nor[ia], noj = at.nor[ja];
    for (int a = 1; a <= noi; ++a)
      for (int b = 1; b <= noj; ++b) h[mb_tri(fi + a - 1, fj + b - 1)] = di[a][b];
    double* wb = w + at.wrow[ia] + (long long)at.lim[ia] * at.cum[ja];
    const double dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
    if (dx * dx + dy * dy + dz * dz < 0.00002) {
      for (int x = 0; x < at.lim[ia] * at.lim[ja]; ++x) wb[x] = 0.0;
      enuc_pairs[q] = 0.0;
      return;
    }
    double p[4][4];
    const double r = rotmat(xi, xj, p);
    double ri[23], gab;
    reppd(ni, nj, r, ri, &gab);
    w_block(ni, nj, p, ri, wb);
    enuc_pairs[q] = ccrep(ni, nj, r / PM7_A0, gab);
  }
}

__global__ void hcore_pairs(int numat, const int* __restrict__ nat, const double* __restrict__ coord, MbAtomsDev at,
                            double* __restrict__ h, double* __restrict__ w, double* __restrict__ enuc_pairs) {
  const long long npair = (long long)numat * (numat - 1) / 2;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < npair; q += (long long)gridDim.x * blockDim.x)
    hcore_pair_one(q, nat, coord, at, h, w, enuc_pairs);
}

// Diagonal H block of atom A in reference accumulation order + one-centre W.
__device__ void hcore_atom_one(int A, int numat, const int* __restrict__ nat, const double* __restrict__ coord,
                               const MbAtomsDev& at, double* __restrict__ h, double* __restrict__ w) {
  const int nA = nat[A], fA = at.first[A], noA = at.nor[A], lA = at.lim[A];
  const Pm7Elem& E = c_P.el[nA];
  double blk[10];
  for (int x = 0; x < 10; ++x) blk[x] = 0.0;
  blk[0] = E.uss;
  if (noA == 4) { blk[2] = E.upp; blk[5] = E.upp; blk[9] = E.upp; }
  const double* xa = coord + 3 * A;
  for (int B = 0; B < numat; ++B) {
    if (B == A) continue;
    const double* xb = coord + 3 * B;
    const double dx = xa[0] - xb[0], dy = xa[1] - xb[1], dz = xa[2] - xb[2];
    if (dx * dx + dy * dy + dz * dz < 0.00002) continue;
    const int nB = nat[B];
    double p[4][4], core[5][3], e1b[10], e2a[10];
    if (B < A) {  // pair (A first, B second): A receives e1b
      const double r = rotmat(xa, xb, p);
      core_terms(nA, nB, r, core);
      elenuc(p, core, noA, at.nor[B], e1b, e2a);
      for (int x = 0; x < lA; ++x) blk[x] = blk[x] + e1b[x] * 1.0;
    } else {      // pair (B first, A second): A receives e2a
      const double r = rotmat(xb, xa, p);
      core_terms(nB, nA, r, core);
      elenuc(p, core, at.nor[B], noA, e1b, e2a);
      for (int x = 0; x < lA; ++x) blk[x] = blk[x] + e2a[x] * 1.0;
    }
  }
  for (int a = 0, x = 0; a < noA; ++a)
    for (int b = 0; b <= a; ++b, ++x) h[mb_tri(fA + a, fA + b)] = blk[x];
  // wstore (mndod.F90:2027)
  double* w1 = w + at.wrow[A] + (long long)lA * at.cum[A];
  for (int x = 0; x < lA * lA; ++x) w1[x] = 0.0;
#define WS(a, b) w1[((a) - 1) + lA * ((b) - 1)]
  WS(1, 1) = E.gss;
  if (noA == 4) {
    const int ipx = 3, ipy = 6, ipz = 10;
    WS(ipx, 1) = E.gsp; WS(ipy, 1) = E.gsp; WS(ipz, 1) = E.gsp;
    WS(1, ipx) = E.gsp; WS(1, ipy) = E.gsp; WS(1, ipz) = E.gsp;
    WS(ipx, ipx) = E.gpp; WS(ipy, ipy) = E.gpp; WS(ipz, ipz) = E.gpp;
    WS(ipy, ipx) = E.gp2; WS(ipz, ipx) = E.gp2; WS(ipz, ipy) = E.gp2;
    WS(ipx, ipy) = E.gp2; WS(ipx, ipz) = E.gp2; WS(ipy, ipz) = E.gp2;
    WS(2, 2) = E.hsp; WS(4, 4) = E.hsp; WS(7, 7) = E.hsp;
    WS(5, 5) = 0.5 * (E.gpp - E.gp2); WS(8, 8) = 0.5 * (E.gpp - E.gp2); WS(9, 9) = 0.5 * (E.gpp - E.gp2);
  }
#undef WS
}

__global__ void hcore_diag(int numat, const int* __restrict__ nat, const double* __restrict__ coord, MbAtomsDev at,
                           double* __restrict__ h, double* __restrict__ w) {
  const int A = blockIdx.x * blockDim.x + threadIdx.x;
  if (A < numat) hcore_atom_one(A, numat, nat, coord, at, h, w);
}

// ---- many molecules in one launch: a global pair or atom index is mapped to
// its molecule by a binary search over the prefix offsets.
__device__ __forceinline__ int batch_find(const long long* off, int nmol, long long q) {
  int lo = 0, hi = nmol;  // largest m < nmol with off[m] <= q
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= q) lo = mid; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ MbAtomsDev batch_atoms(const MbHcoreBatch& B, int m) {
  const long long a0 = B.atom_off[m];
  MbAtomsDev at;
  at.numat = (int)(B.atom_off[m + 1] - a0);
  at.first = B.first + a0;
  at.nor = B.nor + a0;
  at.lim = B.lim + a0;
  at.wrow = B.wrow + a0;
  at.cum = B.cum + a0;
  return at;
}

__global__ void hcore_pairs_batch(MbHcoreBatch B) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < B.pair_off[B.nmol];
       q += (long long)gridDim.x * blockDim.x) {
    const int m = batch_find(B.pair_off, B.nmol, q);
    const MbAtomsDev at = batch_atoms(B, m);
    const long long a0 = B.atom_off[m];
    hcore_pair_one(q - B.pair_off[m], B.nat + a0, B.coord + 3 * a0, at, B.h + B.hoff[m], B.w + B.woff[m],
                   B.enuc_pairs + B.pair_off[m]);
  }
}

__global__ void hcore_diag_batch(MbHcoreBatch B) {
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < B.atom_off[B.nmol];
       g += (long long)gridDim.x * blockDim.x) {
    const int m = batch_find(B.atom_off, B.nmol, g);
    const MbAtomsDev at = batch_atoms(B, m);
    const long long a0 = B.atom_off[m];
    hcore_atom_one((int)(g - a0), at.numat, B.nat + a0, B.coord + 3 * a0, at, B.h + B.hoff[m], B.w + B.woff[m]);
  }
}

// Fixed-order two-level reduction of the pair energies.
__global__ void enuc_sum(long long npair, const double* __restrict__ e, double* __restrict__ out) {
  __shared__ double sh[1024];
  double s = 0.0;
  for (long long q = threadIdx.x; q < npair; q += blockDim.x) s += e[q];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sh[0];
}

// enuc_sum for every molecule (block m: molecule m, the same order).
__global__ void enuc_sum_batch(MbHcoreBatch B) {
  const int m = blockIdx.x;
  const long long p0 = B.pair_off[m], np = B.pair_off[m + 1] - p0;
  __shared__ double sh[1024];
  double s = 0.0;
  for (long long q = threadIdx.x; q < np; q += blockDim.x) s += B.enuc_pairs[p0 + q];
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st) sh[threadIdx.x] += sh[threadIdx.x + st];
    __syncthreads();
  }
  if (threadIdx.x == 0) B.enuclr[m] = np > 0 ? sh[0] : 0.0;
}

// ---- hcore_for_MOZYME (MOZYME/hcore_for_MOZYME.F90, molecular, mode 0) on
// fillij's pair-block storage.  Stored pairs get the full integrals (the
// bodies above); the diagonal blocks take every partner's core attraction
// in the reference's order (with PM7's feathering the exact term beyond 7 A
// is the point charge outer1/outer2 use); the core-core energy of a pair
// that is not stored is outer1's or outer2's (tore_i tore_j times the
// point-charge or monopole integral).
__global__ void mz_hcore_pairs(MbMzLayout L, const int* __restrict__ nat, const double* __restrict__ coord,
                               double* __restrict__ h, double* __restrict__ w, double* __restrict__ enuc_entry) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < L.npairs;
       e += (long long)gridDim.x * blockDim.x) {
    const int ia = L.pair_i[e], ja = L.pair_j[e];
    if (ia == ja) {
      enuc_entry[e] = 0.0;
      continue;
    }
    const int ni = nat[ia], nj = nat[ja];
    const double* xi = coord + 3 * ia;
    const double* xj = coord + 3 * ja;
    const int noi = L.iorbs[ia], noj = L.iorbs[ja];
    double di[5][5];
    h1elec(ni, nj, xi, xj, di);
    double* hb = h + L.pair_off[e];
    for (int a = 1; a <= noi; ++a)
      for (int b = 1; b <= noj; ++b) hb[(a - 1) * noj + (b - 1)] = di[a][b];
    const int li = noi * (noi + 1) / 2, lj = noj * (noj + 1) / 2;
    double* wb = w + L.pair_woff[e];
    const double dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
    if (dx * dx + dy * dy + dz * dz < 0.00002) {
      for (int x = 0; x < li * lj; ++x) wb[x] = 0.0;
      enuc_entry[e] = 0.0;
      continue;
    }
    double p[4][4];
    const double r = rotmat(xi, xj, p);
    double ri[23], gab;
    reppd(ni, nj, r, ri, &gab);
    w_block(ni, nj, p, ri, wb);
    enuc_entry[e] = ccrep(ni, nj, r / PM7_A0, gab);
  }
}

// The diagonal-block terms of a pair outside cutof2: outer2 (MOZYME/outer2.F90,
// mode 0: reppd's monopole and dipoles along the unit vector j -> i) in
// cutof1's band, outer1 (MOZYME/outer1.F90, mode 0: a feathered point charge)
// beyond it.  e1b: atom i's block, e2a: atom j's (packed, 10 for sp).
__device__ void mz_outer_terms(int ni, int nj, const double* ci, const double* cj, bool band, double* e1b,
                               double* e2a) {
  for (int k = 0; k < 10; ++k) { e1b[k] = 0.0; e2a[k] = 0.0; }
  const Pm7Elem& I = c_P.el[ni];
  const Pm7Elem& J = c_P.el[nj];
  if (!band) {
    const double rij = sqrt((ci[0] - cj[0]) * (ci[0] - cj[0]) + (ci[1] - cj[1]) * (ci[1] - cj[1]) +
                            (ci[2] - cj[2]) * (ci[2] - cj[2]));
    const double r = rij / PM7_A0;
    double aee = 0.5 / I.am + 0.5 / J.am;
    aee = aee * aee;
    double ww = PM7_EV / sqrt(r * r + aee), point, cst;
    to_point(rij, &point, &cst);
    ww = ww * cst + (1.0 - cst) * point;
    const int dg[4] = {0, 2, 5, 9};
    for (int k = 0; k < 4; ++k) {
      e1b[dg[k]] = -ww * J.tore;
      e2a[dg[k]] = -ww * I.tore;
    }
    return;
  }
  double x[3] = {ci[0] - cj[0], ci[1] - cj[1], ci[2] - cj[2]};
  const double rij = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
  double ri[23], gab;
  reppd(ni, nj, rij, ri, &gab);
  const double a = 1.0 / rij;
  x[0] *= a; x[1] *= a; x[2] *= a;
  if (fabs(x[2]) > 0.99999999) x[2] = x[2] >= 0.0 ? 1.0 : -1.0;
  const double w1 = ri[1];
  e1b[0] = -w1 * J.tore;
  e2a[0] = -w1 * I.tore;
  if (J.natorb > 1) {
    const double w2 = -ri[5] * x[0], w3 = -ri[5] * x[1], w4 = -ri[5] * x[2];
    e2a[1] = -w2 * I.tore; e2a[2] = -w1 * I.tore; e2a[3] = -w3 * I.tore;
    e2a[5] = -w1 * I.tore; e2a[6] = -w4 * I.tore; e2a[9] = -w1 * I.tore;
  }
  if (I.natorb > 1) {
    const double w5 = -ri[2] * x[0], w6 = -ri[2] * x[1], w7 = -ri[2] * x[2];
    e1b[1] = -w5 * J.tore; e1b[2] = -w1 * J.tore; e1b[3] = -w6 * J.tore;
    e1b[5] = -w1 * J.tore; e1b[6] = -w7 * J.tore; e1b[9] = -w1 * J.tore;
  }
}

// A warp per atom A; the partners B are taken 32 at a time, one per lane,
// and every lane's terms are then added in lane order, so the one-centre
// block and the core-core energy are summed over B in ascending order, the
// reference loop's order, bit for bit.
__global__ void __launch_bounds__(128) mz_hcore_diag(MbMzLayout L, const int* __restrict__ nat,
                                                     const double* __restrict__ coord, double* __restrict__ h,
                                                     double* __restrict__ w, const double* __restrict__ enuc_entry,
                                                     double* __restrict__ enuc_atom) {
  __shared__ int entry_of[4][32];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int A = blockIdx.x * 4 + wib;
  if (A >= L.numat) return;  // warp-uniform
  const int nA = nat[A], noA = L.iorbs[A], lA = noA * (noA + 1) / 2;
  const Pm7Elem& E = c_P.el[nA];
  double blk[10];
  for (int x = 0; x < 10; ++x) blk[x] = 0.0;
  blk[0] = E.uss;
  if (noA == 4) { blk[2] = E.upp; blk[5] = E.upp; blk[9] = E.upp; }
  const double* xa = coord + 3 * A;
  int ep = L.pair_ptr[A];                 // A's stored partners (ascending), then its own block
  const int ediag = L.pair_ptr[A + 1] - 1;
  double en = 0.0;
  for (int b0 = 0; b0 < L.numat; b0 += 32) {
    const int B = b0 + lane;
    // which partners of this chunk are stored pairs, and their entries
    entry_of[wib][lane] = -1;
    __syncwarp();
    {
      const int e = ep + lane;
      const int pj = e < ediag ? L.pair_j[e] : -1;
      const bool in = pj >= b0 && pj < b0 + 32;
      if (in) entry_of[wib][pj - b0] = e;
      ep += __popc(__ballot_sync(0xffffffffu, in));
    }
    __syncwarp();
    const int my_entry = entry_of[wib][lane];
    double cen = 0.0;        // this lane's core-core term (B < A)
    double c[10];            // this lane's contribution to A's one-centre block
    for (int x = 0; x < 10; ++x) c[x] = 0.0;
    bool has_c = false;
    if (B < L.numat && B != A) {
      const double* xb = coord + 3 * B;
      const double dx = xa[0] - xb[0], dy = xa[1] - xb[1], dz = xa[2] - xb[2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      const int nB = nat[B];
      if (B < A) {
        if (my_entry >= 0) {
          cen = enuc_entry[my_entry];
        } else if (r2 < L.cutof1) {       // outer2: monopole term
          double ri[23], gab;
          reppd(nA, nB, sqrt(r2), ri, &gab);
          cen = c_P.el[nA].tore * c_P.el[nB].tore * ri[1];
        } else {                          // outer1: feathered point charge
          const double rij = sqrt(r2), rb = rij / PM7_A0;
          double aee = 0.5 / E.am + 0.5 / c_P.el[nB].am;
          aee = aee * aee;
          double ww = PM7_EV / sqrt(rb * rb + aee), point, cst;
          to_point(rij, &point, &cst);
          ww = ww * cst + (1.0 - cst) * point;
          cen = c_P.el[nA].tore * c_P.el[nB].tore * ww;
        }
      }
      if (!(r2 < 0.00002)) {
        double e1b[10], e2a[10];
        has_c = true;
        if (!(r2 < L.cutof2) && sqrt(r2) < 7.0) {
          // a far pair inside PM7's 7 A feathering radius (a cutoff below
          // 7 A): outer1's or outer2's terms; beyond 7 A elenuc's feathered
          // integrals are the same point charges
          if (B < A) {
            mz_outer_terms(nA, nB, xa, xb, r2 < L.cutof1, e1b, e2a);
            for (int x = 0; x < 10; ++x) if (x < lA) c[x] = e1b[x];
          } else {
            mz_outer_terms(nB, nA, xb, xa, r2 < L.cutof1, e1b, e2a);
            for (int x = 0; x < 10; ++x) if (x < lA) c[x] = e2a[x];
          }
        } else {
          double p[4][4], core[5][3];
          if (B < A) {
            const double r = rotmat(xa, xb, p);
            core_terms(nA, nB, r, core);
            elenuc(p, core, noA, L.iorbs[B], e1b, e2a);
            for (int x = 0; x < 10; ++x) if (x < lA) c[x] = e1b[x];
          } else {
            const double r = rotmat(xb, xa, p);
            core_terms(nB, nA, r, core);
            elenuc(p, core, L.iorbs[B], noA, e1b, e2a);
            for (int x = 0; x < 10; ++x) if (x < lA) c[x] = e2a[x];
          }
        }
      }
    }
    // the lanes' terms in ascending B
    const unsigned cmask = __ballot_sync(0xffffffffu, has_c);
    const unsigned emask = __ballot_sync(0xffffffffu, B < A);
    for (int src = 0; src < 32; ++src) {
      const double ce = __shfl_sync(0xffffffffu, cen, src);
      if ((emask >> src) & 1u) en += ce;
#pragma unroll
      for (int x = 0; x < 10; ++x) {
        if (x < lA) {  // lA is the warp's own, so every lane takes the shuffle or none
          const double v = __shfl_sync(0xffffffffu, c[x], src);
          if ((cmask >> src) & 1u) blk[x] = blk[x] + v * 1.0;
        }
      }
    }
    __syncwarp();
  }
  if (lane != 0) return;
  enuc_atom[A] = en;
  double* hd = h + L.pair_off[ediag];
  for (int x = 0; x < lA; ++x) hd[x] = blk[x];
  double* w1 = w + L.pair_woff[ediag];
  for (int x = 0; x < lA * lA; ++x) w1[x] = 0.0;
#define WS(a, b) w1[((a) - 1) + lA * ((b) - 1)]
  WS(1, 1) = E.gss;
  if (noA == 4) {
    const int ipx = 3, ipy = 6, ipz = 10;
    WS(ipx, 1) = E.gsp; WS(ipy, 1) = E.gsp; WS(ipz, 1) = E.gsp;
    WS(1, ipx) = E.gsp; WS(1, ipy) = E.gsp; WS(1, ipz) = E.gsp;
    WS(ipx, ipx) = E.gpp; WS(ipy, ipy) = E.gpp; WS(ipz, ipz) = E.gpp;
    WS(ipy, ipx) = E.gp2; WS(ipz, ipx) = E.gp2; WS(ipz, ipy) = E.gp2;
    WS(ipx, ipy) = E.gp2; WS(ipx, ipz) = E.gp2; WS(ipy, ipz) = E.gp2;
    WS(2, 2) = E.hsp; WS(4, 4) = E.hsp; WS(7, 7) = E.hsp;
    WS(5, 5) = 0.5 * (E.gpp - E.gp2); WS(8, 8) = 0.5 * (E.gpp - E.gp2); WS(9, 9) = 0.5 * (E.gpp - E.gp2);
  }
#undef WS
}

// ---------------------------------------------------------------- gradients
// Density blocks of the diatomic (atom 1 = jj, atom 2 = ii > jj): atom 1's,
// atom 2's, and rows of atom 2 by columns of atom 1.
struct PairDens {
  double p1[4][4], p2[4][4], p21[4][4];
};

__device__ __forceinline__ int pairix(int a, int b) {  // 0-based pair index of local orbitals a, b
  return a > b ? a * (a + 1) / 2 + b : b * (b + 1) / 2 + a;
}

// Energy of the diatomic in dhc's form (forces/dhc.F90:59-173, a molecule,
// RHF): h1elec's resonance block, the electron-core blocks, the two-centre
// Coulomb and exchange terms with the density fixed, helect over the pair's
// orbitals (doubled), and ccrep's core-core term; eV.  Like dhc it leaves out
// every term that does not depend on the pair's geometry.
__device__ double dhc_energy(int n1, int n2, const double* x1, const double* x2, const PairDens& d) {
  const int nor1 = c_P.el[n1].natorb, nor2 = c_P.el[n2].natorb;
  const int lim1 = nor1 * (nor1 + 1) / 2, lim2 = nor2 * (nor2 + 1) / 2;
  double di[5][5];
  h1elec(n1, n2, x1, x2, di);  // di[a][b]: a on atom 1, b on atom 2
  double h1[10], h2[10], wb[100], enuc = 0.0;
  for (int x = 0; x < 10; ++x) { h1[x] = 0.0; h2[x] = 0.0; }
  for (int x = 0; x < 100; ++x) wb[x] = 0.0;
  const double dx = x2[0] - x1[0], dy = x2[1] - x1[1], dz = x2[2] - x1[2];
  if (dx * dx + dy * dy + dz * dz >= 0.00002) {
    double p[4][4];
    const double r = rotmat(x2, x1, p);  // rotate(ni = atom 2, nj = atom 1) as dhc calls it
    double ri[23], gab;
    reppd(n2, n1, r, ri, &gab);
    w_block(n2, n1, p, ri, wb);  // lim2 x lim1, atom 1's pair index fastest
    double core[5][3];
    core_terms(n2, n1, r, core);
    elenuc(p, core, nor2, nor1, h2, h1);  // atom 2's electrons: e1b; atom 1's: e2a
    enuc = ccrep(n2, n1, r / PM7_A0, gab);
  }
  // Coulomb terms on each atom's block from the other atom's density, and the
  // energy of the diagonal blocks: sum' P (H + F), F = H + G
  double e = 0.0;
  for (int a = 0; a < nor1; ++a)
    for (int b = 0; b <= a; ++b) {
      const int q = pairix(a, b);
      double g = 0.0;
      for (int x = 0; x < nor2; ++x)
        for (int y = 0; y < nor2; ++y) g += d.p2[x][y] * wb[pairix(x, y) * lim1 + q];
      const double wgt = a == b ? 0.5 : 1.0;
      e += wgt * d.p1[a][b] * (2.0 * h1[q] + g);
    }
  for (int a = 0; a < nor2; ++a)
    for (int b = 0; b <= a; ++b) {
      const int q = pairix(a, b);
      double g = 0.0;
      for (int x = 0; x < nor1; ++x)
        for (int y = 0; y < nor1; ++y) g += d.p1[x][y] * wb[q * lim1 + pairix(x, y)];
      const double wgt = a == b ? 0.5 : 1.0;
      e += wgt * d.p2[a][b] * (2.0 * h2[q] + g);
    }
  // the off-diagonal block: resonance and exchange (kab), PA = P / 2
  for (int mu = 0; mu < nor2; ++mu)
    for (int nu = 0; nu < nor1; ++nu) {
      double k = 0.0;
      for (int la = 0; la < nor2; ++la)
        for (int si = 0; si < nor1; ++si) k += 0.5 * d.p21[la][si] * wb[pairix(mu, la) * lim1 + pairix(nu, si)];
      e += d.p21[mu][nu] * (2.0 * di[nu + 1][mu + 1] - k);
    }
  (void)lim2;
  // 2 * helect(PA, H, F) with PA = P/2 is sum' P (H + F) = e
  return e + enuc;
}

// dcart (forces/dcart.F90:60-300) for a molecule with the default finite
// difference (no FORCE keyword): pair q = (ii, jj), jj < ii, with atom jj
// moved by chnge/2 along all three axes, then atom ii by chnge along each
// axis in turn; deriv = (E0 - Ek) * fpc_9 / chnge, kcal/mol/A.
__global__ void dcart_pairs(int numat, const int* __restrict__ nat, const double* __restrict__ coord, MbAtomsDev at,
                            const double* __restrict__ ptot, double* __restrict__ deriv) {
  const long long npair = (long long)numat * (numat - 1) / 2;
  const double chnge = 1.0e-4, chnge2 = chnge * 0.5;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < npair;
       q += (long long)gridDim.x * blockDim.x) {
    long long i = (long long)((sqrt(8.0 * (double)q + 1.0) + 1.0) * 0.5);
    while (i * (i - 1) / 2 > q) --i;
    while ((i + 1) * i / 2 <= q) ++i;
    const int ii = (int)i, jj = (int)(q - i * (i - 1) / 2);
    const int f1 = at.first[jj], f2 = at.first[ii], no1 = at.nor[jj], no2 = at.nor[ii];
    PairDens d;
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) {
        d.p1[a][b] = (a < no1 && b < no1) ? ptot[mb_tri(f1 + (a > b ? a : b), f1 + (a > b ? b : a))] : 0.0;
        d.p2[a][b] = (a < no2 && b < no2) ? ptot[mb_tri(f2 + (a > b ? a : b), f2 + (a > b ? b : a))] : 0.0;
        d.p21[a][b] = (a < no2 && b < no1) ? ptot[mb_tri(f2 + a, f1 + b)] : 0.0;
      }
    double x1[3], x2[3];
    for (int k = 0; k < 3; ++k) {
      x1[k] = coord[3 * jj + k] + chnge2;
      x2[k] = coord[3 * ii + k];
    }
    const int n1 = nat[jj], n2 = nat[ii];
    const double aa = dhc_energy(n1, n2, x1, x2, d);
    for (int k = 0; k < 3; ++k) {
      x2[k] = x2[k] + chnge;
      const double ee = dhc_energy(n1, n2, x1, x2, d);
      x2[k] = x2[k] - chnge2;
      x2[k] = x2[k] - chnge2;
      deriv[3 * q + k] = (aa - ee) * PM7_FPC9 / chnge;
    }
  }
}

// dxyz of atom a in dcart's accumulation order: the pairs (a, jj < a), then
// the pairs (ii > a, a), each ascending.
__global__ void dcart_sum(int numat, const double* __restrict__ deriv, double* __restrict__ dxyz) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * numat) return;
  const int a = t / 3, k = t - 3 * a;
  double g = 0.0;
  for (int b = 0; b < a; ++b) g = g - deriv[3 * ((long long)a * (a - 1) / 2 + b) + k];
  for (int b = a + 1; b < numat; ++b) g = g + deriv[3 * ((long long)b * (b - 1) / 2 + a) + k];
  dxyz[t] = g;
}

bool g_params_uploaded = false;

int upload_params() {
  if (g_params_uploaded) return MB_OK;
  Pm7Params P;
  pm7_init(&P);
  DevParams D;
  memcpy(D.el, P.el, sizeof(D.el));
  memcpy(D.xfac, P.xfac, sizeof(D.xfac));
  memcpy(D.alpb, P.alpb, sizeof(D.alpb));
  D.par1 = P.par1; D.par2 = P.par2; D.par3 = P.par3; D.par4 = P.par4;
  MB_CUDA(cudaMemcpyToSymbol(c_P, &D, sizeof(D)));
  g_params_uploaded = true;
  return MB_OK;
}

}  // namespace

extern "C" int mb_hcore_dev(const int* nat_d, const double* coord_d, const MbAtomsDev* at, int numat, double* h,
                            double* w, double* enuc_pairs, cudaStream_t stream) {
  MB_TRY(upload_params());
  const long long npair = (long long)numat * (numat - 1) / 2;
  if (npair > 0) {
    int blocks = (int)((npair + 127) / 128);
    if (blocks > 148 * 32) blocks = 148 * 32;
    hcore_pairs<<<blocks, 128, 0, stream>>>(numat, nat_d, coord_d, *at, h, w, enuc_pairs);
    MB_LAUNCH_CHECK();
  }
  hcore_diag<<<(numat + 63) / 64, 64, 0, stream>>>(numat, nat_d, coord_d, *at, h, w);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

extern "C" int mb_hcore_batch_dev(const MbHcoreBatch* b, cudaStream_t stream) {
  if (!b || b->nmol <= 0) return mb_set_error(MB_ERR_ARG, "mb_hcore_batch_dev: bad args");
  MB_TRY(upload_params());
  const long long npair = b->npair_tot, natom = b->natom_tot;
  if (npair > 0) {
    const int blocks = (int)std::min<long long>((npair + 127) / 128, 148LL * 32);
    hcore_pairs_batch<<<blocks, 128, 0, stream>>>(*b);
    MB_LAUNCH_CHECK();
  }
  const int blocks = (int)std::min<long long>((natom + 63) / 64, 148LL * 32);
  hcore_diag_batch<<<blocks, 64, 0, stream>>>(*b);
  MB_LAUNCH_CHECK();
  enuc_sum_batch<<<b->nmol, 1024, 0, stream>>>(*b);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

extern "C" int mb_hcore_finish(int numat, const MbAtomsDev* at, const int* nat_d, double* h, const double* e1b,
                               double* enuclr_dev, const double* enuc_pairs, cudaStream_t stream) {
  (void)at; (void)nat_d; (void)h; (void)e1b;
  const long long npair = (long long)numat * (numat - 1) / 2;
  if (npair == 0) {
    MB_CUDA(cudaMemsetAsync(enuclr_dev, 0, sizeof(double), stream));
    return MB_OK;
  }
  enuc_sum<<<1, 1024, 0, stream>>>(npair, enuc_pairs, enuclr_dev);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

// hcore_for_MOZYME on the pair blocks: h (layout mpack), w (layout nw: the
// stored pairs' two-centre blocks and every atom's one-centre block),
// *enuclr_dev (device) the core-core energy over every atom pair.  ws:
// mb_mz_hcore_ws_bytes(layout) bytes of device scratch.
extern "C" size_t mb_mz_hcore_ws_bytes(const MbMzLayout* L) {
  return L ? sizeof(double) * (size_t)(L->npairs + L->numat) : 0;
}

extern "C" int mb_mz_hcore_dev(const MbMzLayout* L, const int* nat_d, const double* coord_d, double* h, double* w,
                               double* enuclr_dev, void* ws, cudaStream_t stream) {
  if (!L || !nat_d || !coord_d || !h || !w || !enuclr_dev || !ws || L->numat <= 0)
    return mb_set_error(MB_ERR_ARG, "mb_mz_hcore_dev: bad args");
  // Far pairs past PM7's 7 A feathering (mndod.F90:800-822) take the
  // rotated core attraction, which there is outer1's and outer2's point
  // charge; those inside 7 A (a cutoff below 7 A) take outer1's and outer2's
  // own terms, and every far pair the outer core-core term.
  MB_TRY(upload_params());
  double* enuc_entry = (double*)ws;
  double* enuc_atom = enuc_entry + L->npairs;
  if (L->npairs > 0) {
    const int blocks = (int)std::min<long long>((L->npairs + 127) / 128, 148LL * 32);
    mz_hcore_pairs<<<blocks, 128, 0, stream>>>(*L, nat_d, coord_d, h, w, enuc_entry);
    MB_LAUNCH_CHECK();
  }
  mz_hcore_diag<<<(L->numat + 3) / 4, 128, 0, stream>>>(*L, nat_d, coord_d, h, w, enuc_entry, enuc_atom);
  MB_LAUNCH_CHECK();
  enuc_sum<<<1, 1024, 0, stream>>>(L->numat, enuc_atom, enuclr_dev);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

extern "C" size_t mb_dcart_ws_bytes(int numat) {
  if (numat < 2) return 0;
  return sizeof(double) * 3 * ((size_t)numat * (numat - 1) / 2);
}

// Cartesian gradient of the SCF energy (dcart, forces/dcart.F90:16-300, a
// molecule, RHF): dxyz_dev[3a + k] in kcal/mol/A for the packed density p.
extern "C" int mb_dcart_dev(const int* nat_d, const double* coord_d, const MbAtomsDev* at, int numat, const double* p,
                            double* dxyz_dev, void* ws, size_t ws_bytes, cudaStream_t stream) {
  if (!at || numat <= 0 || !nat_d || !coord_d || !p || !dxyz_dev) return mb_set_error(MB_ERR_ARG, "mb_dcart_dev: bad args");
  if (ws_bytes < mb_dcart_ws_bytes(numat) || (numat > 1 && !ws))
    return mb_set_error(MB_ERR_ARG, "mb_dcart_dev: workspace smaller than mb_dcart_ws_bytes(numat)");
  MB_TRY(upload_params());
  const long long npair = (long long)numat * (numat - 1) / 2;
  if (npair > 0) {
    int blocks = (int)((npair + 127) / 128);
    if (blocks > 148 * 32) blocks = 148 * 32;
    dcart_pairs<<<blocks, 128, 0, stream>>>(numat, nat_d, coord_d, *at, p, (double*)ws);
    MB_LAUNCH_CHECK();
    dcart_sum<<<(3 * numat + 127) / 128, 128, 0, stream>>>(numat, (const double*)ws, dxyz_dev);
    MB_LAUNCH_CHECK();
  } else {
    MB_CUDA(cudaMemsetAsync(dxyz_dev, 0, sizeof(double) * 3 * (size_t)numat, stream));
  }
  return MB_OK;
}
