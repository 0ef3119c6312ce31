// Batched SCF: many small molecules (n <= 128 basis functions), each SCF run
// start to finish by one CTA of a persistent kernel.
//
// A CTA takes the next molecule from a shared counter (uneven sizes balance
// themselves) and restates iter (SCF/iter.F90:16-1107) for it in the same
// form as mb_scf_run with full diagonalisation every iteration: level shift,
// Fock build, energy, convergence test, eigensolve, density, cnvg, and the
// exit diagonalisation.  Every thread computes the control scalars from the
// same CTA-wide values (so they agree bit for bit); the CTA runs the phases
// between barriers:
//   * Fock: thread per atom folds its diagonal block's contributions in the
//     reference order (pairs with lower atoms, its one-centre terms, pairs
//     with higher atoms) and writes the exchange blocks of its lower pairs --
//     the operation order of fock2/fock1, so F is bit-identical to the oracle;
//   * eigensolve of the packed F in shared memory: Householder reduction to
//     tridiagonal form, eigenvalues 0..nocc by 5-section Sturm counts (four
//     lanes per eigenvalue), occupied eigenvectors of T by inverse iteration
//     (thread per vector, clusters re-orthogonalised), back-transformation;
//   * density P = 2 Z Z^T over the occupied vectors; cnvg with its diagonal
//     statistics in the reference's order (bit-identical).
// Matrices live in shared memory (packed F, the n x nocc vectors) and in a
// CTA-private global scratch (the packed F, P, PA, P_old, the LU factors).
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "mb_common.cuh"
#include "pm7_params.h"

extern "C" int mb_hcore_dev(const int* nat_d, const double* coord_d, const MbAtomsDev* at, int numat, double* h,
                            double* w, double* enuc_pairs, cudaStream_t stream);
extern "C" int mb_hcore_finish(int numat, const MbAtomsDev* at, const int* nat_d, double* h, const double* e1b,
                               double* enuclr_dev, const double* enuc_pairs, cudaStream_t stream);

namespace {

constexpr int BT_T = 256;         // threads per CTA
constexpr int BT_NMAX = 128;      // basis functions per molecule
constexpr int BT_ZMAX = 11008;    // n * nocc doubles in shared memory

struct Mol {
  int n, nclose, numat, aoff;  // aoff: first atom in the concatenated atom tables
  long long hoff, woff;        // offsets into packed arrays / W
  int doff, pad;               // offset into per-orbital arrays
  double enuclr, atheat;
};

struct BatchArgs {
  const Mol* mol;
  const int* order;          // molecules in the order the CTAs take them
  int nmol;
  const int* first;          // molecule-local first orbital of each atom
  const int* nor;
  const double* h;
  const double* w;
  const long long* wrow;     // molecule-local W offsets of each atom's first pair block
  const int* lim;
  const int* cum;
  const double* pdiag;
  double* f;
  double* p;
  double* pa;
  double* pold;
  double* pold2;
  double* scratch;           // per CTA: 3 * BT_NMAX * BT_NMAX doubles (LU factors)
  double* escf;
  double* ee;
  int* niter;
  int* conv;
  double* homo;
  double* lumo;
  int* next;
  int* status;
  int itrmax;
  double scfcrt;
};

__device__ __forceinline__ long long tri(long long r, long long c) { return r * (r + 1) / 2 + c; }
__device__ __forceinline__ int indx1(int i, int j) { if (i < j) { int t = i; i = j; j = t; } return (i * (i - 1)) / 2 + j; }

__constant__ int c_bpidx[16] = {1, 2, 4, 7, 2, 3, 5, 8, 4, 5, 6, 9, 7, 8, 9, 10};

// ------------------------------------------------------------ Fock (one atom)
// F(a's diagonal block) and the exchange blocks of pairs (a, b < a), in the
// operation order of fock2 (SCF/fock2.F90:149-298) and fock1 (SCF/fock1.F90).
__device__ void fock_atom(const BatchArgs& B, const Mol& M, int a, const double* __restrict__ ptot,
                          const double* __restrict__ p, double* __restrict__ f) {
  const int* first = B.first + M.aoff;
  const int* nor = B.nor + M.aoff;
  const long long* wrow = B.wrow + M.aoff;
  const int* lim = B.lim + M.aoff;
  const int* cum = B.cum + M.aoff;
  const double* w = B.w + M.woff;
  const int ia = first[a] + 1, ib = first[a] + nor[a];  // 1-based orbitals
  const int na = nor[a];
  const int nd = na * (na + 1) / 2;
  double acc[10];
  for (int t = 0; t < nd; ++t) {
    int r = 0;
    while ((r + 1) * (r + 2) / 2 <= t) ++r;
    const int c = t - r * (r + 1) / 2;
    acc[t] = f[tri(ia - 1 + r, ia - 1 + c)];
  }
  auto pairw = [&](int hi, int lo) { return w + wrow[hi] + (long long)lim[hi] * cum[lo]; };
  auto pk = [&](int r1, int c1) -> double {  // packed element, 1-based orbitals
    const int mx = r1 > c1 ? r1 : c1, mn = r1 < c1 ? r1 : c1;
    return ptot[tri(mx - 1, mn - 1)];
  };
  // contribution of pair (hi, lo) to atom a's diagonal block
  auto pair_terms = [&](int hi, int lo) {
    const double* wk = pairw(hi, lo);
    const int ha = first[hi] + 1, hb = first[hi] + nor[hi];
    const int la = first[lo] + 1, lb = first[lo] + nor[lo];
    if (hb - ha >= 3 && lb - la >= 3) {
      // jab: hi's block gets sumb (from lo's density), lo's block gets suma
      const int oa = (a == hi) ? la : ha;  // the other atom's first orbital
      for (int q = 0; q < 10; ++q) {
        double s;
        if (a == hi) {
          s = DMUL(pk(oa + 0, oa + 0), wk[q * 10 + c_bpidx[0] - 1]);
          for (int m = 1; m < 16; ++m) s = DADD(s, DMUL(pk(oa + m / 4, oa + m % 4), wk[q * 10 + c_bpidx[m] - 1]));
        } else {
          s = DMUL(pk(oa + 0, oa + 0), wk[(c_bpidx[0] - 1) * 10 + q]);
          for (int m = 1; m < 16; ++m) s = DADD(s, DMUL(pk(oa + m / 4, oa + m % 4), wk[(c_bpidx[m] - 1) * 10 + q]));
        }
        acc[q] = DADD(acc[q], s);
      }
    } else if (hb - ha >= 3 && la == lb) {  // hi heavy, lo light
      const double pl = ptot[tri(la - 1, la - 1)];
      if (a == hi) {
        int k = 0;
        for (int i = 0; i <= 3; ++i) {
          for (int j = 1; j <= i; ++j) {
            acc[i * (i + 1) / 2 + j - 1] = DADD(acc[i * (i + 1) / 2 + j - 1], DMUL(pl, wk[j + k - 1]));
          }
          if (i > 0) k += i;
          k += 1;
          acc[i * (i + 1) / 2 + i] = DADD(acc[i * (i + 1) / 2 + i], DMUL(pl, wk[k - 1]));
        }
      } else {
        double sumdia = 0.0, sumoff = 0.0;
        int k = 0;
        for (int i = 0; i <= 3; ++i) {
          for (int j = 1; j <= i; ++j) sumoff = DADD(sumoff, DMUL(pk(ha + i, ha + j - 1), wk[j + k - 1]));
          if (i > 0) k += i;
          k += 1;
          sumdia = DADD(sumdia, DMUL(pk(ha + i, ha + i), wk[k - 1]));
        }
        acc[0] = DADD(DADD(acc[0], DMUL(sumoff, 2.0)), sumdia);
      }
    } else if (lb - la >= 3 && ha == hb) {  // hi light, lo heavy
      const double ph = ptot[tri(ha - 1, ha - 1)];
      if (a == lo) {
        int k = 0;
        for (int i = 0; i <= 3; ++i) {
          for (int j = 1; j <= i; ++j) acc[i * (i + 1) / 2 + j - 1] = DADD(acc[i * (i + 1) / 2 + j - 1], DMUL(ph, wk[j + k - 1]));
          if (i > 0) k += i;
          k += 1;
          acc[i * (i + 1) / 2 + i] = DADD(acc[i * (i + 1) / 2 + i], DMUL(ph, wk[k - 1]));
        }
      } else {
        double sumdia = 0.0, sumoff = 0.0;
        int k = 0;
        for (int i = 0; i <= 3; ++i) {
          for (int j = 1; j <= i; ++j) sumoff = DADD(sumoff, DMUL(pk(la + i, la + j - 1), wk[j + k - 1]));
          if (i > 0) k += i;
          k += 1;
          sumdia = DADD(sumdia, DMUL(pk(la + i, la + i), wk[k - 1]));
        }
        acc[0] = DADD(DADD(acc[0], DMUL(sumoff, 2.0)), sumdia);
      }
    } else {  // light-light
      const double po = (a == hi) ? ptot[tri(la - 1, la - 1)] : ptot[tri(ha - 1, ha - 1)];
      acc[0] = DADD(acc[0], DMUL(po, wk[0]));
    }
  };
  for (int b = 0; b < a; ++b) pair_terms(a, b);
  // fock1: one-centre terms of atom a
  {
    const int il = nd;
    const double* wo = w + wrow[a] + (long long)lim[a] * cum[a];
    for (int i = ia; i <= ib; ++i) {
      const int iw = i - ia + 1;
      for (int j = ia; j <= i; ++j) {
        const int jw = j - ia + 1;
        const int ijw = (iw * (iw - 1)) / 2 + jw;
        double sum = 0.0;
        for (int k = ia; k <= ib; ++k) {
          const int kw = k - ia + 1;
          for (int l = ia; l <= ib; ++l) {
            const int lw = l - ia + 1;
            const int klw = indx1(kw, lw), ikw = indx1(kw, jw), jlw = indx1(lw, iw);
            const double pt = pk(k, l), ps = p[tri((k > l ? k : l) - 1, (k < l ? k : l) - 1)];
            sum = DSUB(DADD(sum, DMUL(pt, wo[(ijw - 1) + il * (klw - 1)])), DMUL(ps, wo[(ikw - 1) + il * (jlw - 1)]));
          }
        }
        acc[ijw - 1] = DADD(acc[ijw - 1], sum);
      }
    }
  }
  for (int b = a + 1; b < M.numat; ++b) pair_terms(b, a);
  for (int t = 0; t < nd; ++t) {
    int r = 0;
    while ((r + 1) * (r + 2) / 2 <= t) ++r;
    const int c = t - r * (r + 1) / 2;
    f[tri(ia - 1 + r, ia - 1 + c)] = acc[t];
  }
  // exchange blocks of the pairs (a, b < a): one subtraction per element
  for (int b = 0; b < a; ++b) {
    const double* wk = pairw(a, b);
    const int ja = first[b] + 1, jb = first[b] + nor[b];
    if (ib - ia >= 3 && jb - ja >= 3) {
      for (int mu = 1; mu <= 4; ++mu)
        for (int nu = 1; nu <= 4; ++nu) {
          double s = 0.0;
          bool firstt = true;
          for (int lam = 1; lam <= 4; ++lam)
            for (int sig = 1; sig <= 4; ++sig) {
              const double t = DMUL(p[tri(ia + lam - 2, ja + sig - 2)], wk[(indx1(mu, lam) - 1) * 10 + indx1(nu, sig) - 1]);
              if (firstt) { s = t; firstt = false; } else s = DADD(s, t);
            }
          const long long idx = tri(ia + mu - 2, ja + nu - 2);
          f[idx] = DSUB(f[idx], s);
        }
    } else if (ib - ia >= 3 && ja == jb) {
      for (int i = ia; i <= ib; ++i) {
        double sum = 0.0;
        for (int j = 1; j <= ib - ia + 1; ++j) sum = DADD(sum, DMUL(p[tri(j - 1 + ia - 1, ja - 1)], wk[indx1(i - ia + 1, j) - 1]));
        const long long idx = tri(i - 1, ja - 1);
        f[idx] = DSUB(f[idx], sum);
      }
    } else if (jb - ja >= 3 && ia == ib) {
      for (int i = 0; i < 4; ++i) {
        double sum = 0.0;
        for (int l = 1; l <= 4; ++l) sum = DADD(sum, DMUL(p[tri(ia - 1, ja - 1) + l - 1], wk[indx1(i + 1, l) - 1]));
        const long long idx = tri(ia - 1, ja - 1) + i;
        f[idx] = DSUB(f[idx], sum);
      }
    } else {
      const long long ij = tri(ia - 1, ja - 1);
      f[ij] = DSUB(f[ij], DMUL(p[ij], wk[0]));
    }
  }
}

// Sturm count of T - x I (d, e2 = e^2).
__device__ int sturm(int n, const double* d, const double* e2, double x, double pivmin) {
  int cnt = 0;
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  cnt += q < 0.0;
  for (int i = 1; i < n; ++i) {
    q = d[i] - x - e2[i - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    cnt += q < 0.0;
  }
  return cnt;
}

struct Smem {
  double* A;     // packed lower, n(n+1)/2
  double* Z;     // n x nz, Z[i * nz + m]
  double* d;
  double* e;
  double* e2;
  double* tau;
  double* pv;    // p / w vector
  double* v;     // current Householder vector (full length n)
  double* eig;   // eigenvalues 0 .. nz
  double* red;   // reduction scratch (BT_T)
  double* scal;  // scalars
};

// Sum over the CTA, the same value in every thread: butterfly within each
// warp (commutative pairs, so every lane holds the same bits), then the warp
// sums in a fixed order.
__device__ double block_sum_all(double x, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = x;
  __syncthreads();
  double r = red[0];
#pragma unroll
  for (int q = 1; q < BT_T / 32; ++q) r += red[q];
  __syncthreads();
  return r;
}

// Eigenvalues 0..nz of the packed symmetric matrix in S.A (destroyed) and the
// eigenvectors of the lowest nz (in S.Z), using U (3 * n * nz doubles,
// global) for the LU factors.
__device__ void cta_eigh(int n, int nz, Smem& S, double* U) {
  const int tid = threadIdx.x;
  // ---- Householder reduction (lower, column k below the diagonal)
  for (int k = 0; k < n - 2; ++k) {
    double part = 0.0;
    for (int i = k + 2 + tid; i < n; i += BT_T) {
      const double x = S.A[tri(i, k)];
      part += x * x;
    }
    const double sigma = block_sum_all(part, S.red);
    if (tid == 0) {
      const double alpha = S.A[tri(k + 1, k)];
      double beta, tau, scal;
      if (sigma == 0.0) { beta = alpha; tau = 0.0; scal = 0.0; }
      else {
        beta = -copysign(sqrt(alpha * alpha + sigma), alpha);
        tau = (beta - alpha) / beta;
        scal = 1.0 / (alpha - beta);
      }
      S.scal[0] = tau;
      S.scal[1] = scal;
      S.e[k] = beta;
      S.tau[k] = tau;
      S.d[k] = S.A[tri(k, k)];
    }
    __syncthreads();
    const double tau = S.scal[0], scal = S.scal[1];
    for (int i = tid; i < n; i += BT_T) {
      double vi = 0.0;
      if (i == k + 1) vi = 1.0;
      else if (i > k + 1) {
        vi = S.A[tri(i, k)] * scal;
        S.A[tri(i, k)] = vi;  // reflector kept below the subdiagonal
      }
      S.v[i] = vi;
    }
    __syncthreads();
    if (tau == 0.0) continue;
    // p = tau A22 v over rows k+1..n-1
    double pvp = 0.0;
    for (int i = k + 1 + tid; i < n; i += BT_T) {
      double s = 0.0;
      for (int j = k + 1; j <= i; ++j) s += S.A[tri(i, j)] * S.v[j];
      for (int j = i + 1; j < n; ++j) s += S.A[tri(j, i)] * S.v[j];
      s *= tau;
      S.pv[i] = s;
      pvp += s * S.v[i];
    }
    const double dot = block_sum_all(pvp, S.red);
    const double kk = 0.5 * tau * dot;
    for (int i = k + 1 + tid; i < n; i += BT_T) S.pv[i] = S.pv[i] - kk * S.v[i];
    __syncthreads();
    // A22 -= v w^T + w v^T (lower triangle)
    const int m = n - k - 1;
    const long long cnt = (long long)m * (m + 1) / 2;
    for (long long q = tid; q < cnt; q += BT_T) {
      int r = (int)((sqrt(8.0 * (double)q + 1.0) - 1.0) * 0.5);
      while ((long long)r * (r + 1) / 2 > q) --r;
      while ((long long)(r + 1) * (r + 2) / 2 <= q) ++r;
      const int c = (int)(q - (long long)r * (r + 1) / 2);
      const int i = k + 1 + r, j = k + 1 + c;
      S.A[tri(i, j)] -= S.v[i] * S.pv[j] + S.pv[i] * S.v[j];
    }
    __syncthreads();
  }
  if (tid == 0) {
    if (n >= 2) {
      S.d[n - 2] = S.A[tri(n - 2, n - 2)];
      S.e[n - 2] = S.A[tri(n - 1, n - 2)];
      S.tau[n - 2] = 0.0;
    }
    S.d[n - 1] = S.A[tri(n - 1, n - 1)];
  }
  __syncthreads();
  // ---- bounds, e^2
  if (tid == 0) {
    double lo = 1e300, hi = -1e300, em = 0.0;
    for (int i = 0; i < n; ++i) {
      const double r = (i > 0 ? fabs(S.e[i - 1]) : 0.0) + (i < n - 1 ? fabs(S.e[i]) : 0.0);
      lo = fmin(lo, S.d[i] - r);
      hi = fmax(hi, S.d[i] + r);
      if (i < n - 1) { S.e2[i] = S.e[i] * S.e[i]; em = fmax(em, S.e2[i]); }
    }
    const double tnorm = fmax(fabs(lo), fabs(hi));
    const double pad = 2.0 * 2.220446049250313e-16 * tnorm * n + 1e-300;
    S.scal[4] = lo - pad;
    S.scal[5] = hi + pad;
    S.scal[6] = fmax(1e-290, 2.2250738585072014e-308 * fmax(1.0, em));
    S.scal[7] = tnorm;
  }
  __syncthreads();
  // ---- eigenvalues 0..nz by 5-section, four lanes per eigenvalue.  Every
  // lane runs the same rounds and steps (groups that have converged idle), so
  // the 4-lane shuffles always see a converged warp.
  {
    const int grp = tid >> 2, ln = tid & 3, base = tid & 31 & ~3;
    const double pivmin = S.scal[6];
    const double eps = 2.220446049250313e-16;
    const int nev = ((nz > 1 ? nz : 1) + 1 < n ? (nz > 1 ? nz : 1) + 1 : n);  // through the LUMO
    const int rounds = (nev + BT_T / 4 - 1) / (BT_T / 4);
    for (int rd = 0; rd < rounds; ++rd) {
      const int mm = rd * (BT_T / 4) + grp;
      const bool active = mm < nev;
      double lo = S.scal[4], hi = S.scal[5];
      bool done = !active;
      for (int it = 0; it < 100; ++it) {
        if (!done && hi - lo <= 2.0 * eps * fmax(fabs(lo), fabs(hi)) + pivmin) done = true;
        const double x = lo + (hi - lo) * ((double)(ln + 1) / 5.0);
        const int cnt = done ? 0 : sturm(n, S.d, S.e2, x, pivmin);
        const int flag = cnt > mm ? 1 : 0;
        int above = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) above |= __shfl_sync(0xffffffffu, flag, base + q) << q;
        double xs[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) xs[q] = __shfl_sync(0xffffffffu, x, base + q);
        if (!done) {
          double nlo = lo, nhi = hi;
          if (above == 0) {
            nlo = xs[3];
          } else {
            const int firstl = __ffs(above) - 1;
            nhi = xs[firstl];
            if (firstl > 0) nlo = xs[firstl - 1];
          }
          if (!(nlo > lo) && !(nhi < hi)) done = true;
          lo = nlo;
          hi = nhi;
        }
        if (__all_sync(0xffffffffu, done)) break;
      }
      if (active && ln == 0) S.eig[mm] = 0.5 * (lo + hi);
    }
  }
  __syncthreads();
  // ---- eigenvectors 0..nz-1 of T by inverse iteration (thread per cluster start)
  {
    const double tnorm = S.scal[7];
    const double ortol = 1.0e-8 * tnorm;
    const double eps = 2.220446049250313e-16;
    const double tiny = eps * fmax(tnorm, 1e-300);
    for (int m0 = tid; m0 < nz; m0 += BT_T) {
      if (m0 > 0 && !(S.eig[m0] - S.eig[m0 - 1] > ortol)) continue;
      int m1 = m0 + 1;
      while (m1 < nz && !(S.eig[m1] - S.eig[m1 - 1] > ortol)) ++m1;
      double* u0 = U + (long long)m0 * 3 * n;
      double* u1 = u0 + n;
      double* u2 = u1 + n;
      double lam_prev = 0.0;
      for (int mv = m0; mv < m1; ++mv) {
        double lam = S.eig[mv];
        if (mv > m0) {
          const double pertol = 10.0 * fabs(eps * lam) + tiny;
          if (lam - lam_prev < pertol) lam = lam_prev + pertol;
        }
        lam_prev = lam;
        double* x = S.Z + mv;  // stride nz
        unsigned long long s = 0x9E3779B97F4A7C15ull ^ (unsigned long long)(mv + 1) * 0xBF58476D1CE4E5B9ull;
        for (int i = 0; i < n; ++i) {
          s ^= s >> 31; s *= 0x94D049BB133111EBull; s ^= s >> 29;
          x[(long long)i * nz] = ((double)(s >> 11) * (1.0 / 9007199254740992.0)) - 0.5;
        }
        const int nits = (m1 - m0 > 1) ? 4 : 2;
        for (int itr = 0; itr < nits; ++itr) {
          // LU with partial pivoting of T - lam I, forward and back substitution
          double dd = S.d[0] - lam, du = n > 1 ? S.e[0] : 0.0, du2 = 0.0, xr = x[0];
          for (int i = 0; i < n - 1; ++i) {
            const double sub = S.e[i], dn = S.d[i + 1] - lam, en = (i + 1 < n - 1) ? S.e[i + 1] : 0.0;
            const double xn = x[(long long)(i + 1) * nz];
            if (fabs(dd) >= fabs(sub)) {
              double pv = dd;
              if (fabs(pv) < tiny) pv = copysign(tiny, pv == 0.0 ? 1.0 : pv);
              const double l = sub / pv;
              u0[i] = pv; u1[i] = du; u2[i] = du2;
              x[(long long)i * nz] = xr;
              dd = dn - l * du; du = en; du2 = 0.0; xr = xn - l * xr;
            } else {
              const double l = dd / sub;
              u0[i] = sub; u1[i] = dn; u2[i] = en;
              x[(long long)i * nz] = xn;
              const double ndd = du - l * dn, ndu = -l * en;
              dd = ndd; du = ndu; du2 = 0.0; xr = xr - l * xn;
            }
          }
          double last = dd;
          if (fabs(last) < tiny) last = copysign(tiny, last == 0.0 ? 1.0 : last);
          u0[n - 1] = last;
          double x1 = xr / last, x2 = 0.0;
          x[(long long)(n - 1) * nz] = x1;
          for (int i = n - 2; i >= 0; --i) {
            const double vv = (x[(long long)i * nz] - u1[i] * x1 - u2[i] * x2) / u0[i];
            x[(long long)i * nz] = vv;
            x2 = x1;
            x1 = vv;
          }
          for (int q = m0; q < mv; ++q) {  // re-orthogonalise against earlier members
            double dt = 0.0;
            for (int i = 0; i < n; ++i) dt += S.Z[(long long)i * nz + q] * x[(long long)i * nz];
            for (int i = 0; i < n; ++i) x[(long long)i * nz] -= dt * S.Z[(long long)i * nz + q];
          }
          double mx = 0.0, ss = 0.0;
          for (int i = 0; i < n; ++i) mx = fmax(mx, fabs(x[(long long)i * nz]));
          const double inv = mx > 0.0 ? 1.0 / mx : 0.0;
          for (int i = 0; i < n; ++i) { const double t = x[(long long)i * nz] * inv; ss += t * t; }
          const double sc = ss > 0.0 ? inv / sqrt(ss) : 0.0;
          for (int i = 0; i < n; ++i) x[(long long)i * nz] *= sc;
        }
      }
    }
  }
  __syncthreads();
  // ---- back-transformation Z <- H_0 ... H_{n-3} Z (thread per vector column)
  for (int k = n - 3; k >= 0; --k) {
    const double tau = S.tau[k];
    if (tau != 0.0) {
      for (int mcol = tid; mcol < nz; mcol += BT_T) {
        double s = S.Z[(long long)(k + 1) * nz + mcol];
        for (int i = k + 2; i < n; ++i) s += S.A[tri(i, k)] * S.Z[(long long)i * nz + mcol];
        s *= tau;
        S.Z[(long long)(k + 1) * nz + mcol] -= s;
        for (int i = k + 2; i < n; ++i) S.Z[(long long)i * nz + mcol] -= s * S.A[tri(i, k)];
      }
    }
  }
  __syncthreads();
}

// F of the molecule (H, the shifted start when use_shift, then fock2 + fock1).
__device__ void cta_fock(const BatchArgs& B, const Mol& M, double shift, bool use_shift, double* f,
                         const double* p, const double* pa, const double* h) {
  const long long mp = (long long)M.n * (M.n + 1) / 2;
  for (long long idx = threadIdx.x; idx < mp; idx += BT_T) {
    double v = h[idx];
    if (use_shift) {
      v = DADD(DADD(h[idx], DMUL(shift, pa[idx])), DMUL((double)(idx + 1), 1.0e-16));
      long long r = (long long)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
      while (r * (r + 1) / 2 > idx) --r;
      while ((r + 1) * (r + 2) / 2 <= idx) ++r;
      if (idx - r * (r + 1) / 2 == r) v = DSUB(v, shift);
    }
    f[idx] = v;
  }
  __syncthreads();
  for (int a = threadIdx.x; a < M.numat; a += BT_T) fock_atom(B, M, a, p, pa, f);
  __syncthreads();
}

// helect: sum_{i>j} p (h + f) + 0.5 sum_i p_ii (h_ii + f_ii), fixed order.
__device__ double cta_helect(int n, const double* p, const double* h, const double* f, double* red) {
  double s = 0.0, dsum = 0.0;
  for (int r = threadIdx.x; r < n; r += BT_T) {
    const long long base = (long long)r * (r + 1) / 2;
    double a = 0.0;
    for (int c = 0; c < r; ++c) a += p[base + c] * (h[base + c] + f[base + c]);
    s += a;
    dsum += p[base + r] * (h[base + r] + f[base + r]);
  }
  const double a = block_sum_all(s, red);
  const double b = block_sum_all(dsum, red);
  return a + 0.5 * b;
}

// cnvg (SCF/cnvg.F90:16-145) on the molecule's packed arrays; returns pl.
__device__ double cta_cnvg(int n, double* pnew, double* p, double* p1, int niter, double* red, double* scal) {
  if (threadIdx.x == 0) {
    const bool extrap = (niter % 3) != 0;
    double pl = 0.0, faca = 0.0, facb = 0.0, sum1 = 0.0;
    for (int i = 0; i < n; ++i) {
      const long long k = tri(i, i);
      const double a = pnew[k];
      sum1 = DADD(sum1, a);
      const double sa = fabs(DSUB(a, p[k]));
      if (sa > pl) pl = sa;
      if (!extrap) {
        faca = DADD(faca, DMUL(sa, sa));
        const double t = DADD(DSUB(a, DMUL(2.0, p[k])), p1[i]);
        facb = DADD(facb, DMUL(t, t));
      }
    }
    double fac = 0.0;
    if (facb > 1.0e-10 && faca < DMUL(100.0, facb)) fac = sqrt(faca / facb);
    scal[8] = fac;
    scal[9] = pl;
    scal[10] = sum1;
    for (int i = 0; i < n; ++i) {
      const long long k = tri(i, i);
      p1[i] = p[k];
      p[k] = pnew[k];
    }
  }
  __syncthreads();
  const double fac = scal[8];
  for (int r = 0; r < n; ++r) {
    const long long base = (long long)r * (r + 1) / 2;
    for (int c = threadIdx.x; c < r; c += BT_T) {
      const long long idx = base + c;
      const double a = pnew[idx];
      const double v = DADD(a, DMUL(fac, DSUB(a, p[idx])));
      p[idx] = v;
      pnew[idx] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double rhfuhf = 2.0;
    const double damp = (niter > 3) ? 0.05 : 1.0e10;
    double sum2 = 0.0;
    double* pd = red;  // n <= 128 <= BT_T
    for (int i = 0; i < n; ++i) {
      double v = p[tri(i, i)];
      const double dlt = DSUB(v, p1[i]);
      if (fabs(dlt) > damp) v = DADD(p1[i], copysign(damp, dlt));
      else v = DADD(v, DMUL(fac, dlt));
      const double t = v > 0.0 ? v : 0.0;
      v = t < rhfuhf ? t : rhfuhf;
      sum2 = DADD(sum2, v);
      pd[i] = v;
    }
    const double sum0 = scal[10];
    double sum1 = sum0;
    for (int guard = 0; guard < 1000; ++guard) {
      const double sum = sum2 > 1.0e-3 ? sum1 / sum2 : 0.0;
      sum1 = sum0;
      if (sum2 < 1.0e-3 || fabs(DSUB(sum, 1.0)) < 1.0e-5) break;
      sum2 = 0.0;
      for (int i = 0; i < n; ++i) {
        double v = DADD(DMUL(pd[i], sum), 1.0e-20);
        v = v > 0.0 ? v : 0.0;
        if (v > rhfuhf) {
          v = rhfuhf;
          sum1 = DSUB(sum1, rhfuhf);
        } else {
          sum2 = DADD(sum2, v);
        }
        pd[i] = v;
      }
    }
    for (int i = 0; i < n; ++i) {
      p[tri(i, i)] = pd[i];
      pnew[tri(i, i)] = pd[i];
    }
  }
  __syncthreads();
  return scal[9];
}

// Full diagonalisation of the molecule's F (packed, perturbed i*1e-10 in place
// as eigenvectors_LAPACK does), occupied vectors in S.Z, eigenvalues in S.eig.
__device__ void cta_diag(const Mol& M, double* f, Smem& S, double* U) {
  const int n = M.n;
  const long long mp = (long long)n * (n + 1) / 2;
  for (int i = threadIdx.x; i < n; i += BT_T) {
    const long long k = tri(i, i);
    f[k] = DADD(f[k], DMUL((double)(i + 1), 1.0e-10));
  }
  __syncthreads();
  for (long long q = threadIdx.x; q < mp; q += BT_T) S.A[q] = f[q];
  __syncthreads();
  cta_eigh(n, M.nclose, S, U);
}

__device__ void cta_density(const Mol& M, const Smem& S, double* p, double* pa) {
  const int n = M.n, nz = M.nclose;
  const long long mp = (long long)n * (n + 1) / 2;
  for (long long q = threadIdx.x; q < mp; q += BT_T) {
    long long r = (long long)((sqrt(8.0 * (double)q + 1.0) - 1.0) * 0.5);
    while (r * (r + 1) / 2 > q) --r;
    while ((r + 1) * (r + 2) / 2 <= q) ++r;
    const long long c = q - r * (r + 1) / 2;
    double s = 0.0;
    for (int m = 0; m < nz; ++m) s += S.Z[r * nz + m] * S.Z[c * nz + m];
    p[q] = 2.0 * s;
  }
  __syncthreads();
  (void)pa;
}

__global__ void __launch_bounds__(BT_T, 1) scf_batch_kernel(BatchArgs B) {
  extern __shared__ double smem[];
  __shared__ int s_m;
  const int tid = threadIdx.x;
  double* Ushared = B.scratch + (long long)blockIdx.x * 3 * BT_NMAX * BT_NMAX;
  for (;;) {
    if (tid == 0) s_m = atomicAdd(B.next, 1);
    __syncthreads();
    const int m = s_m;
    __syncthreads();
    if (m >= B.nmol) break;
    const int mi = B.order[m];
    const Mol M = B.mol[mi];
    const int n = M.n, nclose = M.nclose;
    const long long mp = (long long)n * (n + 1) / 2;
    Smem S;
    S.A = smem;
    S.Z = S.A + (BT_NMAX * (BT_NMAX + 1)) / 2;
    S.d = S.Z + BT_ZMAX;
    S.e = S.d + BT_NMAX;
    S.e2 = S.e + BT_NMAX;
    S.tau = S.e2 + BT_NMAX;
    S.pv = S.tau + BT_NMAX;
    S.v = S.pv + BT_NMAX;
    S.eig = S.v + BT_NMAX;
    S.red = S.eig + BT_NMAX + 1;
    S.scal = S.red + BT_T;
    double* f = B.f + M.hoff;
    double* p = B.p + M.hoff;
    double* pa = B.pa + M.hoff;
    double* pold = B.pold + M.hoff;
    double* pold2 = B.pold2 + M.doff;
    const double* h = B.h + M.hoff;
    // ---- first-call setup (iter.F90:123-221): diagonal guess
    const double w1 = (double)nclose / ((double)nclose + 1.0e-6 + (double)nclose);
    for (long long q = tid; q < mp; q += BT_T) { p[q] = 0.0; pa[q] = 0.0; pold[q] = 0.0; }
    __syncthreads();
    for (int i = tid; i < n; i += BT_T) {
      const long long j = tri(i, i);
      const double pd = B.pdiag[M.doff + i];
      p[j] = pd;
      pa[j] = DMUL(DMUL(pd, w1), 1.0);
      pold[j] = pa[j];
      pold2[i] = pa[j];
    }
    __syncthreads();
    // control scalars: every thread holds the same copy
    double shift = 1.0, shfmax = 20.0, pl = 1.0, ten = -80.0, shfto = 0.0, shftbo = 0.0, shiftb = 0.0;
    const double bshift = -80.0, plchek = 0.005, trans = 0.2;
    bool newdg = false, oknewd = fabs(bshift) < 0.001;
    const double selcon = fmin(fmin(B.scfcrt * 100.0, 0.1), fmax(0.0, B.scfcrt));
    const double pltest = 0.05 * sqrt(fabs(selcon));
    int iredy = 1, niter = 0;
    double eold = 1.0e2, diff = 0.0, escf = 0.0, ee = 0.0, sellim = 0.0;
    bool ready = false, converged = false;
    double eig_homo = 0.0, eig_lumo = 0.0;
    const int ihomo = nclose > 1 ? nclose : 1;
    const double enrgy = PM7_FPC9;
    for (;;) {
      ++niter;
      if (niter > B.itrmax) break;
      bool use_shift = false;
      if (fabs(shift) > 1.0e-10 && bshift != 0.0) {
        if (niter > 1) {
          if (newdg) {
            if (diff > 0.0) { shift = 1.0; if (diff > 1) newdg = false; }
            else shift = -0.1;
          } else {
            shift = (ihomo < n) ? ten + eig_lumo - eig_homo + shift : 0.0;
          }
          if (diff > 0.0) {
            if (shift > 4.0) shfmax = 4.5;
            if (shift > shfmax) shfmax = fmax(shfmax - 0.5, 0.0);
          }
          shift = fmax(-20.0, fmin(shfmax, shift));
          if (fabs(shift - shfmax) < 1.0e-5) shfmax = shfmax + 0.01;
        }
        if (pl > plchek) { shftbo = shiftb; shfto = shift; }
        else { shiftb = shftbo; shift = shfto; }
        if (ihomo < n) eig_lumo = eig_lumo + shift;
        use_shift = true;
      }
      double cur_shift = shift;
      for (;;) {  // label 320
        cta_fock(B, M, cur_shift, use_shift, f, p, pa, h);
        ee = cta_helect(n, pa, h, f, S.red) * 2.0;
        escf = (ee + M.enuclr) * enrgy + M.atheat;
        diff = escf - eold;
        if (diff > 0) ten = ten - 1.0; else ten = ten * 0.975 + 0.05;
        sellim = fmax(selcon, 1.0e-15 * fmax(fabs(ee), 1.0));
        const bool conv = niter > 4 && (pl == 0.0 || (pl < pltest && fabs(diff) < sellim)) && ready;
        if (conv) {
          if (fabs(shift) < 1.0e-10) { converged = true; break; }
          shift = 0.0;
          shiftb = 0.0;
          use_shift = false;
          cur_shift = 0.0;
          continue;
        }
        break;
      }
      if (converged) break;
      ready = iredy > 0 && (fabs(diff) < sellim * 10.0 || pl == 0.0);
      ++iredy;
      eold = escf;
      cta_diag(M, f, S, Ushared);
      eig_homo = S.eig[ihomo - 1];
      eig_lumo = ihomo < n ? S.eig[ihomo] : 0.0;
      cta_density(M, S, p, pa);
      pl = cta_cnvg(n, p, pold, pold2, niter, S.red, S.scal);
      for (long long q = tid; q < mp; q += BT_T) pa[q] = p[q] * 0.5;
      __syncthreads();
      if (!isfinite(pl)) break;
      oknewd = pl < sellim || oknewd;
      newdg = (pl < trans && oknewd) || newdg;
      if (pl < trans * 0.3333) oknewd = true;
    }
    // ---- label 600: final energy and exit diagonalisation
    ee = cta_helect(n, pa, h, f, S.red) * 2.0;
    for (long long q = tid; q < mp; q += BT_T) S.A[q] = f[q];
    __syncthreads();
    for (int i = tid; i < n; i += BT_T) S.A[tri(i, i)] = DADD(S.A[tri(i, i)], DMUL((double)(i + 1), 1.0e-10));
    __syncthreads();
    cta_eigh(n, nclose, S, Ushared);
    if (tid == 0) {
      B.escf[mi] = (ee + M.enuclr) * enrgy + M.atheat;
      B.ee[mi] = ee;
      B.niter[mi] = niter;
      B.conv[mi] = converged ? 1 : 0;
      B.homo[mi] = S.eig[ihomo - 1];
      B.lumo[mi] = ihomo < n ? S.eig[ihomo] : 0.0;
    }
    __syncthreads();
  }
}

size_t batch_smem() {
  return sizeof(double) * ((size_t)(BT_NMAX * (BT_NMAX + 1)) / 2 + BT_ZMAX + 7 * BT_NMAX + 1 + BT_T + 32);
}

}  // namespace

struct mb_batch {
  int nmol = 0;
  std::vector<Mol> hmol;
  Mol* mol = nullptr;
  int *order = nullptr, *first = nullptr, *nor = nullptr, *lim = nullptr, *cum = nullptr, *nat = nullptr, *next = nullptr,
      *niter = nullptr, *conv = nullptr, *status = nullptr;
  long long* wrow = nullptr;
  double *coord = nullptr, *h = nullptr, *w = nullptr, *pdiag = nullptr, *f = nullptr, *p = nullptr, *pa = nullptr,
         *pold = nullptr, *pold2 = nullptr, *scratch = nullptr, *escf = nullptr, *ee = nullptr, *homo = nullptr,
         *lumo = nullptr, *enuc = nullptr, *epairs = nullptr;
  long long tot_mp = 0, tot_w = 0;
  int tot_n = 0, tot_at = 0, grid = 0;
  cudaStream_t stream = nullptr;
};

static void batch_free(mb_batch* b) {
  if (!b) return;
  void* ptrs[] = {b->mol, b->order, b->first, b->nor, b->lim, b->cum, b->nat, b->next, b->niter, b->conv, b->status, b->wrow,
                  b->coord, b->h, b->w, b->pdiag, b->f, b->p, b->pa, b->pold, b->pold2, b->scratch, b->escf, b->ee,
                  b->homo, b->lumo, b->enuc, b->epairs};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
}

extern "C" int mb_batch_create(int nmol, const int* numat, const int* nat, const double* coord, mb_batch** out) {
  if (nmol <= 0 || !numat || !nat || !coord || !out) return mb_set_error(MB_ERR_ARG, "mb_batch_create: bad args");
  *out = nullptr;
  static Pm7Params P;
  static bool pinit = false;
  if (!pinit) { pm7_init(&P); pinit = true; }
  mb_batch* b = new mb_batch();
  b->nmol = nmol;
  b->hmol.resize(nmol);
  std::vector<int> first, nor, lim, cum;
  std::vector<long long> wrow;
  std::vector<double> pdiag;
  long long hoff = 0, woff = 0, maxpairs = 0;
  int aoff = 0, doff = 0;
  for (int m = 0; m < nmol; ++m) {
    Mol& M = b->hmol[m];
    const int na = numat[m];
    int ia = 0, nelec = 0, ncum = 0;
    double atheat = 0.0, eat = 0.0;
    long long wr = 0;
    std::vector<int> lm(na);
    for (int a = 0; a < na; ++a) {
      const int z = nat[aoff + a];
      if (!pm7_supported(z)) { batch_free(b); return mb_set_error(MB_ERR_UNSUPPORTED, "element outside H, C, O"); }
      const Pm7Elem& e = P.el[z];
      first.push_back(ia);
      nor.push_back(e.natorb);
      lm[a] = e.natorb == 1 ? 1 : 10;
      lim.push_back(lm[a]);
      cum.push_back(ncum);
      ncum += lm[a];
      for (int q = 0; q < e.natorb; ++q) pdiag.push_back(e.natorb == 1 ? e.tore : e.tore * 0.25);
      ia += e.natorb;
      nelec += (int)e.tore;
      atheat += e.eheat;
      eat += e.eisol;
    }
    // W: for atom a, its pair blocks with lower atoms (lim[a] x lim[b]) then its own block
    for (int a = 0; a < na; ++a) {
      wrow.push_back(wr);
      wr += (long long)lm[a] * (cum[aoff + a] + lm[a]);
    }
    if (nelec % 2 || ia > BT_NMAX || (long long)ia * (nelec / 2) > BT_ZMAX) {
      batch_free(b);
      return mb_set_error(MB_ERR_UNSUPPORTED, "batched SCF: closed shell, n <= 128 and n * nocc <= 11008 only");
    }
    M.n = ia;
    M.nclose = nelec / 2;
    M.numat = na;
    M.aoff = aoff;
    M.hoff = hoff;
    M.woff = woff;
    M.doff = doff;
    M.enuclr = 0.0;
    M.atheat = atheat - eat * PM7_FPC9;
    hoff += (long long)ia * (ia + 1) / 2;
    woff += wr;
    doff += ia;
    aoff += na;
    maxpairs = std::max<long long>(maxpairs, (long long)na * (na - 1) / 2);
  }
  b->tot_mp = hoff;
  b->tot_w = woff;
  b->tot_n = doff;
  b->tot_at = aoff;
  cudaError_t e = cudaSuccess;
#define BALLOC(ptr, bytes) if (e == cudaSuccess) e = cudaMalloc((void**)&(ptr), (bytes))
  BALLOC(b->mol, sizeof(Mol) * nmol);
  BALLOC(b->order, sizeof(int) * nmol);
  BALLOC(b->first, sizeof(int) * aoff);
  BALLOC(b->nor, sizeof(int) * aoff);
  BALLOC(b->lim, sizeof(int) * aoff);
  BALLOC(b->cum, sizeof(int) * aoff);
  BALLOC(b->wrow, sizeof(long long) * aoff);
  BALLOC(b->nat, sizeof(int) * aoff);
  BALLOC(b->coord, sizeof(double) * 3 * aoff);
  BALLOC(b->h, sizeof(double) * hoff);
  BALLOC(b->w, sizeof(double) * woff);
  BALLOC(b->pdiag, sizeof(double) * doff);
  BALLOC(b->f, sizeof(double) * hoff);
  BALLOC(b->p, sizeof(double) * hoff);
  BALLOC(b->pa, sizeof(double) * hoff);
  BALLOC(b->pold, sizeof(double) * hoff);
  BALLOC(b->pold2, sizeof(double) * doff);
  BALLOC(b->escf, sizeof(double) * nmol);
  BALLOC(b->ee, sizeof(double) * nmol);
  BALLOC(b->homo, sizeof(double) * nmol);
  BALLOC(b->lumo, sizeof(double) * nmol);
  BALLOC(b->enuc, sizeof(double) * nmol);
  BALLOC(b->niter, sizeof(int) * nmol);
  BALLOC(b->conv, sizeof(int) * nmol);
  BALLOC(b->next, sizeof(int));
  BALLOC(b->status, sizeof(int));
  BALLOC(b->epairs, sizeof(double) * (maxpairs + 1));
#undef BALLOC
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMemcpy(b->first, first.data(), sizeof(int) * aoff, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->nor, nor.data(), sizeof(int) * aoff, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->lim, lim.data(), sizeof(int) * aoff, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->cum, cum.data(), sizeof(int) * aoff, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->wrow, wrow.data(), sizeof(long long) * aoff, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->nat, nat, sizeof(int) * aoff, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->coord, coord, sizeof(double) * 3 * aoff, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->pdiag, pdiag.data(), sizeof(double) * doff, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    int r = mb_set_cuda_error(e, "mb_batch_create", __FILE__, __LINE__);
    batch_free(b);
    return r;
  }
  // integrals per molecule on the GPU (hcore), then E_nuc
  for (int m = 0; m < nmol; ++m) {
    const Mol& M = b->hmol[m];
    MbAtomsDev at;
    at.numat = M.numat;
    at.first = b->first + M.aoff;
    at.nor = b->nor + M.aoff;
    at.lim = b->lim + M.aoff;
    at.wrow = b->wrow + M.aoff;
    at.cum = b->cum + M.aoff;
    int rc = mb_hcore_dev(b->nat + M.aoff, b->coord + 3 * M.aoff, &at, M.numat, b->h + M.hoff, b->w + M.woff,
                          b->epairs, b->stream);
    if (rc == MB_OK)
      rc = mb_hcore_finish(M.numat, &at, b->nat + M.aoff, b->h + M.hoff, nullptr, b->enuc + m, b->epairs, b->stream);
    if (rc != MB_OK) { batch_free(b); return rc; }
  }
  std::vector<double> en(nmol);
  e = cudaMemcpyAsync(en.data(), b->enuc, sizeof(double) * nmol, cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  if (e != cudaSuccess) {
    int r = mb_set_cuda_error(e, "mb_batch_create integrals", __FILE__, __LINE__);
    batch_free(b);
    return r;
  }
  for (int m = 0; m < nmol; ++m) b->hmol[m].enuclr = en[m];
  // molecules largest first, so the last wave is not a long one
  std::vector<int> order(nmol);
  for (int m = 0; m < nmol; ++m) order[m] = m;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->hmol[x].n > b->hmol[y].n; });
  e = cudaMemcpy(b->mol, b->hmol.data(), sizeof(Mol) * nmol, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(b->order, order.data(), sizeof(int) * nmol, cudaMemcpyHostToDevice);
  int dev = 0, sms = 0, per = 0;
  const size_t smem = batch_smem();
  if (e == cudaSuccess) e = cudaFuncSetAttribute(scf_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, scf_batch_kernel, BT_T, smem);
  if (e != cudaSuccess || per < 1) {
    int r = e != cudaSuccess ? mb_set_cuda_error(e, "mb_batch_create kernel setup", __FILE__, __LINE__)
                             : mb_set_error(MB_ERR_CUDA, "batched SCF kernel does not fit on an SM");
    batch_free(b);
    return r;
  }
  b->grid = std::min(nmol, sms * per);
  e = cudaMalloc((void**)&b->scratch, sizeof(double) * 3 * BT_NMAX * BT_NMAX * (size_t)b->grid);
  if (e != cudaSuccess) {
    int r = mb_set_cuda_error(e, "mb_batch_create scratch", __FILE__, __LINE__);
    batch_free(b);
    return r;
  }
  *out = b;
  return MB_OK;
}

extern "C" int mb_batch_destroy(mb_batch* b) {
  if (b) {
    cudaStreamSynchronize(b->stream);
    batch_free(b);
  }
  return MB_OK;
}

extern "C" int mb_batch_nmol(const mb_batch* b) { return b ? b->nmol : 0; }

extern "C" int mb_batch_run(mb_batch* b, const mb_scf_opts* opts_in, double* escf, int* niter, int* converged,
                            double* t_ms) {
  if (!b) return mb_set_error(MB_ERR_ARG, "mb_batch_run: null batch");
  mb_scf_opts o;
  if (opts_in) o = *opts_in; else mb_scf_opts_default(&o);
  BatchArgs A;
  A.mol = b->mol;
  A.order = b->order;
  A.nmol = b->nmol;
  A.first = b->first;
  A.nor = b->nor;
  A.h = b->h;
  A.w = b->w;
  A.wrow = b->wrow;
  A.lim = b->lim;
  A.cum = b->cum;
  A.pdiag = b->pdiag;
  A.f = b->f;
  A.p = b->p;
  A.pa = b->pa;
  A.pold = b->pold;
  A.pold2 = b->pold2;
  A.scratch = b->scratch;
  A.escf = b->escf;
  A.ee = b->ee;
  A.niter = b->niter;
  A.conv = b->conv;
  A.homo = b->homo;
  A.lumo = b->lumo;
  A.next = b->next;
  A.status = b->status;
  A.itrmax = o.itrmax;
  A.scfcrt = o.scfcrt;
  cudaEvent_t e0, e1;
  MB_CUDA(cudaEventCreate(&e0));
  MB_CUDA(cudaEventCreate(&e1));
  MB_CUDA(cudaMemsetAsync(b->next, 0, sizeof(int), b->stream));
  MB_CUDA(cudaEventRecord(e0, b->stream));
  scf_batch_kernel<<<b->grid, BT_T, batch_smem(), b->stream>>>(A);
  MB_LAUNCH_CHECK();
  MB_CUDA(cudaEventRecord(e1, b->stream));
  MB_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  MB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (t_ms) *t_ms = ms;
  if (escf) MB_CUDA(cudaMemcpy(escf, b->escf, sizeof(double) * b->nmol, cudaMemcpyDeviceToHost));
  if (niter) MB_CUDA(cudaMemcpy(niter, b->niter, sizeof(int) * b->nmol, cudaMemcpyDeviceToHost));
  if (converged) MB_CUDA(cudaMemcpy(converged, b->conv, sizeof(int) * b->nmol, cudaMemcpyDeviceToHost));
  return MB_OK;
}

extern "C" int mb_batch_get_density(mb_batch* b, int m, double* p) {
  if (!b || m < 0 || m >= b->nmol || !p) return mb_set_error(MB_ERR_ARG, "mb_batch_get_density: bad args");
  const Mol& M = b->hmol[m];
  MB_CUDA(cudaMemcpy(p, b->p + M.hoff, sizeof(double) * (size_t)M.n * (M.n + 1) / 2, cudaMemcpyDeviceToHost));
  return MB_OK;
}

extern "C" int mb_batch_get_hw(mb_batch* b, int m, double* h, double* w, double* enuclr) {
  if (!b || m < 0 || m >= b->nmol) return mb_set_error(MB_ERR_ARG, "mb_batch_get_hw: bad args");
  const Mol& M = b->hmol[m];
  const long long wlen = (m + 1 < b->nmol ? b->hmol[m + 1].woff : b->tot_w) - M.woff;
  if (h) MB_CUDA(cudaMemcpy(h, b->h + M.hoff, sizeof(double) * (size_t)M.n * (M.n + 1) / 2, cudaMemcpyDeviceToHost));
  if (w) MB_CUDA(cudaMemcpy(w, b->w + M.woff, sizeof(double) * (size_t)wlen, cudaMemcpyDeviceToHost));
  if (enuclr) *enuclr = M.enuclr;
  return MB_OK;
}
