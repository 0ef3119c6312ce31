// Two- and one-centre Fock build for the dense NDDO SCF (sp basis).
//
// Replaces fock2 (SCF/fock2.F90:16-374, sp branches :149-298), jab
// (integrals/jab.F90), kab (integrals/kab.F90) and fock1 (SCF/fock1.F90) as
// called from iter (SCF/iter.F90:553), including iter's level-shifted start
// value F = H + shift*PA + 1e-16*i, F_ii -= shift (SCF/iter.F90:317-324).
//
// Result is bit-identical to the reference loop order: every element of F
// receives its contributions in the same sequence (partner atoms in ascending
// order with the one-centre term at the atom's own position), each
// contribution is formed with the same term order, and no FMA is used.
//
// Design: one CTA per atom A owns A's diagonal block.  Its threads walk all
// partner atoms B in chunks: each thread evaluates one pair (A,B) -- the
// Coulomb contribution to A's diagonal block into shared memory and, for
// B < A, the complete exchange block F(A,B) straight to global memory.  Then
// up to ten owner threads fold the chunk's contributions into their running
// sums in partner order.  Every W block is read twice (once by each of its
// atoms' CTAs); all other traffic is one pass over P, PA, H and F.
#include "mb_common.cuh"

namespace {

constexpr int kChunk = 128;

__constant__ int c_pidx[16] = {1, 2, 4, 7, 2, 3, 5, 8, 4, 5, 6, 9, 7, 8, 9, 10};

__device__ __forceinline__ int pair1(int a, int b) {  // 1-based pair index of orbitals a, b (1..4)
  return a > b ? a * (a - 1) / 2 + b : b * (b - 1) / 2 + a;
}

struct FockArgs {
  MbAtoms at;
  double* f;
  const double* h;
  const double* ptot;
  const double* pa;
  const double* w;
  double shift;
  int use_shift;
};

__device__ __forceinline__ double f_start(const FockArgs& a, long long idx, bool diag) {
  if (!a.use_shift) return a.h[idx];
  double v = DADD(DADD(a.h[idx], DMUL(a.shift, a.pa[idx])), DMUL((double)(idx + 1), 1.0e-16));
  if (diag) v = DSUB(v, a.shift);
  return v;
}

__global__ void __launch_bounds__(kChunk) fock2_kernel(FockArgs a) {
  const int A = blockIdx.x;
  const int tid = threadIdx.x;
  const int numat = a.at.numat;
  const int fA = a.at.first[A], nA = a.at.nor[A], lA = a.at.lim[A];
  const long long wrowA = a.at.wrow[A];

  __shared__ double s_c[kChunk][11];  // per-partner contributions (10 + second add)
  __shared__ unsigned char s_two[kChunk];

  // Owner thread e < lA keeps the running value of A's diagonal-block element e.
  double run = 0.0, f1 = 0.0;
  long long own_idx = 0;
  if (tid < lA) {
    int iw = 1, jw = 1;  // local (row, col), 1-based, from packed element tid
    {
      int e = tid, r = 1;
      while (e >= r) { e -= r; ++r; }
      iw = r; jw = e + 1;
    }
    own_idx = mb_tri(fA + iw - 1, fA + jw - 1);
    run = f_start(a, own_idx, iw == jw);
    // fock1 (SCF/fock1.F90): one-centre Coulomb and exchange for element (iw, jw)
    const double* w1 = a.w + wrowA + (long long)lA * a.at.cum[A];
    const int ilim = lA;
    const int ijw = iw * (iw - 1) / 2 + jw;
    double sum = 0.0;
    for (int kw = 1; kw <= nA; ++kw)
      for (int lw = 1; lw <= nA; ++lw) {
        int ip = kw > lw ? kw : lw, jp = kw < lw ? kw : lw;
        long long ijp = mb_tri(fA + ip - 1, fA + jp - 1);
        int klw = ip * (ip - 1) / 2 + jp;
        int im = kw > jw ? kw : jw, jm = kw < jw ? kw : jw;
        int ikw = im * (im - 1) / 2 + jm;
        im = lw > iw ? lw : iw; jm = lw < iw ? lw : iw;
        int jlw = im * (im - 1) / 2 + jm;
        sum = DSUB(DADD(sum, DMUL(a.ptot[ijp], w1[(ijw - 1) + ilim * (klw - 1)])),
                   DMUL(a.pa[ijp], w1[(ikw - 1) + ilim * (jlw - 1)]));
      }
    f1 = sum;
  }

  for (int q0 = 0; q0 < numat; q0 += kChunk) {
    const int B = q0 + tid;
    if (B < numat && B != A) {
      const int fB = a.at.first[B], nB = a.at.nor[B], lB = a.at.lim[B];
      double* c = s_c[tid];
      s_two[tid] = 0;
      if (B < A) {
        // pair (ii = A, jj = B); W block is lA x lB with B's pair index fastest
        const double* wk = a.w + wrowA + (long long)lA * a.at.cum[B];
        if (nA == 4 && nB == 4) {
          double pjb[16];
#pragma unroll
          for (int x = 0; x < 4; ++x)
#pragma unroll
            for (int y = 0; y < 4; ++y) {
              int r = fB + (x > y ? x : y), cc = fB + (x < y ? x : y);
              pjb[x * 4 + y] = a.ptot[mb_tri(r, cc)];
            }
#pragma unroll
          for (int q = 0; q < 10; ++q) {
            double sb = DMUL(pjb[0], wk[q * 10 + c_pidx[0] - 1]);
#pragma unroll
            for (int m = 1; m < 16; ++m) sb = DADD(sb, DMUL(pjb[m], wk[q * 10 + c_pidx[m] - 1]));
            c[q] = sb;
          }
          // kab exchange on the off-diagonal block (A rows, B columns)
          double pk[16];
#pragma unroll
          for (int x = 0; x < 4; ++x)
#pragma unroll
            for (int y = 0; y < 4; ++y) pk[x * 4 + y] = a.pa[mb_tri(fA + x, fB + y)];
#pragma unroll
          for (int mu = 1; mu <= 4; ++mu)
#pragma unroll
            for (int nu = 1; nu <= 4; ++nu) {
              double s = 0.0;
#pragma unroll
              for (int lam = 1; lam <= 4; ++lam)
#pragma unroll
                for (int sig = 1; sig <= 4; ++sig) {
                  double t = DMUL(pk[(lam - 1) * 4 + sig - 1],
                                  wk[(pair1(mu, lam) - 1) * 10 + pair1(nu, sig) - 1]);
                  s = (lam == 1 && sig == 1) ? t : DADD(s, t);
                }
              long long idx = mb_tri(fA + mu - 1, fB + nu - 1);
              a.f[idx] = DSUB(f_start(a, idx, false), s);
            }
        } else if (nA == 4 && nB == 1) {
          const double pb = a.ptot[mb_tri(fB, fB)];
#pragma unroll
          for (int q = 0; q < 10; ++q) c[q] = DMUL(pb, wk[q]);
#pragma unroll
          for (int i = 1; i <= 4; ++i) {
            double sum = 0.0;
#pragma unroll
            for (int j = 1; j <= 4; ++j) sum = DADD(sum, DMUL(a.pa[mb_tri(fA + j - 1, fB)], wk[pair1(i, j) - 1]));
            long long idx = mb_tri(fA + i - 1, fB);
            a.f[idx] = DSUB(f_start(a, idx, false), sum);
          }
        } else if (nA == 1 && nB == 4) {
          double sumoff = 0.0, sumdia = 0.0;
          int k = 0;
#pragma unroll
          for (int i = 0; i <= 3; ++i) {
            for (int j = 1; j <= i; ++j)
              sumoff = DADD(sumoff, DMUL(a.ptot[mb_tri(fB + i, fB + j - 1)], wk[j + k - 1]));
            k += i + 1;
            sumdia = DADD(sumdia, DMUL(a.ptot[mb_tri(fB + i, fB + i)], wk[k - 1]));
          }
          c[0] = DMUL(sumoff, 2.0);
          c[1] = sumdia;
          s_two[tid] = 1;
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            double sum = 0.0;
#pragma unroll
            for (int l = 1; l <= 4; ++l) sum = DADD(sum, DMUL(a.pa[mb_tri(fA, fB + l - 1)], wk[pair1(i + 1, l) - 1]));
            long long idx = mb_tri(fA, fB + i);
            a.f[idx] = DSUB(f_start(a, idx, false), sum);
          }
        } else {
          c[0] = DMUL(a.ptot[mb_tri(fB, fB)], wk[0]);
          long long idx = mb_tri(fA, fB);
          a.f[idx] = DSUB(f_start(a, idx, false), DMUL(a.pa[idx], wk[0]));
        }
      } else {
        // pair (ii = B, jj = A); W block is lB x lA with A's pair index fastest
        const double* wk = a.w + a.at.wrow[B] + (long long)lB * a.at.cum[A];
        if (nA == 4 && nB == 4) {
          double pja[16];
#pragma unroll
          for (int x = 0; x < 4; ++x)
#pragma unroll
            for (int y = 0; y < 4; ++y) {
              int r = fB + (x > y ? x : y), cc = fB + (x < y ? x : y);
              pja[x * 4 + y] = a.ptot[mb_tri(r, cc)];
            }
#pragma unroll
          for (int q = 0; q < 10; ++q) {
            double sa = DMUL(pja[0], wk[(c_pidx[0] - 1) * 10 + q]);
#pragma unroll
            for (int m = 1; m < 16; ++m) sa = DADD(sa, DMUL(pja[m], wk[(c_pidx[m] - 1) * 10 + q]));
            c[q] = sa;
          }
        } else if (nA == 4 && nB == 1) {
          // reference branch "jb - ja >= 3 .and. ia == ib": B light (ii), A heavy (jj)
          const double pb = a.ptot[mb_tri(fB, fB)];
#pragma unroll
          for (int q = 0; q < 10; ++q) c[q] = DMUL(pb, wk[q]);
        } else if (nA == 1 && nB == 4) {
          // reference branch "ib - ia >= 3 .and. ja == jb": B heavy (ii), A light (jj)
          double sumoff = 0.0, sumdia = 0.0;
          int k = 0;
#pragma unroll
          for (int i = 0; i <= 3; ++i) {
            for (int j = 1; j <= i; ++j)
              sumoff = DADD(sumoff, DMUL(a.ptot[mb_tri(fB + i, fB + j - 1)], wk[j + k - 1]));
            k += i + 1;
            sumdia = DADD(sumdia, DMUL(a.ptot[mb_tri(fB + i, fB + i)], wk[k - 1]));
          }
          c[0] = DMUL(sumoff, 2.0);
          c[1] = sumdia;
          s_two[tid] = 1;
        } else {
          c[0] = DMUL(a.ptot[mb_tri(fB, fB)], wk[0]);
        }
      }
    }
    __syncthreads();
    if (tid < lA) {
      const int nq = min(kChunk, numat - q0);
      for (int t = 0; t < nq; ++t) {
        const int Bq = q0 + t;
        if (Bq == A) {
          run = DADD(run, f1);
        } else {
          run = DADD(run, s_c[t][tid]);
          if (s_two[t]) run = DADD(run, s_c[t][1]);
        }
      }
    }
    __syncthreads();
  }
  if (tid < lA) a.f[own_idx] = run;
}

}  // namespace

extern "C" int mb_fock2_dev(const MbAtomsDev* atoms, double* f, const double* h, const double* ptot,
                            const double* pa, const double* w, double shift, int use_shift,
                            cudaStream_t stream) {
  if (!atoms || atoms->numat <= 0) return mb_set_error(MB_ERR_ARG, "mb_fock2_dev: no atoms");
  FockArgs a;
  a.at.numat = atoms->numat;
  a.at.first = atoms->first;
  a.at.nor = atoms->nor;
  a.at.lim = atoms->lim;
  a.at.wrow = atoms->wrow;
  a.at.cum = atoms->cum;
  a.f = f;
  a.h = h;
  a.ptot = ptot;
  a.pa = pa;
  a.w = w;
  a.shift = shift;
  a.use_shift = use_shift;
  mb_kstat_mark(MB_KSTAT_FOCK, stream, true);
  fock2_kernel<<<atoms->numat, kChunk, 0, stream>>>(a);
  mb_kstat_mark(MB_KSTAT_FOCK, stream, false);
  MB_LAUNCH_CHECK();
  return MB_OK;
}
