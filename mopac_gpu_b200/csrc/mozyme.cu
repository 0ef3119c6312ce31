// MOZYME localized-MO path: sparse pair-block storage and the kernels on it.
//
// Storage (MOZYME/fillij.F90:20-230, first call, molecular): for atom i in
// order, the blocks of partners j < i with r^2 < cutof2 (iorbs(i) x
// iorbs(j), atom i's orbitals outer), then atom i's own lower triangle.  The
// device layout keeps it as per-atom pair lists: pair entries of atom i are
// its partners in ascending j followed by the diagonal entry (j = i), each
// with its block offset -- the same offsets the reference's nijbo holds.
//
// LMOs (MOZYME_C: ncf, nncf, icocc, ncocc, cocc) are uploaded as given plus an
// inverted index: for every atom, the LMOs that contain it in ascending LMO
// order with the offset of that atom's coefficients in cocc.
//
// density_for_MOZYME (MOZYME/density_for_MOZYME.F90:16-342) is scattered
// LMO by LMO in the reference; here each stored block gathers its LMOs by a
// merge of the two atoms' LMO lists in ascending LMO order, so every element
// sees the same additions in the same order as the reference's loop and the
// result is bit-identical, without atomics.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "mb_common.cuh"
#include "pm7_params.h"

namespace {

__device__ __forceinline__ int pair_elems(int io, int jo, bool diag) { return diag ? io * (io + 1) / 2 : io * jo; }

// Adds the contributions of the LMOs matched in this chunk (bit m of mask:
// lane m holds the match's coefficient offsets on atom i, my_ca, and on atom
// j, my_cb), in lane order, to this lane's element (j1, k1).  Eight matches'
// coefficients are loaded before their products are added, so the loads
// overlap; the additions keep the reference's order.
__device__ __forceinline__ void mz_density_add(unsigned mask, int my_ca, int my_cb, bool act, int j1, int k1,
                                               const double* __restrict__ cocc, double& acc) {
  while (mask) {  // warp-uniform
    double va[8], vb[8];
    bool hv[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      hv[q] = mask != 0;
      const int src = hv[q] ? __ffs(mask) - 1 : 0;
      if (hv[q]) mask &= mask - 1;
      const int ca = __shfl_sync(0xffffffffu, my_ca, src), cb = __shfl_sync(0xffffffffu, my_cb, src);
      va[q] = (hv[q] && act) ? __ldg(cocc + ca + j1) : 0.0;
      vb[q] = (hv[q] && act) ? __ldg(cocc + cb + k1) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q)
      if (hv[q] && act) acc = DADD(acc, DMUL(vb[q], va[q]));
  }
}

// One warp per stored block (grid-stride over pair entries).  The block's
// element (j1, k1) sums c(LMO, j1 on atom i) c(LMO, k1 on atom j) over the
// LMOs on both atoms in ascending LMO order (density_for_MOZYME.F90's order):
// the shorter of the two atoms' ascending LMO lists is taken 32 entries at a
// time, one per lane, each searched in the longer list, and the matches of
// the chunk are added in order.
__global__ void __launch_bounds__(256) mz_density_kernel(MbMzLayout L, MbMzLmos Q, int mode, const double* __restrict__ partp,
                                                        double* __restrict__ p, double spinfa, int scale) {
  const int lane = threadIdx.x & 31;
  const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long e = warp0; e < L.npairs; e += nw) {
    const int i = L.pair_i[e], j = L.pair_j[e];
    const bool diag = (i == j);
    const int io = L.iorbs[i], jo = L.iorbs[j];
    const int ne = pair_elems(io, jo, diag);
    const long long off = L.pair_off[e];
    int j1 = 0, k1 = 0;
    if (diag) {
      // lower triangle, row j1 outer: element index lane = j1 (j1 + 1) / 2 + k1
      while ((j1 + 1) * (j1 + 2) / 2 <= lane) ++j1;
      k1 = lane - j1 * (j1 + 1) / 2;
    } else if (jo > 0) {
      j1 = lane / jo;
      k1 = lane - j1 * jo;
    }
    const bool act = lane < ne;
    double acc = 0.0;
    if (act) {
      if (mode == -1) acc = DMUL(-0.5, partp[off + lane]);
      else if (mode != 0) acc = DMUL(0.5, partp[off + lane]);
    }
    const int a0 = Q.atom_ptr[i], ae = Q.atom_ptr[i + 1];
    if (diag) {
      // every LMO on the atom meets itself
      for (int base = a0; base < ae; base += 32) {
        const int idx = base + lane;
        const int c = idx < ae ? Q.atom_coff[idx] : 0;
        const unsigned mask = __ballot_sync(0xffffffffu, idx < ae);
        mz_density_add(mask, c, c, act, j1, k1, Q.cocc, acc);
      }
    } else {
      const int b0 = Q.atom_ptr[j], be = Q.atom_ptr[j + 1];
      const bool short_i = (ae - a0) <= (be - b0);  // walk atom i's list, search atom j's
      const int s0 = short_i ? a0 : b0, se = short_i ? ae : be;
      int lo = short_i ? b0 : a0;
      const int le = short_i ? be : ae;
      for (int base = s0; base < se && lo < le; base += 32) {
        const int idx = base + lane;
        const int x = idx < se ? __ldg(Q.atom_lmo + idx) : 0x7fffffff;
        int lb = lo, ub = le;  // first entry >= x in the longer list
        while (lb < ub) {
          const int mid = (lb + ub) >> 1;
          if (__ldg(Q.atom_lmo + mid) < x) lb = mid + 1;
          else ub = mid;
        }
        const bool hit = idx < se && lb < le && __ldg(Q.atom_lmo + lb) == x;
        int my_ca = 0, my_cb = 0;
        if (hit) {
          const int cs = Q.atom_coff[idx], cl = Q.atom_coff[lb];
          my_ca = short_i ? cs : cl;
          my_cb = short_i ? cl : cs;
        }
        const unsigned mask = __ballot_sync(0xffffffffu, hit);
        lo = __shfl_sync(0xffffffffu, lb, 31);  // the chunk's largest entry bounds the next search
        mz_density_add(mask, my_ca, my_cb, act, j1, k1, Q.cocc, acc);
      }
    }
    if (act) p[off + lane] = scale ? DMUL(spinfa, acc) : acc;
  }
}

// Partial sums of p(h + f) over all elements and over the diagonal ones.
__global__ void __launch_bounds__(256) mz_helecz_partials(long long mpack, int norbs, const long long* __restrict__ idiag,
                                                         const double* __restrict__ p, const double* __restrict__ h,
                                                         const double* __restrict__ f, double* __restrict__ part) {
  __shared__ double sa[256], sd[256];
  double s = 0.0, d = 0.0;
  for (long long m = blockIdx.x * (long long)blockDim.x + threadIdx.x; m < mpack; m += (long long)gridDim.x * blockDim.x)
    s += p[m] * (h[m] + f[m]);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < norbs; q += (long long)gridDim.x * blockDim.x) {
    const long long m = idiag[q] - 1;
    d += p[m] * (h[m] + f[m]);
  }
  sa[threadIdx.x] = s;
  sd[threadIdx.x] = d;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      sa[threadIdx.x] += sa[threadIdx.x + w];
      sd[threadIdx.x] += sd[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = sa[0];
    part[2 * blockIdx.x + 1] = sd[0];
  }
}

// ee = (sum_all - sum_diag) + 0.5 sum_diag, the blocks' weights in helecz.
__global__ void mz_helecz_final(int nblocks, const double* __restrict__ part, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0, d = 0.0;
    for (int b = 0; b < nblocks; ++b) {
      s += part[2 * b];
      d += part[2 * b + 1];
    }
    *out = (s - d) + 0.5 * d;
  }
}

// cnvgz (MOZYME/cnvgz.F90:16-85), step 1: gather the diagonals, max|pnew - p|.
__global__ void __launch_bounds__(256) mz_cnvgz_gather(int norbs, long long mpack, const long long* __restrict__ idiag,
                                                      const double* __restrict__ pnew, const double* __restrict__ p,
                                                      double* __restrict__ p2, double* __restrict__ p3,
                                                      unsigned long long* __restrict__ pmax_bits) {
  __shared__ double sm[256];
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < norbs; q += (long long)gridDim.x * blockDim.x) {
    const long long j = idiag[q] - 1;
    p3[q] = pnew[j];
    p2[q] = p[j];
  }
  double m = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < mpack; i += (long long)gridDim.x * blockDim.x)
    m = fmax(m, fabs(DSUB(pnew[i], p[i])));
  sm[threadIdx.x] = m;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + w]);
    __syncthreads();
  }
  // non-negative doubles order like their bit patterns
  if (threadIdx.x == 0) atomicMax(pmax_bits, (unsigned long long)__double_as_longlong(sm[0]));
}

// Step 2 (one thread, reference order): faca, facb and the extrapolation factor.
__global__ void mz_cnvgz_factor(int norbs, int niter, int use3, const double* __restrict__ p1,
                                const double* __restrict__ p2, const double* __restrict__ p3, double* __restrict__ fac) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double f = 0.0;  // 0: no extrapolation
  if (use3 && niter % 3 == 0) {
    double faca = 0.0, facb = 0.0;
    for (int i = 0; i < norbs; ++i) {
      const double sa = fabs(DSUB(p3[i], p2[i]));
      faca = DADD(faca, DMUL(sa, sa));
      const double t = DADD(DSUB(p3[i], DMUL(2.0, p2[i])), p1[i]);
      facb = DADD(facb, DMUL(t, t));
    }
    if (facb > 0.0 && faca < DMUL(100.0, facb)) f = sqrt(faca / facb);
  }
  *fac = f;
}

// Step 3: pnew = pnew + fac (pnew - p) where a factor was found; then p = pnew
// is done after damping.
__global__ void __launch_bounds__(256) mz_cnvgz_extrap(long long mpack, const double* __restrict__ fac,
                                                      double* __restrict__ pnew, const double* __restrict__ p) {
  const double f = *fac;
  if (f == 0.0) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < mpack; i += (long long)gridDim.x * blockDim.x)
    pnew[i] = DADD(pnew[i], DMUL(f, DSUB(pnew[i], p[i])));
}

// Step 4: damping of the diagonal (niter > 3, pmax > 0.05) and p1 = p2.
__global__ void __launch_bounds__(256) mz_cnvgz_damp(int norbs, int niter, int use3, const long long* __restrict__ idiag,
                                                    const unsigned long long* __restrict__ pmax_bits,
                                                    double* __restrict__ pnew, double* __restrict__ p1,
                                                    const double* __restrict__ p2, const double* __restrict__ p3) {
  const double damp = 0.05;
  const double pmax = __longlong_as_double((long long)*pmax_bits);
  const bool on = use3 && niter > 3 && pmax > damp;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < norbs; q += (long long)gridDim.x * blockDim.x) {
    if (on) {
      const double dlt = DSUB(p3[q], p2[q]);
      if (fabs(dlt) > damp) {
        const long long j = idiag[q] - 1;
        double v = DADD(p2[q], copysign(damp, dlt));
        v = fmax(v, 0.0);
        pnew[j] = fmin(2.0, v);
      }
    }
    p1[q] = p2[q];
  }
}

__global__ void __launch_bounds__(256) copy_kernel(long long n, const double* __restrict__ src, double* __restrict__ dst) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

// ------------------------------------------------------------- fock2z
constexpr double MZ_EV = 27.211386245988;
constexpr double MZ_A0 = 0.529177210903;

// The element parameters of fock2z's far-pair terms inside PM7's 7 A
// feathering radius (am, ad, dd by atomic number), for cutoffs below 7 A.
struct MzFar {
  double am[9], ad[9], dd[9];
};
__constant__ MzFar c_far;

int far_params_init() {
  static std::mutex mu;
  static bool done = false;
  std::lock_guard<std::mutex> lk(mu);
  if (done) return MB_OK;
  Pm7Params P;
  pm7_init(&P);
  MzFar h;
  for (int z = 0; z < 9; ++z) {
    h.am[z] = P.el[z].am;
    h.ad[z] = P.el[z].ad;
    h.dd[z] = P.el[z].dd;
  }
  MB_CUDA(cudaMemcpyToSymbol(c_far, &h, sizeof(h)));
  done = true;
  return MB_OK;
}

// to_point (integrals/mndod.F90:3462-3486) with trunc_1 = 7, trunc_2 = 0.22:
// the point-charge repulsion and the NDDO weight.
__device__ __forceinline__ double mz_feather(double r, double* point) {
  *point = DMUL(MZ_EV, MZ_A0) / r;
  return r < 7.0 ? 1.0 - exp(-(r - 7.0) * (r - 7.0) * 0.22) : 0.0;
}
__constant__ int c_pidx[16] = {1, 2, 4, 7, 2, 3, 5, 8, 4, 5, 6, 9, 7, 8, 9, 10};

__device__ __forceinline__ int tri1(int i, int j) {  // 1-based packed index of (i, j)
  const int a = i > j ? i : j, b = i < j ? i : j;
  return (a * (a - 1)) / 2 + b;
}

// qe(a): electrons on each atom, chrge_for_MOZYME (MOZYME/chrge_for_MOZYME.F90).
__global__ void mz_chrge(MbMzLayout L, const double* __restrict__ p, double* __restrict__ qe) {
  for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < L.numat; a += gridDim.x * blockDim.x) {
    long long ii = L.pair_off[L.pair_ptr[a + 1] - 1];
    double sum = 0.0;
    for (int j = 1; j <= L.iorbs[a]; ++j) {
      ii += j;
      sum = DADD(sum, p[ii - 1]);
    }
    qe[a] = sum;
  }
}

// Contribution of stored partner b to element t (0-based triangle position) of
// atom a's diagonal block, as fz2n adds it during pair (max(a,b), min(a,b)).
// A light atom with a heavy partner receives two additions in a row,
// f = (f + sumoff * 2) + sumdia, as Fortran evaluates the statement; the
// second one comes back in *second (and true).
__device__ double mz_pair_diag_term(int a, int b, int t, const MbMzLayout& L, const double* __restrict__ wk,
                                    const double* __restrict__ p, double* second, bool* has_second) {
  *has_second = false;
  const int ia = L.iorbs[a], ib = L.iorbs[b];
  const long long db = L.pair_off[L.pair_ptr[b + 1] - 1];
  if (ia >= 3 && ib >= 3) {
    // jab: the higher atom gets sumb (the lower atom's density), the lower one suma
    int i5 = 1;
    while ((i5 * (i5 + 1)) / 2 <= t) ++i5;  // row of triangle position t (0-based t)
    const int i6 = t - (i5 * (i5 - 1)) / 2 + 1;
    const int i = (i5 * (i5 - 1)) / 2 + i6 - 1;  // running index of jab's output loop = t
    double s = 0.0;
    for (int j = 0; j < 16; ++j) {
      const int jr = j / 4 + 1, jc = j % 4 + 1;
      const double pb = p[db + tri1(jr, jc) - 1];
      const double wv = (a > b) ? wk[i * 10 + c_pidx[j] - 1] : wk[(c_pidx[j] - 1) * 10 + i];
      s = DADD(s, DMUL(pb, wv));
    }
    return s;
  }
  if (ia >= 3) {  // a heavy, b light: a's element t gets ptot(b) w(t+1)
    return DMUL(p[db], wk[t]);
  }
  if (ib >= 3) {  // a light, b heavy: sumoff * 2 + sumdia over b's triangle
    double sumoff = 0.0, sumdia = 0.0;
    int k = 0;
    for (int i = 1; i <= 4; ++i) {
      for (int j = 1; j <= i - 1; ++j) {
        ++k;
        sumoff = DADD(sumoff, DMUL(p[db + tri1(i, j) - 1], wk[k - 1]));
      }
      ++k;
      sumdia = DADD(sumdia, DMUL(p[db + tri1(i, i) - 1], wk[k - 1]));
    }
    *second = sumdia;
    *has_second = true;
    return DMUL(sumoff, 2.0);
  }
  return DMUL(p[db], wk[0]);  // light-light
}

// Diagonal blocks: one warp per atom.  Lanes evaluate 32 partners at a time
// (stored pairs: their integral terms; the others: qe(b) ev a0 / r on the s
// and p diagonal), then lane t folds element t over the 32 partners in
// ascending order -- the order in which fz2n's pair loop reaches atom a -- and
// the one-centre terms come last.
// nat (device, may be null) is read only for far pairs inside 7 A, which a
// cutoff of 7 A or more never has.
__global__ void __launch_bounds__(128) mz_fock_diag(MbMzLayout L, const int* __restrict__ nat,
                                                   const double* __restrict__ coord,
                                                   const double* __restrict__ w, const double* __restrict__ p,
                                                   const double* __restrict__ qe, const double* __restrict__ h,
                                                   double* __restrict__ f) {
  __shared__ double s_c[4][32][10];
  __shared__ double s_x[4][32];          // second addition (light atom, heavy partner)
  __shared__ double s_d[4][32][3];       // a far pair's three dipole additions on every diagonal element
  __shared__ unsigned short s_m[4][32];  // bit t: element t gets s_c; bit 14: diagonal elements then get
                                         // s_d[0..2]; bit 15: element 0 then gets s_x
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  const int a = blockIdx.x * 4 + wl;
  if (a >= L.numat) return;
  const int ia = L.iorbs[a];
  const int ne = ia * (ia + 1) / 2;
  const long long da = L.pair_off[L.pair_ptr[a + 1] - 1];
  double acc = lane < ne ? h[da + lane] : 0.0;
  const int nb0 = L.nbr_ptr[a], nb1 = L.nbr_ptr[a + 1];
  const double evA0 = DMUL(MZ_EV, MZ_A0);
  for (int base = 0; base < L.numat; base += 32) {
    const int b = base + lane;
    unsigned short mask = 0;
    if (b < L.numat && b != a) {
      // r^2 as fillij forms it (higher atom minus lower atom), so the stored test agrees with the layout
      const int hi = a > b ? a : b, lo = a > b ? b : a;
      const double dx = DSUB(coord[3 * hi], coord[3 * lo]);
      const double dy = DSUB(coord[3 * hi + 1], coord[3 * lo + 1]);
      const double dz = DSUB(coord[3 * hi + 2], coord[3 * lo + 2]);
      const double r2 = DADD(DADD(DMUL(dx, dx), DMUL(dy, dy)), DMUL(dz, dz));
      if (r2 < L.cutof2) {
        int lo_i = nb0, hi_i = nb1 - 1, e = -1;
        while (lo_i <= hi_i) {
          const int mid = (lo_i + hi_i) >> 1;
          const int v = L.nbr_atom[mid];
          if (v == b) { e = mid; break; }
          if (v < b) lo_i = mid + 1; else hi_i = mid - 1;
        }
        if (e >= 0) {
          const double* wk = w + L.pair_woff[L.nbr_entry[e]];
          double second = 0.0;
          bool two = false;
          for (int t = 0; t < ne; ++t) s_c[wl][lane][t] = mz_pair_diag_term(a, b, t, L, wk, p, &second, &two);
          mask = (unsigned short)((1u << ne) - 1u);
          if (two) {
            s_x[wl][lane] = second;
            mask |= (unsigned short)0x8000u;
          }
        }
      } else {
        // a pair outside cutof2 (fock2z.F90:440-634): the point-charge
        // monopole w1 = ev a0 / r, feathered inside 7 A (w1 const + (1 -
        // const) point, which is the point charge itself where const = 0),
        // and inside cutof1 the dipole terms, which vanish beyond 7 A
        const double rij = sqrt(r2);
        double point;
        const double cst = mz_feather(rij, &point);
        double w1 = point;
        const int ii = a > b ? a : b, jj = a > b ? b : a;  // the pair loop's roles
        if (cst != 0.0) {
          const int ni = nat[ii], nj = nat[jj];
          const double aee = 0.5 / c_far.am[ni] + 0.5 / c_far.am[nj];
          w1 = MZ_EV / sqrt(r2 / (MZ_A0 * MZ_A0) + aee * aee);
          w1 = w1 * cst + (1.0 - cst) * point;
        }
        const double c = DMUL(qe[b], w1);
        const int dg[4] = {0, 2, 5, 9};
        for (int q = 0; q < ia; ++q) {
          s_c[wl][lane][dg[q]] = c;
          mask |= (unsigned short)(1u << dg[q]);
        }
        if (cst != 0.0 && r2 < L.cutof1) {  // fock2z.F90:490-634
          const int ni = nat[ii], nj = nat[jj];
          const int iab = L.iorbs[ii], jba = L.iorbs[jj];
          const double ux = dx / rij, uy = dy / rij;
          double uz = dz / rij;
          if (fabs(uz) > 0.99999999) uz = copysign(1.0, uz);
          double w2 = 0.0, w3 = 0.0, w4 = 0.0, w5 = 0.0, w6 = 0.0, w7 = 0.0;
          if (iab > 1) {
            const double da = c_far.dd[ni], ade = 0.5 / c_far.ad[ni] + 0.5 / c_far.am[nj];
            const double rp = sqrt((rij / MZ_A0 + da) * (rij / MZ_A0 + da) + ade * ade);
            const double rm = sqrt((rij / MZ_A0 - da) * (rij / MZ_A0 - da) + ade * ade);
            const double ri2 = MZ_EV * (0.5 / rp - 0.5 / rm) * cst;
            w5 = ri2 * ux; w6 = ri2 * uy; w7 = ri2 * uz;
          }
          if (jba > 1) {
            const double da = c_far.dd[nj], ade = 0.5 / c_far.am[ni] + 0.5 / c_far.ad[nj];
            const double rp = sqrt((rij / MZ_A0 + da) * (rij / MZ_A0 + da) + ade * ade);
            const double rm = sqrt((rij / MZ_A0 - da) * (rij / MZ_A0 - da) + ade * ade);
            const double ri5 = -MZ_EV * (0.5 / rp - 0.5 / rm) * cst;
            w2 = ri5 * ux; w3 = ri5 * uy; w4 = ri5 * uz;
          }
          // this atom's p-s elements take the partner's charge times its own
          // dipole integrals; its diagonal takes the partner's p-s densities
          // times the partner's, doubled
          const bool mine_p = a == ii ? iab > 1 : jba > 1;
          const bool part_p = a == ii ? jba > 1 : iab > 1;
          const double qa = qe[b];
          const double ma[3] = {a == ii ? w5 : w2, a == ii ? w6 : w3, a == ii ? w7 : w4};
          const double mb[3] = {a == ii ? w2 : w5, a == ii ? w3 : w6, a == ii ? w4 : w7};
          if (mine_p) {
            const int sp[3] = {1, 3, 6};
            for (int q = 0; q < 3; ++q) {
              s_c[wl][lane][sp[q]] = DMUL(qa, ma[q]);
              mask |= (unsigned short)(1u << sp[q]);
            }
          }
          if (part_p) {
            const long long pb = L.pair_off[L.pair_ptr[b + 1] - 1];
            s_d[wl][lane][0] = DMUL(DMUL(p[pb + 1], mb[0]), 2.0);
            s_d[wl][lane][1] = DMUL(DMUL(p[pb + 3], mb[1]), 2.0);
            s_d[wl][lane][2] = DMUL(DMUL(p[pb + 6], mb[2]), 2.0);
            mask |= (unsigned short)0x4000u;
          }
        }
      }
    }
    s_m[wl][lane] = mask;
    __syncwarp();
    if (lane < ne) {
      const int nt = min(32, L.numat - base);
      for (int t = 0; t < nt; ++t) {
        const unsigned mk = s_m[wl][t];
        if (mk & (1u << lane)) acc = DADD(acc, s_c[wl][t][lane]);
        if ((mk & 0x4000u) && (lane == 0 || lane == 2 || lane == 5 || lane == 9)) {
          acc = DADD(acc, s_d[wl][t][0]);
          acc = DADD(acc, s_d[wl][t][1]);
          acc = DADD(acc, s_d[wl][t][2]);
        }
        if ((mk & 0x8000u) && lane == 0) acc = DADD(acc, s_x[wl][t]);
      }
    }
    __syncwarp();
  }
  // fock1_for_MOZYME
  if (lane < ne) {
    const int ilim = ne;
    const double* wo = w + L.pair_woff[L.pair_ptr[a + 1] - 1];
    int i = 1;
    while ((i * (i + 1)) / 2 <= lane) ++i;
    const int j = lane - (i * (i - 1)) / 2 + 1;
    const int ijw = (i * (i - 1)) / 2 + j;
    double sum = 0.0;
    for (int k = 1; k <= ia; ++k)
      for (int l = 1; l <= ia; ++l) {
        const int ijp = tri1(k, l);
        const int ikw = tri1(k, j), jlw = tri1(l, i);
        const double pv = p[da + ijp - 1];
        sum = DSUB(DADD(sum, DMUL(pv, wo[(ijw - 1) + ilim * (ijp - 1)])), DMUL(DMUL(0.5, pv), wo[(ikw - 1) + ilim * (jlw - 1)]));
      }
    f[da + lane] = DADD(acc, sum);
  }
}

// Off-diagonal blocks of stored pairs: F = H - exchange, 16 lanes per pair.
__global__ void __launch_bounds__(256) mz_fock_pairs(MbMzLayout L, const double* __restrict__ w,
                                                    const double* __restrict__ p, const double* __restrict__ h,
                                                    double* __restrict__ f) {
  const long long g = (blockIdx.x * (long long)blockDim.x + threadIdx.x);
  const long long e = g >> 4;
  const int t = (int)(g & 15);
  if (e >= L.npairs) return;
  const int ii = L.pair_i[e], jj = L.pair_j[e];
  if (ii == jj) return;
  const int ia = L.iorbs[ii], ib = L.iorbs[jj];
  const long long off = L.pair_off[e];
  const double* wk = w + L.pair_woff[e];
  if (ia >= 3 && ib >= 3) {
    const int mu = t / 4 + 1, nu = t % 4 + 1;
    double s = 0.0;
    for (int i2 = 0; i2 < 16; ++i2) {
      const int lam = i2 / 4 + 1, sig = i2 % 4 + 1;
      s = DADD(s, DMUL(p[off + i2], wk[(tri1(mu, lam) - 1) * 10 + tri1(nu, sig) - 1]));
    }
    f[off + t] = DSUB(h[off + t], DMUL(s, 0.5));
  } else if (ia >= 3 || ib >= 3) {
    if (t >= 4) return;
    double s = 0.0;
    for (int j = 1; j <= 4; ++j) s = DADD(s, DMUL(p[off + j - 1], wk[c_pidx[t * 4 + j - 1] - 1]));
    f[off + t] = DSUB(h[off + t], DMUL(s, 0.5));
  } else {
    if (t != 0) return;
    f[off] = DSUB(h[off], DMUL(DMUL(p[off], wk[0]), 0.5));
  }
}

int grid_for(long long n) {
  long long b = (n + 255) / 256;
  return (int)(b > 148 * 8 ? 148 * 8 : (b < 1 ? 1 : b));
}

template <class T>
int upload(const std::vector<T>& v, const T** out, size_t capacity = 0) {
  T* d = nullptr;
  const size_t n = v.size() > capacity ? v.size() : capacity;
  if (n > 0) {
    MB_CUDA(cudaMalloc(&d, sizeof(T) * n));
    if (!v.empty()) MB_CUDA(cudaMemcpy(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  }
  *out = d;
  return MB_OK;
}

// ---------------------------------------------------------------- LMO index on the device
// The per-atom index (atom_ptr, atom_lmo, atom_coff) rebuilt from the LMOs'
// own arrays, as build_atom_index does on the host: each atom's LMOs in
// ascending order with the offset of the atom's coefficients in the LMO.

// Per LMO (one warp, lanes over its atoms): count its atoms, and the
// coefficient offset of every entry (a warp scan of the atoms' orbital counts).
__global__ void mzr_count(int numat, int nlmo, const int* __restrict__ iorbs, const int* __restrict__ ncf,
                          const int* __restrict__ nncf, const int* __restrict__ icocc, const int* __restrict__ ncocc,
                          long long nentries, long long ncoeff, int* __restrict__ cnt, int* __restrict__ ecoff,
                          int* __restrict__ err) {
  const int lane = threadIdx.x & 31;
  const int i = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  if (i >= nlmo) return;  // warp-uniform
  const long long j0 = nncf[i], j1 = j0 + ncf[i];
  if (j0 < 0 || j1 > nentries) {
    if (lane == 0) atomicOr(err, 1);
    return;
  }
  long long c = ncocc[i];
  for (long long q0 = j0; q0 < j1; q0 += 32) {
    const long long jj = q0 + lane;
    int a = -1, no = 0;
    if (jj < j1) {
      a = icocc[jj] - 1;
      if (a < 0 || a >= numat) atomicOr(err, 1);
      else no = iorbs[a];
    }
    int incl = no;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += t;
    }
    if (jj < j1 && a >= 0 && a < numat) {
      atomicAdd(&cnt[a], 1);
      ecoff[jj] = (int)(c + incl - no);
    }
    c += __shfl_sync(0xffffffffu, incl, 31);
  }
  if (lane == 0 && c > ncoeff) atomicOr(err, 2);
}

// Exclusive scan of the counts into atom_ptr (numat + 1 entries); one CTA.
__global__ void mzr_scan(int numat, const int* __restrict__ cnt, int* __restrict__ ptr) {
  __shared__ int s_warp[32];
  __shared__ int s_carry;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  if (tid == 0) s_carry = 0;
  __syncthreads();
  for (int b0 = 0; b0 < numat; b0 += blockDim.x) {
    const int a = b0 + tid;
    int v = a < numat ? cnt[a] : 0;
    int incl = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += t;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    int off = s_carry;
    for (int w = 0; w < warp; ++w) off += s_warp[w];
    if (a < numat) ptr[a] = off + incl - v;
    __syncthreads();
    if (tid == 0) {
      int tot = 0;
      for (int w = 0; w < nw; ++w) tot += s_warp[w];
      s_carry += tot;
    }
    __syncthreads();
  }
  if (tid == 0) ptr[numat] = s_carry;
}

// Per LMO (one warp, lanes over its atoms): drop every entry into its atom's
// segment (any order).
__global__ void mzr_scatter(int numat, int nlmo, const int* __restrict__ ncf, const int* __restrict__ nncf,
                            const int* __restrict__ icocc, long long nentries, const int* __restrict__ ptr,
                            const int* __restrict__ ecoff, int* __restrict__ cursor,
                            unsigned long long* __restrict__ tmp, int* __restrict__ err) {
  const int lane = threadIdx.x & 31;
  const int i = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  if (i >= nlmo) return;
  const long long j0 = nncf[i], j1 = j0 + ncf[i];
  if (j0 < 0 || j1 > nentries) return;
  for (long long jj = j0 + lane; jj < j1; jj += 32) {
    const int a = icocc[jj] - 1;
    if (a < 0 || a >= numat) continue;
    const long long at = (long long)ptr[a] + atomicAdd(&cursor[a], 1);
    if (at >= nentries) { atomicOr(err, 4); continue; }  // overlapping atom lists
    tmp[at] = ((unsigned long long)(unsigned)i << 32) | (unsigned)ecoff[jj];
  }
}

// Per atom: each entry's place is the number of entries with a smaller LMO
// index (ties, which well-formed LMOs do not have, broken by position).
__global__ void mzr_order(const int* __restrict__ ptr, const unsigned long long* __restrict__ tmp, long long nentries,
                          int* __restrict__ atom_lmo, int* __restrict__ atom_coff) {
  constexpr int kStage = 2048;
  __shared__ unsigned s_key[kStage];
  const int a = blockIdx.x;
  const int b = ptr[a], m = ptr[a + 1] - b;
  if ((long long)b + m > nentries) return;  // flagged by mzr_scatter
  const bool staged = m <= kStage;
  if (staged)
    for (int e = threadIdx.x; e < m; e += blockDim.x) s_key[e] = (unsigned)(tmp[b + e] >> 32);
  __syncthreads();
  for (int e = threadIdx.x; e < m; e += blockDim.x) {
    const unsigned long long v = tmp[b + e];
    const unsigned key = (unsigned)(v >> 32);
    int rank = 0;
    for (int f = 0; f < m; ++f) {
      const unsigned k2 = staged ? s_key[f] : (unsigned)(tmp[b + f] >> 32);
      rank += (k2 < key) || (k2 == key && f < e);
    }
    atom_lmo[b + rank] = (int)key;
    atom_coff[b + rank] = (int)(unsigned)(v & 0xffffffffull);
  }
}

}  // namespace

extern "C" int mb_mz_layout_create(int numat, const int* iorbs, const double* coord, double cutof1, double cutof2,
                                   MbMzLayout* out, long long* nijbo) {
  if (numat <= 0 || !iorbs || !coord || !out) return mb_set_error(MB_ERR_ARG, "mb_mz_layout_create: bad args");
  memset(out, 0, sizeof(*out));
  for (int i = 0; i < numat; ++i)
    if (iorbs[i] < 0 || iorbs[i] > 4) return mb_set_error(MB_ERR_UNSUPPORTED, "MOZYME layout: s and p shells only");
  for (long long q = 0; q < 3LL * numat; ++q)
    if (!isfinite(coord[q])) return mb_set_error(MB_ERR_ARG, "MOZYME layout: non-finite coordinate");
  std::vector<int> pi, pj, ptr(numat + 1, 0);
  std::vector<long long> po;
  long long mpack = 0;
  auto r2_of = [&](int i, int j) {
    const double dx = coord[3 * i] - coord[3 * j], dy = coord[3 * i + 1] - coord[3 * j + 1],
                 dz = coord[3 * i + 2] - coord[3 * j + 2];
    return dx * dx + dy * dy + dz * dz;
  };
  if (nijbo) {
    // every pair's class is wanted: the full triangle
    for (int i = 0; i < numat; ++i) {
      ptr[i] = (int)pi.size();
      const int io = iorbs[i];
      for (int j = 0; j < i; ++j) {
        const double r = r2_of(i, j);
        long long v;
        if (r < cutof2) {
          v = mpack;
          pi.push_back(i);
          pj.push_back(j);
          po.push_back(mpack);
          mpack += (long long)io * iorbs[j];
        } else {
          v = r < cutof1 ? -2 : -1;
        }
        nijbo[(long long)i * numat + j] = nijbo[(long long)j * numat + i] = v;
      }
      pi.push_back(i);
      pj.push_back(i);
      po.push_back(mpack);
      nijbo[(long long)i * numat + i] = mpack;
      mpack += (long long)io * (io + 1) / 2;
    }
  } else {
    // Only the stored pairs (r^2 < cutof2) are wanted: candidates come from a
    // grid of cells at least the cutoff wide (a partner within the cutoff is
    // in the same or a neighbouring cell), each atom's stored partners j < i
    // sorted ascending, so the entries are the full triangle's, in its order.
    double lo[3] = {coord[0], coord[1], coord[2]}, hi[3] = {coord[0], coord[1], coord[2]};
    for (int i = 1; i < numat; ++i)
      for (int d = 0; d < 3; ++d) {
        lo[d] = std::min(lo[d], coord[3 * i + d]);
        hi[d] = std::max(hi[d], coord[3 * i + d]);
      }
    const double rc = cutof2 > 0.0 ? sqrt(cutof2) : 0.0;
    int nc[3];
    double edge[3];
    long long ncell = 1;
    for (int d = 0; d < 3; ++d) {
      const double ext = hi[d] - lo[d];
      int k = rc > 0.0 ? (int)std::min(256.0, floor(ext / (rc * (1.0 + 1.0e-9) + 1.0e-9))) : 1;
      if (k < 1) k = 1;
      nc[d] = k;
      edge[d] = std::max(ext / k, rc * (1.0 + 1.0e-9) + 1.0e-9);
      ncell *= k;
    }
    auto cell_of = [&](int i, int d) {
      int c = (int)((coord[3 * i + d] - lo[d]) / edge[d]);
      return c < 0 ? 0 : (c >= nc[d] ? nc[d] - 1 : c);
    };
    std::vector<int> cstart(ncell + 1, 0), catom(numat), acell(numat);
    for (int i = 0; i < numat; ++i) {
      acell[i] = (cell_of(i, 0) * nc[1] + cell_of(i, 1)) * nc[2] + cell_of(i, 2);
      cstart[acell[i] + 1]++;
    }
    for (long long c = 0; c < ncell; ++c) cstart[c + 1] += cstart[c];
    {
      std::vector<int> fill(cstart.begin(), cstart.end() - 1);
      for (int i = 0; i < numat; ++i) catom[fill[acell[i]]++] = i;  // ascending atoms in every cell
    }
    std::vector<int> cand;
    for (int i = 0; i < numat; ++i) {
      ptr[i] = (int)pi.size();
      const int io = iorbs[i];
      cand.clear();
      if (rc > 0.0) {
        const int cx = cell_of(i, 0), cy = cell_of(i, 1), cz = cell_of(i, 2);
        for (int x = std::max(cx - 1, 0); x <= std::min(cx + 1, nc[0] - 1); ++x)
          for (int y = std::max(cy - 1, 0); y <= std::min(cy + 1, nc[1] - 1); ++y)
            for (int z = std::max(cz - 1, 0); z <= std::min(cz + 1, nc[2] - 1); ++z) {
              const long long c = ((long long)x * nc[1] + y) * nc[2] + z;
              for (int q = cstart[c]; q < cstart[c + 1]; ++q) {
                const int j = catom[q];
                if (j >= i) break;
                if (r2_of(i, j) < cutof2) cand.push_back(j);
              }
            }
        std::sort(cand.begin(), cand.end());
      }
      for (int j : cand) {
        pi.push_back(i);
        pj.push_back(j);
        po.push_back(mpack);
        mpack += (long long)io * iorbs[j];
      }
      pi.push_back(i);
      pj.push_back(i);
      po.push_back(mpack);
      mpack += (long long)io * (io + 1) / 2;
    }
  }
  ptr[numat] = (int)pi.size();
  // integral blocks in entry order: the dense W's layout without the far pairs
  std::vector<long long> woff(pi.size());
  long long nw = 0;
  for (size_t e = 0; e < pi.size(); ++e) {
    woff[e] = nw;
    const int a = iorbs[pi[e]], b = iorbs[pj[e]];
    if (pi[e] == pj[e]) {
      const long long il = (long long)a * (a + 1) / 2;
      nw += il * il;
    } else {
      nw += (a >= 3 && b >= 3) ? 100 : ((a >= 3 || b >= 3) ? 10 : 1);
    }
  }
  // stored partners of every atom in both directions, ascending
  std::vector<int> ncount(numat + 1, 0);
  for (size_t e = 0; e < pi.size(); ++e)
    if (pi[e] != pj[e]) { ncount[pi[e] + 1]++; ncount[pj[e] + 1]++; }
  for (int a = 0; a < numat; ++a) ncount[a + 1] += ncount[a];
  std::vector<int> nat_(ncount[numat]), nfill(ncount.begin(), ncount.end() - 1);
  std::vector<long long> nent(ncount[numat]);
  for (int a = 0; a < numat; ++a) {  // partners b < a from a's own entries, then b > a from later atoms
    for (int e = ptr[a]; e < ptr[a + 1]; ++e)
      if (pj[e] != a) { nat_[nfill[a]] = pj[e]; nent[nfill[a]] = e; nfill[a]++; }
  }
  for (int b = 0; b < numat; ++b)
    for (int e = ptr[b]; e < ptr[b + 1]; ++e)
      if (pj[e] != b) { const int a = pj[e]; nat_[nfill[a]] = b; nent[nfill[a]] = e; nfill[a]++; }
  std::vector<int> io(iorbs, iorbs + numat);
  std::vector<int> fst(numat);
  int norbs = 0;
  for (int a = 0; a < numat; ++a) { fst[a] = norbs; norbs += iorbs[a]; }
  out->norbs = norbs;
  out->numat = numat;
  out->mpack = mpack;
  out->npairs = (long long)pi.size();
  out->nw = nw;
  out->cutof1 = cutof1;
  out->cutof2 = cutof2;
  int rc = upload(io, &out->iorbs);
  if (rc == MB_OK) rc = upload(ptr, &out->pair_ptr);
  if (rc == MB_OK) rc = upload(pi, &out->pair_i);
  if (rc == MB_OK) rc = upload(pj, &out->pair_j);
  if (rc == MB_OK) rc = upload(po, &out->pair_off);
  if (rc == MB_OK) rc = upload(woff, &out->pair_woff);
  if (rc == MB_OK) rc = upload(ncount, &out->nbr_ptr);
  if (rc == MB_OK) rc = upload(nat_, &out->nbr_atom);
  if (rc == MB_OK) rc = upload(nent, &out->nbr_entry);
  if (rc == MB_OK) rc = upload(fst, &out->first);
  if (rc != MB_OK) mb_mz_layout_destroy(out);
  return rc;
}

extern "C" int mb_mz_layout_destroy(MbMzLayout* L) {
  if (!L) return MB_OK;
  cudaFree((void*)L->iorbs);
  cudaFree((void*)L->pair_ptr);
  cudaFree((void*)L->pair_i);
  cudaFree((void*)L->pair_j);
  cudaFree((void*)L->pair_off);
  cudaFree((void*)L->pair_woff);
  cudaFree((void*)L->nbr_ptr);
  cudaFree((void*)L->nbr_atom);
  cudaFree((void*)L->nbr_entry);
  cudaFree((void*)L->first);
  memset(L, 0, sizeof(*L));
  return MB_OK;
}

extern "C" int mb_mz_idiag(const MbMzLayout* L, long long* idiag) {
  if (!L || !idiag) return mb_set_error(MB_ERR_ARG, "mb_mz_idiag: bad args");
  std::vector<int> io(L->numat), ptr(L->numat + 1);
  std::vector<long long> po(L->npairs);
  MB_CUDA(cudaMemcpy(io.data(), L->iorbs, sizeof(int) * L->numat, cudaMemcpyDeviceToHost));
  MB_CUDA(cudaMemcpy(ptr.data(), L->pair_ptr, sizeof(int) * (L->numat + 1), cudaMemcpyDeviceToHost));
  MB_CUDA(cudaMemcpy(po.data(), L->pair_off, sizeof(long long) * L->npairs, cudaMemcpyDeviceToHost));
  long long l = 0;
  for (int i = 0; i < L->numat; ++i) {  // iter_for_MOZYME.F90:183-190
    long long j = po[ptr[i + 1] - 1];    // diagonal block of atom i (0-based)
    for (int k = 1; k <= io[i]; ++k) {
      j += k;
      idiag[l++] = j;  // 1-based position, like the reference
    }
  }
  return MB_OK;
}

static int build_atom_index(int numat, const int* iorbs, int nlmo, const int* ncf, const int* nncf,
                            const int* icocc, const int* ncocc, long long cocc_dim, std::vector<int>& cnt,
                            std::vector<int>& lmo, std::vector<int>& coff) {
  cnt.assign(numat + 1, 0);
  for (int i = 0; i < nlmo; ++i)
    for (int jj = nncf[i]; jj < nncf[i] + ncf[i]; ++jj) {
      const int a = icocc[jj] - 1;
      if (a < 0 || a >= numat) return mb_set_error(MB_ERR_ARG, "MOZYME LMOs: atom number out of range");
      cnt[a + 1]++;
    }
  for (int a = 0; a < numat; ++a) cnt[a + 1] += cnt[a];
  std::vector<int> fill(cnt.begin(), cnt.end() - 1);
  lmo.assign(cnt[numat], 0);
  coff.assign(cnt[numat], 0);
  for (int i = 0; i < nlmo; ++i) {  // ascending LMO order per atom by construction
    long long c = ncocc[i];
    for (int jj = nncf[i]; jj < nncf[i] + ncf[i]; ++jj) {
      const int a = icocc[jj] - 1;
      lmo[fill[a]] = i;
      coff[fill[a]] = (int)c;
      fill[a]++;
      c += iorbs[a];
    }
    if (c > cocc_dim) return mb_set_error(MB_ERR_ARG, "MOZYME LMOs: cocc too short for the atom lists");
  }
  return MB_OK;
}

extern "C" int mb_mz_lmos_create(int numat, const int* iorbs, int nlmo, const int* ncf, const int* nncf,
                                 const int* icocc, const int* ncocc, const double* cocc, long long icocc_dim,
                                 long long cocc_dim, MbMzLmos* out) {
  if (numat <= 0 || nlmo < 0 || !out) return mb_set_error(MB_ERR_ARG, "mb_mz_lmos_create: bad args");
  memset(out, 0, sizeof(*out));
  for (int i = 0; i < nlmo; ++i)
    if ((long long)nncf[i] + ncf[i] > icocc_dim) return mb_set_error(MB_ERR_ARG, "mb_mz_lmos_create: icocc too short");
  std::vector<int> cnt, lmo, coff;
  MB_TRY(build_atom_index(numat, iorbs, nlmo, ncf, nncf, icocc, ncocc, cocc_dim, cnt, lmo, coff));
  std::vector<double> cv(cocc, cocc + cocc_dim);
  std::vector<int> vncf(ncf, ncf + nlmo), vnncf(nncf, nncf + nlmo), vic(icocc, icocc + icocc_dim),
      vnco(ncocc, ncocc + nlmo);
  out->nlmo = nlmo;
  out->nentries = icocc_dim;
  out->ncoeff = cocc_dim;
  // the index arrays hold up to icocc_dim entries, so a refresh never reallocates them
  int rc = upload(cnt, &out->atom_ptr);
  if (rc == MB_OK) rc = upload(lmo, &out->atom_lmo, (size_t)icocc_dim);
  if (rc == MB_OK) rc = upload(coff, &out->atom_coff, (size_t)icocc_dim);
  if (rc == MB_OK) rc = upload(cv, &out->cocc);
  if (rc == MB_OK) rc = upload(vncf, &out->ncf);
  if (rc == MB_OK) rc = upload(vnncf, &out->nncf);
  if (rc == MB_OK) rc = upload(vic, &out->icocc);
  if (rc == MB_OK) rc = upload(vnco, &out->ncocc);
  if (rc != MB_OK) mb_mz_lmos_destroy(out);
  return rc;
}

extern "C" int mb_mz_lmos_refresh(int numat, const int* iorbs, MbMzLmos* Q) {
  if (!Q || !iorbs) return mb_set_error(MB_ERR_ARG, "mb_mz_lmos_refresh: bad args");
  const int n = Q->nlmo;
  std::vector<int> ncf(n), nncf(n), ncocc(n), ic(Q->nentries);
  MB_CUDA(cudaMemcpy(ncf.data(), Q->ncf, sizeof(int) * n, cudaMemcpyDeviceToHost));
  MB_CUDA(cudaMemcpy(nncf.data(), Q->nncf, sizeof(int) * n, cudaMemcpyDeviceToHost));
  MB_CUDA(cudaMemcpy(ncocc.data(), Q->ncocc, sizeof(int) * n, cudaMemcpyDeviceToHost));
  MB_CUDA(cudaMemcpy(ic.data(), Q->icocc, sizeof(int) * Q->nentries, cudaMemcpyDeviceToHost));
  std::vector<int> cnt, lmo, coff;
  MB_TRY(build_atom_index(numat, iorbs, n, ncf.data(), nncf.data(), ic.data(), ncocc.data(), Q->ncoeff, cnt, lmo,
                          coff));
  cudaFree((void*)Q->atom_ptr);
  cudaFree((void*)Q->atom_lmo);
  cudaFree((void*)Q->atom_coff);
  Q->atom_ptr = Q->atom_lmo = Q->atom_coff = nullptr;
  MB_TRY(upload(cnt, &Q->atom_ptr));
  MB_TRY(upload(lmo, &Q->atom_lmo, (size_t)Q->nentries));
  MB_TRY(upload(coff, &Q->atom_coff, (size_t)Q->nentries));
  return MB_OK;
}

// mb_mz_lmos_refresh on the device: the same index, in place (the index
// arrays hold nentries entries from mb_mz_lmos_create), on `stream`, with
// iorbs a device array.  Synchronises the stream once to report malformed
// LMOs as the host version does.
extern "C" int mb_mz_lmos_refresh_dev(int numat, const int* iorbs_dev, MbMzLmos* Q, cudaStream_t stream) {
  if (!Q || !iorbs_dev || numat <= 0) return mb_set_error(MB_ERR_ARG, "mb_mz_lmos_refresh_dev: bad args");
  const int n = Q->nlmo;
  const long long ne = Q->nentries;
  const size_t bytes = sizeof(int) * (2 * (size_t)numat + (size_t)ne + 8) + sizeof(unsigned long long) * (size_t)ne;
  char* ws = nullptr;
  MB_CUDA(mb_malloc_async((void**)&ws, bytes, stream));
  unsigned long long* tmp = (unsigned long long*)ws;
  int* cnt = (int*)(tmp + ne);
  int* cursor = cnt + numat;
  int* ecoff = cursor + numat;
  int* err = ecoff + ne;
  int rc = MB_OK;
  if (cudaMemsetAsync(cnt, 0, sizeof(int) * 2 * (size_t)numat, stream) != cudaSuccess ||
      cudaMemsetAsync(err, 0, sizeof(int), stream) != cudaSuccess)
    rc = mb_set_error(MB_ERR_CUDA, "mb_mz_lmos_refresh_dev: memset");
  const int nb = (int)(((long long)n * 32 + 127) / 128);  // a warp per LMO
  if (rc == MB_OK && n > 0) {
    mzr_count<<<nb, 128, 0, stream>>>(numat, n, iorbs_dev, Q->ncf, Q->nncf, Q->icocc, Q->ncocc, ne, Q->ncoeff, cnt,
                                      ecoff, err);
    if (cudaGetLastError() != cudaSuccess) rc = mb_set_error(MB_ERR_CUDA, "mb_mz_lmos_refresh_dev: count");
  }
  if (rc == MB_OK) {
    mzr_scan<<<1, 1024, 0, stream>>>(numat, cnt, (int*)Q->atom_ptr);
    if (cudaGetLastError() != cudaSuccess) rc = mb_set_error(MB_ERR_CUDA, "mb_mz_lmos_refresh_dev: scan");
  }
  if (rc == MB_OK && n > 0) {
    mzr_scatter<<<nb, 128, 0, stream>>>(numat, n, Q->ncf, Q->nncf, Q->icocc, ne, Q->atom_ptr, ecoff, cursor, tmp,
                                        err);
    if (cudaGetLastError() != cudaSuccess) rc = mb_set_error(MB_ERR_CUDA, "mb_mz_lmos_refresh_dev: scatter");
  }
  if (rc == MB_OK) {
    mzr_order<<<numat, 128, 0, stream>>>(Q->atom_ptr, tmp, ne, (int*)Q->atom_lmo, (int*)Q->atom_coff);
    if (cudaGetLastError() != cudaSuccess) rc = mb_set_error(MB_ERR_CUDA, "mb_mz_lmos_refresh_dev: order");
  }
  int herr = 0;
  if (rc == MB_OK && (cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
                      cudaStreamSynchronize(stream) != cudaSuccess))
    rc = mb_set_error(MB_ERR_CUDA, "mb_mz_lmos_refresh_dev: status");
  cudaFreeAsync(ws, stream);
  if (rc != MB_OK) return rc;
  if (herr & 1) return mb_set_error(MB_ERR_ARG, "MOZYME LMOs: atom number out of range");
  if (herr & 2) return mb_set_error(MB_ERR_ARG, "MOZYME LMOs: cocc too short for the atom lists");
  if (herr & 4) return mb_set_error(MB_ERR_ARG, "MOZYME LMOs: atom lists overlap in icocc");
  return MB_OK;
}

extern "C" int mb_mz_lmos_destroy(MbMzLmos* Q) {
  if (!Q) return MB_OK;
  cudaFree((void*)Q->atom_ptr);
  cudaFree((void*)Q->atom_lmo);
  cudaFree((void*)Q->atom_coff);
  cudaFree((void*)Q->cocc);
  cudaFree((void*)Q->ncf);
  cudaFree((void*)Q->nncf);
  cudaFree((void*)Q->icocc);
  cudaFree((void*)Q->ncocc);
  memset(Q, 0, sizeof(*Q));
  return MB_OK;
}

extern "C" int mb_mz_density_dev(const MbMzLayout* L, const MbMzLmos* Q, int mode, const double* partp, double* p,
                                 cudaStream_t stream) {
  if (!L || !Q || !p || (mode != 0 && !partp)) return mb_set_error(MB_ERR_ARG, "mb_mz_density_dev: bad args");
  if (L->npairs == 0) return MB_OK;
  const double spinfa = (mode == 0 || mode == 1) ? 2.0 : (mode == -1 ? -2.0 : 1.0);
  const int scale = fabs(spinfa - 1.0) > 1.0e-10;
  long long blocks = (L->npairs * 32 + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  mz_density_kernel<<<(int)blocks, 256, 0, stream>>>(*L, *Q, mode, partp, p, spinfa, scale);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

extern "C" size_t mb_mz_helecz_ws_bytes(void) { return sizeof(double) * 2 * 148 * 4; }

extern "C" int mb_mz_helecz_ws(long long mpack, int norbs, const long long* idiag, const double* p, const double* h,
                               const double* f, double* out, double* ws, cudaStream_t stream) {
  if (!idiag || !p || !h || !f || !out || !ws) return mb_set_error(MB_ERR_ARG, "mb_mz_helecz: bad args");
  const int nb = 148 * 4;
  mz_helecz_partials<<<nb, 256, 0, stream>>>(mpack, norbs, idiag, p, h, f, ws);
  MB_LAUNCH_CHECK();
  mz_helecz_final<<<1, 32, 0, stream>>>(nb, ws, out);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

extern "C" size_t mb_mz_cnvgz_ws_bytes(void) { return 256; }

extern "C" int mb_mz_cnvgz_ws(int norbs, long long mpack, double* pnew, double* p, double* p1, double* p2, double* p3,
                              int niter, const long long* idiag, int use3, double* pmax_out, void* ws,
                              cudaStream_t stream) {
  if (norbs <= 0 || !pnew || !p || !p1 || !p2 || !p3 || !idiag || !pmax_out || !ws)
    return mb_set_error(MB_ERR_ARG, "mb_mz_cnvgz: bad args");
  unsigned long long* bits = (unsigned long long*)ws;
  double* fac = (double*)ws + 1;
  MB_CUDA(cudaMemsetAsync(bits, 0, sizeof(unsigned long long), stream));
  const int g = grid_for(mpack > norbs ? mpack : norbs);
  mz_cnvgz_gather<<<g, 256, 0, stream>>>(norbs, mpack, idiag, pnew, p, p2, p3, bits);
  MB_LAUNCH_CHECK();
  mz_cnvgz_factor<<<1, 32, 0, stream>>>(norbs, niter, use3, p1, p2, p3, fac);
  MB_LAUNCH_CHECK();
  mz_cnvgz_extrap<<<grid_for(mpack), 256, 0, stream>>>(mpack, fac, pnew, p);
  MB_LAUNCH_CHECK();
  mz_cnvgz_damp<<<grid_for(norbs), 256, 0, stream>>>(norbs, niter, use3, idiag, bits, pnew, p1, p2, p3);
  MB_LAUNCH_CHECK();
  copy_kernel<<<grid_for(mpack), 256, 0, stream>>>(mpack, pnew, p);
  MB_LAUNCH_CHECK();
  MB_CUDA(cudaMemcpyAsync(pmax_out, bits, sizeof(double), cudaMemcpyDeviceToDevice, stream));
  return MB_OK;
}

extern "C" size_t mb_mz_fock_ws_bytes(const MbMzLayout* L) {
  return L ? sizeof(double) * (size_t)L->numat : 0;
}

extern "C" int mb_mz_fock_nat_dev(const MbMzLayout* L, const int* nat, const double* coord, const double* w,
                                  const double* ptot, const double* h, double* f, void* ws, cudaStream_t stream) {
  if (!L || !coord || !w || !ptot || !h || !f || !ws) return mb_set_error(MB_ERR_ARG, "mb_mz_fock_dev: bad args");
  // far pairs inside PM7's 7 A feathering radius need the elements
  if (!(L->cutof2 >= 49.0) && !nat)
    return mb_set_error(MB_ERR_UNSUPPORTED, "mb_mz_fock_dev: cutof2 < 49 (7 A) needs nat (mb_mz_fock_nat_dev)");
  if (nat) MB_TRY(far_params_init());
  double* qe = (double*)ws;
  mz_chrge<<<grid_for(L->numat), 256, 0, stream>>>(*L, ptot, qe);
  MB_LAUNCH_CHECK();
  mz_fock_diag<<<(L->numat + 3) / 4, 128, 0, stream>>>(*L, nat, coord, w, ptot, qe, h, f);
  MB_LAUNCH_CHECK();
  const long long thr = L->npairs * 16;
  mz_fock_pairs<<<(unsigned)((thr + 255) / 256), 256, 0, stream>>>(*L, w, ptot, h, f);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

extern "C" int mb_mz_fock_dev(const MbMzLayout* L, const double* coord, const double* w, const double* ptot,
                              const double* h, double* f, void* ws, cudaStream_t stream) {
  return mb_mz_fock_nat_dev(L, nullptr, coord, w, ptot, h, f, ws, stream);
}
