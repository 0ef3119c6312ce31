// diagg1 (MOZYME/diagg1.F90:16-503) on the device: for every virtual LMO psi_i
// the product ws = F psi_i on the LMO's atoms, the LMO energy eigv(i), and
// its interactions fmo(i, j) = <psi_j | ws> with the occupied LMOs, under the
// reference's cutoffs and in its order; optionally the occupied LMO energies.
//
// One CTA per virtual LMO.  Its atoms, their squared coefficients (avir),
// ws and aov live in shared memory; three bitmaps over the atoms (the LMO's
// atoms, the partners of its first atom, the partners of its second atom)
// answer the reference's pair tests in O(1).  Every ws element, eigv and
// every fmo(i, j) is one thread's sequential sum in the reference's term
// order, so all of them are bit-identical.  The interaction list is written
// in two passes: a count per virtual LMO, an exclusive scan on the host, and
// the ordered write (entries for LMO i in ascending j, LMOs in order), which
// reproduces the reference's running counter ijc without a sequential loop.
#include <math.h>
#include <string.h>

#include <vector>

#include <algorithm>

#include "mb_common.cuh"

namespace {

constexpr int MZ_MAXA = 512;  // atoms per virtual LMO handled by one CTA
constexpr int MZ_T = 128;
// diagg1's rebuild: evaluated candidates each warp keeps in shared memory
constexpr int MZD_CAND = 256;
// 32-bit words of diagg1's three atom bitmaps, rounded to an even count so the
// candidate values after them are 8-byte aligned
__host__ __device__ __forceinline__ int mzd_bits_words(int numat) { return (3 * ((numat + 31) / 32) + 1) & ~1; }

__device__ long long pair_offset(const MbMzLayout& L, int a, int b) {
  if (a == b) return L.pair_off[L.pair_ptr[a + 1] - 1];
  int lo = L.nbr_ptr[a], hi = L.nbr_ptr[a + 1] - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int v = L.nbr_atom[mid];
    if (v == b) return L.pair_off[L.nbr_entry[mid]];
    if (v < b) lo = mid + 1; else hi = mid - 1;
  }
  return -1;  // outside cutof2: the reference's nijbo is -1 or -2, tested as < 0
}

// aocc(kk) = sum of squared coefficients of entry kk (one thread per LMO).
__global__ void mzd_aocc(MbMzLmos Q, const int* __restrict__ iorbs, double* __restrict__ aocc) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < Q.nlmo; j += gridDim.x * blockDim.x) {
    const int loopj = Q.ncocc[j];
    int kl = 0;
    for (int kk = Q.nncf[j]; kk < Q.nncf[j] + Q.ncf[j]; ++kk) {
      const int k1 = Q.icocc[kk] - 1;
      double sum = 0.0;
      for (int k = 0; k < iorbs[k1]; ++k) {
        const double c = Q.cocc[loopj + kl];
        sum = DADD(sum, DMUL(c, c));
        ++kl;
      }
      aocc[kk] = sum;
    }
  }
}

struct DiagArgs {
  MbMzLayout L;
  MbMzLmos occ, vir;
  const double* fao;
  const double* p;
  const double* aocc;
  double cutoff, flim, oldlim;
  int mode;                       // 0: count, 1: write (rebuild), 2: recompute on the old list
  int* stash_j;                   // count pass: the appended entries of LMO i (j + 1) at i * stash_cap ..,
  double* stash_v;                //   their values; the write pass then only has to copy them
  int stash_cap;                  //   0: no stash.  Write pass: LMOs with nfmo <= stash_cap are skipped
  const long long* list_off;      // write / recompute: first list position of each virtual LMO
  int* nfmo;                      // count pass: entries per virtual LMO
  int* ifmo;
  double* fmo;
  double* eigv;
  double* sumt_part;              // per virtual LMO, sum of |fmo| in j order
  unsigned long long* tiny_bits;  // max |fmo| (non-negative doubles order like their bits)
  int* err;
};

__device__ __forceinline__ bool bit_test(const unsigned* bm, int a) { return (bm[a >> 5] >> (a & 31)) & 1u; }

// Local index of atom a in the LMO's atom list (sorted copy), or -1.
__device__ __forceinline__ int local_of(const int* s_sorted, const int* s_sidx, int n, int a) {
  int lo = 0, hi = n - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int v = s_sorted[mid];
    if (v == a) return s_sidx[mid];
    if (v < a) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

// fmo(i, j) over occupied LMO j's atoms that belong to virtual LMO i.
__device__ double mzd_fmo(const DiagArgs& A, int j, const unsigned* lat, const int* s_sorted, const int* s_sidx,
                          int nce, const double* s_aov, const int* s_wpos, const double* s_ws, bool* lij) {
  const int loopj = A.occ.ncocc[j];
  double sum = 0.0;
  int kl = 0;
  *lij = false;
  for (int kk = A.occ.nncf[j]; kk < A.occ.nncf[j] + A.occ.ncf[j]; ++kk) {
    const int k1 = A.occ.icocc[kk] - 1;
    const int nk = A.L.iorbs[k1];
    if (!bit_test(lat, k1)) { kl += nk; continue; }
    const int li = local_of(s_sorted, s_sidx, nce, k1);
    if (DMUL(A.aocc[kk], s_aov[li]) < A.cutoff) { kl += nk; continue; }
    *lij = true;
    for (int k = 0; k < nk; ++k) {
      sum = DADD(sum, DMUL(s_ws[s_wpos[li] + k], A.occ.cocc[loopj + kl]));
      ++kl;
    }
  }
  return sum;
}

__global__ void __launch_bounds__(MZ_T) mzd_virtual(DiagArgs A) {
  extern __shared__ unsigned s_bits[];  // lat | near1 | near2, ceil(numat/32) words each
  __shared__ int s_atom[MZ_MAXA], s_wpos[MZ_MAXA + 1], s_sorted[MZ_MAXA], s_sidx[MZ_MAXA];
  __shared__ double s_avir[MZ_MAXA], s_aov[MZ_MAXA], s_ws[4 * MZ_MAXA];
  __shared__ int s_eat[4 * MZ_MAXA];  // the rebuild's candidates (j, appended flag), per warp
  __shared__ double s_val[MZ_T];
  __shared__ int s_flag[MZ_T], s_scan[MZ_T];
  __shared__ long long s_base;
  __shared__ double s_sumt, s_tiny;
  const int i = blockIdx.x, tid = threadIdx.x;
  if (A.mode == 1 && A.stash_cap > 0 && A.nfmo[i] <= A.stash_cap) return;  // copied from the stash
  const MbMzLayout& L = A.L;
  const int nce = A.vir.ncf[i], nn = A.vir.nncf[i], loopi = A.vir.ncocc[i];
  if (nce > MZ_MAXA) {  // uniform over the CTA
    if (tid == 0) atomicExch(A.err, 1);
    return;
  }
  const int words = (L.numat + 31) >> 5;
  unsigned* lat = s_bits;
  unsigned* near1 = s_bits + words;
  unsigned* near2 = s_bits + 2 * words;
  for (int w = tid; w < 3 * words; w += MZ_T) s_bits[w] = 0u;
  __syncthreads();
  for (int t = tid; t < nce; t += MZ_T) s_atom[t] = A.vir.icocc[nn + t] - 1;
  __syncthreads();
  if (tid == 0) {
    int pos = 0;
    for (int t = 0; t < nce; ++t) {
      s_wpos[t] = pos;
      pos += L.iorbs[s_atom[t]];
    }
    s_wpos[nce] = pos;
    s_sumt = 0.0;
    s_tiny = 0.0;
  }
  // the sorted copy: each atom's place is the number of atoms before it in
  // order (ties by list position, which an LMO's distinct atoms never need)
  for (int t = tid; t < nce; t += MZ_T) {
    const int a = s_atom[t];
    int r = 0;
    for (int u = 0; u < nce; ++u) {
      const int b = s_atom[u];
      r += (b < a) || (b == a && u < t);
    }
    s_sorted[r] = a;
    s_sidx[r] = t;
  }
  __syncthreads();
  __syncthreads();
  for (int t = tid; t < nce; t += MZ_T) {
    const int a = s_atom[t];
    double sum = 0.0;
    for (int k = 0; k < L.iorbs[a]; ++k) {
      const double c = A.vir.cocc[loopi + s_wpos[t] + k];
      sum = DADD(sum, DMUL(c, c));
    }
    s_avir[t] = sum;
    atomicOr(&lat[a >> 5], 1u << (a & 31));
  }
  __syncthreads();
  // ws(orbital of atom j1, jx) = sum over the LMO's atoms k1 (in order) of
  // F(k1, j1) psi(k1).  One thread per atom j1: its orbitals share every
  // pair lookup and density test, and each orbital's sum keeps the k1 order.
  for (int jjl = tid; jjl < nce; jjl += MZ_T) {
    const int j1 = s_atom[jjl];
    const int nj = L.iorbs[j1];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int kk = 0; kk < nce; ++kk) {
      const int k1 = s_atom[kk];
      const long long kj = pair_offset(L, k1, j1);
      if (kj < 0 || !(DMUL(s_avir[kk], A.p[kj]) > A.cutoff)) continue;
      const int nk = L.iorbs[k1];
      const double* cv = A.vir.cocc + loopi + s_wpos[kk];
      for (int jx = 1; jx <= nj; ++jx)
        for (int i4 = 1; i4 <= nk; ++i4) {
          long long ii;
          if (nk == 1 && nj == 1) ii = kj + 1;
          else if (k1 > j1) ii = kj + (long long)(i4 - 1) * nj + jx;
          else if (k1 < j1) ii = kj + (long long)(jx - 1) * nk + i4;
          else ii = i4 > jx ? kj + (i4 * (i4 - 1)) / 2 + jx : kj + (jx * (jx - 1)) / 2 + i4;
          acc[jx - 1] = DADD(acc[jx - 1], DMUL(A.fao[ii - 1], cv[i4 - 1]));
        }
    }
    for (int jx = 0; jx < nj; ++jx) s_ws[s_wpos[jjl] + jx] = acc[jx];
  }
  __syncthreads();
  for (int t = tid; t < nce; t += MZ_T) {
    double sum = 0.0;
    for (int k = 0; k < L.iorbs[s_atom[t]]; ++k) sum = DADD(sum, DMUL(s_ws[s_wpos[t] + k], s_ws[s_wpos[t] + k]));
    s_aov[t] = sum;
  }
  __syncthreads();
  if (tid == 0) {  // eigv(i)
    double sum = 0.0;
    for (int kk = 0; kk < nce; ++kk) {
      if (!(DMUL(s_aov[kk], s_avir[kk]) > A.cutoff)) continue;
      for (int k = 0; k < L.iorbs[s_atom[kk]]; ++k)
        sum = DADD(sum, DMUL(s_ws[s_wpos[kk] + k], A.vir.cocc[loopi + s_wpos[kk] + k]));
    }
    A.eigv[i] = sum;
  }
  if (A.mode == 2) {
    // recompute on the previous list: entries of LMO i at list_off[i] ..
    const long long b0 = A.list_off[i];
    const int cnt = A.nfmo[i];
    double lmax = 0.0;
    for (int q = tid; q < cnt; q += MZ_T) {
      const int j = A.ifmo[2 * (b0 + q) + 1] - 1;
      bool lij;
      const double v = mzd_fmo(A, j, lat, s_sorted, s_sidx, nce, s_aov, s_wpos, s_ws, &lij);
      A.fmo[b0 + q] = v;
      lmax = fmax(lmax, fabs(v));
    }
    // |fmo| in list order for sumt, and the maximum
    for (int q0 = 0; q0 < cnt; q0 += MZ_T) {
      __syncthreads();
      const int q = q0 + tid;
      s_val[tid] = q < cnt ? fabs(A.fmo[b0 + q]) : 0.0;
      __syncthreads();
      if (tid == 0) {
        const int m = min(MZ_T, cnt - q0);
        for (int t = 0; t < m; ++t) s_sumt = DADD(s_sumt, s_val[t]);
      }
    }
    if (lmax > 0.0) atomicMax(A.tiny_bits, (unsigned long long)__double_as_longlong(lmax));
    __syncthreads();
    if (tid == 0) A.sumt_part[i] = s_sumt;
    return;
  }
  // rebuild: candidate occupied LMOs j in ascending order
  const int i1 = s_atom[0], i2 = nce > 1 ? s_atom[1] : s_atom[0];
  for (int q = L.nbr_ptr[i1] + tid; q < L.nbr_ptr[i1 + 1]; q += MZ_T) atomicOr(&near1[L.nbr_atom[q] >> 5], 1u << (L.nbr_atom[q] & 31));
  for (int q = L.nbr_ptr[i2] + tid; q < L.nbr_ptr[i2 + 1]; q += MZ_T) atomicOr(&near2[L.nbr_atom[q] >> 5], 1u << (L.nbr_atom[q] & 31));
  if (tid == 0) {
    atomicOr(&near1[i1 >> 5], 1u << (i1 & 31));
    atomicOr(&near2[i2 >> 5], 1u << (i2 & 31));
    s_base = A.mode == 1 ? A.list_off[i] : 0;
  }
  __syncthreads();
  int count = 0;
  const int nocc = A.occ.nlmo;
  // Candidate j of virtual LMO i: evaluated (ev) when its first two atoms see
  // i's first two within the neighbour lists and the F elements between them
  // reach flim; appended (app) when fmo(i, j) also clears oldlim.
  auto candidate = [&](int j, int& ev, int& app, double& val) {
    ev = 0;
    app = 0;
    val = 0.0;
    if (j >= nocc) return;
    const int j1 = A.occ.icocc[A.occ.nncf[j]] - 1;
    const int j2 = A.occ.ncf[j] > 1 ? A.occ.icocc[A.occ.nncf[j] + 1] - 1 : j1;
    const bool b11 = bit_test(near1, j1), b12 = bit_test(near1, j2), b21 = bit_test(near2, j1),
               b22 = bit_test(near2, j2);
    if (!(b11 || b12 || b21 || b22)) return;
    double s = 0.0;
    if (b11) s = fabs(A.fao[pair_offset(L, i1, j1)]);
    if (b12) s = DADD(s, fabs(A.fao[pair_offset(L, i1, j2)]));
    if (b21) s = DADD(s, fabs(A.fao[pair_offset(L, i2, j1)]));
    if (b22) s = DADD(s, fabs(A.fao[pair_offset(L, i2, j2)]));
    if (s >= A.flim) {
      bool lij;
      val = mzd_fmo(A, j, lat, s_sorted, s_sidx, nce, s_aov, s_wpos, s_ws, &lij);
      ev = 1;
      app = (lij && fabs(val) > A.oldlim) ? 1 : 0;
    }
  };
  // Fast path: each warp scans a contiguous quarter of the occupied LMOs and
  // compacts its evaluated candidates, in j order, into shared memory; one
  // barrier, then thread 0 folds them all in
  // j order and ranks the appended ones.  A warp with more than kCand
  // candidates sends the CTA to the chunked loop below.
  static_assert(MZ_T == 128 && 4 * MZD_CAND <= 4 * MZ_MAXA, "four warps share s_eat");
  constexpr int kCand = MZD_CAND;
  double* s_cv = (double*)(s_bits + mzd_bits_words(L.numat));  // 4 * kCand values after the bitmaps
  __shared__ int s_cn[4];
  {
    const int lane = tid & 31, wid = tid >> 5;
    int* cj = s_eat + wid * kCand;  // j + 1, negated when appended
    double* cv = s_cv + wid * kCand;
    const int per = (nocc + 3) / 4, jb = wid * per, je = min(nocc, jb + per);
    int nc = 0;
    for (int j0 = jb; j0 < je; j0 += 32) {
      int ev, app;
      double val;
      candidate(j0 + lane < je ? j0 + lane : nocc, ev, app, val);
      const unsigned evm = __ballot_sync(0xffffffffu, ev);
      const int pos = nc + __popc(evm & ((1u << lane) - 1u));
      if (ev && pos < kCand) {
        cj[pos] = app ? -(j0 + lane + 1) : (j0 + lane + 1);
        cv[pos] = val;
      }
      nc += __popc(evm);
    }
    if (lane == 0) s_cn[wid] = nc;
  }
  __syncthreads();
  if (s_cn[0] <= kCand && s_cn[1] <= kCand && s_cn[2] <= kCand && s_cn[3] <= kCand) {
    if (tid == 0) {  // the ordered fold, and the appended entries in j order
      long long pos = s_base;
      int run = 0;
      for (int w = 0; w < 4; ++w)
        for (int q = 0; q < s_cn[w]; ++q) {
          const double v = s_cv[w * kCand + q];
          s_sumt = DADD(s_sumt, fabs(v));
          s_tiny = fmax(s_tiny, fabs(v));
          const int cj = s_eat[w * kCand + q];
          if (cj < 0) {
            if (A.mode == 1) {
              A.ifmo[2 * pos] = i + 1;
              A.ifmo[2 * pos + 1] = -cj;
              A.fmo[pos] = v;
              ++pos;
            } else if (run < A.stash_cap) {
              A.stash_j[(long long)i * A.stash_cap + run] = -cj;
              A.stash_v[(long long)i * A.stash_cap + run] = v;
            }
            ++run;
          }
        }
      s_scan[0] = run;
    }
    __syncthreads();
    count = s_scan[0];
  } else {
    for (int j0 = 0; j0 < nocc; j0 += MZ_T) {
      const int j = j0 + tid;
      int app, ev;
      double val;
      candidate(j, ev, app, val);
      // evaluated and appended entries of this chunk as warp masks: the
      // ordered fold visits only the evaluated ones, in j order
      const int lane = tid & 31, wid = tid >> 5;
      const unsigned evm = __ballot_sync(0xffffffffu, ev), apm = __ballot_sync(0xffffffffu, app);
      __syncthreads();
      s_val[tid] = fabs(val);
      if (lane == 0) { s_flag[wid] = (int)evm; s_scan[wid] = (int)apm; }
      __syncthreads();
      if (tid == 0) {  // ordered fold of |fmo| for sumt, max for tiny
        for (int w = 0; w < MZ_T / 32; ++w)
          for (unsigned m = (unsigned)s_flag[w]; m; m &= m - 1) {
            const double v = s_val[32 * w + __ffs((int)m) - 1];
            s_sumt = DADD(s_sumt, v);
            s_tiny = fmax(s_tiny, v);
          }
      }
      int before = __popc(apm & ((1u << lane) - 1u)), total = 0;
      for (int w = 0; w < MZ_T / 32; ++w) {
        const int c = __popc((unsigned)s_scan[w]);
        if (w < wid) before += c;
        total += c;
      }
      if (A.mode == 1 && app) {
        const long long pos = s_base + count + before;
        A.ifmo[2 * pos] = i + 1;
        A.ifmo[2 * pos + 1] = j + 1;
        A.fmo[pos] = val;
      } else if (A.mode == 0 && app && count + before < A.stash_cap) {
        A.stash_j[(long long)i * A.stash_cap + count + before] = j + 1;
        A.stash_v[(long long)i * A.stash_cap + count + before] = val;
      }
      count += total;
      __syncthreads();
    }
  }
  __syncthreads();
  if (tid == 0) {
    if (A.mode == 0) A.nfmo[i] = count;
    A.sumt_part[i] = s_sumt;
    if (s_tiny > 0.0) atomicMax(A.tiny_bits, (unsigned long long)__double_as_longlong(s_tiny));
  }
}

// Occupied LMO energies psi^T F psi with the reference's cutoff (one thread per LMO).
__global__ void mzd_occ_energy(MbMzLayout L, MbMzLmos Q, const double* __restrict__ fao, const double* __restrict__ p,
                               const double* __restrict__ aocc, double cutoff, double* __restrict__ eigs) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < Q.nlmo; i += gridDim.x * blockDim.x) {
    const int loopi = Q.ncocc[i], nn = Q.nncf[i], nc = Q.ncf[i];
    double sum = 0.0;
    int jl = loopi;
    for (int j = nn; j < nn + nc; ++j) {
      const int j1 = Q.icocc[j] - 1;
      const int nj = L.iorbs[j1];
      int kl = loopi;
      for (int k = nn; k < nn + nc; ++k) {
        const int k1 = Q.icocc[k] - 1;
        const int nk = L.iorbs[k1];
        const long long k1j1 = pair_offset(L, k1, j1);
        // avir(k1) of this LMO equals aocc of k1's entry
        if (k1j1 >= 0 && DMUL(DMUL(aocc[k], p[k1j1]), aocc[k]) >= cutoff) {
          for (int jx = 1; jx <= nj; ++jx) {
            double sum1 = 0.0;
            if (k1 > j1) {
              for (int i4 = 1; i4 <= nk; ++i4)
                sum1 = DADD(sum1, DMUL(fao[k1j1 + (long long)(i4 - 1) * nj + jx - 1], Q.cocc[kl + i4 - 1]));
            } else if (k1 < j1) {
              for (int i4 = 1; i4 <= nk; ++i4)
                sum1 = DADD(sum1, DMUL(fao[k1j1 + (long long)(jx - 1) * nk + i4 - 1], Q.cocc[kl + i4 - 1]));
            } else {
              for (int j4 = 1; j4 <= jx; ++j4)
                sum1 = DADD(sum1, DMUL(fao[k1j1 + (jx * (jx - 1)) / 2 + j4 - 1], Q.cocc[kl + j4 - 1]));
              for (int i4 = jx + 1; i4 <= nk; ++i4)
                sum1 = DADD(sum1, DMUL(fao[k1j1 + (i4 * (i4 - 1)) / 2 + jx - 1], Q.cocc[kl + i4 - 1]));
            }
            sum = DADD(sum, DMUL(Q.cocc[jl + jx - 1], sum1));
          }
        }
        kl += nk;
      }
      jl += nj;
    }
    eigs[i] = sum;
  }
}

inline size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

extern "C" size_t mb_mz_diagg1_ws_bytes(const MbMzLayout* L, const MbMzLmos* occ, const MbMzLmos* vir) {
  if (!L || !occ || !vir) return 0;
  return al256(sizeof(double) * (size_t)(occ->nentries + 1)) + al256(sizeof(double) * (size_t)(vir->nlmo + 1)) +
         al256(sizeof(long long) * (size_t)(vir->nlmo + 1)) + al256(sizeof(unsigned long long)) + al256(sizeof(int)) +
         256;
}

namespace {
// The write pass for stashed LMOs: entries of virtual LMO i (count pass, j
// order) into the list at list_off[i].
__global__ void mzd_copy_stash(int nvir, const int* __restrict__ nfmo, const long long* __restrict__ list_off,
                               const int* __restrict__ sj, const double* __restrict__ sv, int stash_cap,
                               int* __restrict__ ifmo, double* __restrict__ fmo) {
  const int i = blockIdx.x;
  if (i >= nvir) return;
  const int n = nfmo[i];
  if (n > stash_cap) return;
  const long long b = list_off[i];
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    ifmo[2 * (b + k)] = i + 1;
    ifmo[2 * (b + k) + 1] = sj[(long long)i * stash_cap + k];
    fmo[b + k] = sv[(long long)i * stash_cap + k];
  }
}
}  // namespace

extern "C" int mb_mz_diagg1_dev(const MbMzLayout* L, const MbMzLmos* occ, const MbMzLmos* vir, const double* fao,
                                const double* p, int idiagg, double* state, int* nfmo, int* ifmo, double* fmo,
                                long long* nij, double* eigv, double* eigs, int* eigs_done, double* sumt, void* ws,
                                cudaStream_t stream) {
  if (!L || !occ || !vir || !fao || !p || !state || !nfmo || !ifmo || !fmo || !nij || !eigv || !eigs || !eigs_done ||
      !sumt || !ws)
    return mb_set_error(MB_ERR_ARG, "mb_mz_diagg1_dev: bad args");
  const int nvir = vir->nlmo;
  double fref = state[0], safety = state[1], oldlim = state[2], tiny = state[3];
  const long long cap = *nij;
  char* b = (char*)ws;
  double* aocc = (double*)b; b += al256(sizeof(double) * (size_t)(occ->nentries + 1));
  double* sumt_part = (double*)b; b += al256(sizeof(double) * (size_t)(nvir + 1));
  long long* list_off = (long long*)b; b += al256(sizeof(long long) * (size_t)(nvir + 1));
  unsigned long long* tiny_bits = (unsigned long long*)b; b += al256(sizeof(unsigned long long));
  int* err = (int*)b;
  // scalars as the reference sets them on entry (diagg1.F90:85-94)
  const double cutlim = 1.0e-8;
  double cutoff = cutlim > tiny * 10.0 * cutlim ? cutlim : tiny * 10.0 * cutlim;
  const double flim = 3.0 < fref * 0.5 ? 3.0 : fref * 0.5;
  fref = 0.0;
  if (idiagg <= 5) cutoff = cutlim;
  MB_CUDA(cudaMemsetAsync(tiny_bits, 0, sizeof(unsigned long long), stream));
  MB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), stream));
  mzd_aocc<<<(occ->nlmo + 127) / 128, 128, 0, stream>>>(*occ, L->iorbs, aocc);
  MB_LAUNCH_CHECK();
  DiagArgs A;
  A.L = *L;
  A.occ = *occ;
  A.vir = *vir;
  A.fao = fao;
  A.p = p;
  A.aocc = aocc;
  A.cutoff = cutoff;
  A.flim = flim;
  A.oldlim = oldlim;
  A.list_off = list_off;
  A.nfmo = nfmo;
  A.stash_j = nullptr;
  A.stash_v = nullptr;
  A.stash_cap = 0;
  A.ifmo = ifmo;
  A.fmo = fmo;
  A.eigv = eigv;
  A.sumt_part = sumt_part;
  A.tiny_bits = tiny_bits;
  A.err = err;
  const size_t smem = sizeof(unsigned) * (size_t)mzd_bits_words(L->numat) + sizeof(double) * 4 * MZD_CAND;
  if (smem > 160 * 1024) return mb_set_error(MB_ERR_UNSUPPORTED, "mb_mz_diagg1_dev: too many atoms for the bitmaps");
  static bool attr = false;
  if (!attr) {
    MB_CUDA(cudaFuncSetAttribute(mzd_virtual, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    attr = true;
  }
  const bool rebuild = idiagg <= 5 || idiagg % 2 == 0;
  std::vector<int> cnt(nvir);
  std::vector<long long> off(nvir + 1, 0);
  long long total = 0;
  if (rebuild) {
    // the count pass also keeps each LMO's appended entries (up to stash_cap,
    // at most 512 MB in all); the write pass then copies them and recomputes
    // only the LMOs that had more
    const int stash_cap = (int)std::min<long long>(1024, (512ll << 20) / (12ll * std::max(nvir, 1)));
    char* stash = nullptr;
    if (stash_cap >= 16) {
      MB_CUDA(mb_malloc_async((void**)&stash, (size_t)nvir * stash_cap * 12, stream));
      A.stash_v = (double*)stash;
      A.stash_j = (int*)(stash + (size_t)nvir * stash_cap * 8);
      A.stash_cap = stash_cap;
    }
    A.mode = 0;
    mzd_virtual<<<nvir, MZ_T, smem, stream>>>(A);
    MB_LAUNCH_CHECK();
    MB_CUDA(cudaMemcpyAsync(cnt.data(), nfmo, sizeof(int) * nvir, cudaMemcpyDeviceToHost, stream));
    MB_CUDA(cudaStreamSynchronize(stream));
    bool over = false;
    for (int i = 0; i < nvir; ++i) {
      off[i + 1] = off[i] + cnt[i];
      over = over || cnt[i] > A.stash_cap;
    }
    total = off[nvir];
    if (total > cap) {
      if (stash) cudaFreeAsync(stash, stream);
      return mb_set_error(MB_ERR_UNSUPPORTED, "mb_mz_diagg1_dev: interaction list exceeds its capacity");
    }
    MB_CUDA(cudaMemcpyAsync(list_off, off.data(), sizeof(long long) * nvir, cudaMemcpyHostToDevice, stream));
    if (A.stash_cap > 0) {
      mzd_copy_stash<<<nvir, 128, 0, stream>>>(nvir, nfmo, list_off, A.stash_j, A.stash_v, A.stash_cap, ifmo, fmo);
      MB_LAUNCH_CHECK();
    }
    if (over) {  // recomputes the same values, sums and maxima for the LMOs past the stash
      A.mode = 1;
      mzd_virtual<<<nvir, MZ_T, smem, stream>>>(A);
      MB_LAUNCH_CHECK();
    }
    if (stash) MB_CUDA(cudaFreeAsync(stash, stream));
  } else {
    MB_CUDA(cudaMemcpyAsync(cnt.data(), nfmo, sizeof(int) * nvir, cudaMemcpyDeviceToHost, stream));
    MB_CUDA(cudaStreamSynchronize(stream));
    for (int i = 0; i < nvir; ++i) off[i + 1] = off[i] + cnt[i];
    total = off[nvir] < cap ? off[nvir] : cap;
    MB_CUDA(cudaMemcpyAsync(list_off, off.data(), sizeof(long long) * nvir, cudaMemcpyHostToDevice, stream));
    A.mode = 2;
    mzd_virtual<<<nvir, MZ_T, smem, stream>>>(A);
    MB_LAUNCH_CHECK();
  }
  std::vector<double> sp(nvir);
  unsigned long long tb = 0;
  int herr = 0;
  MB_CUDA(cudaMemcpyAsync(sp.data(), sumt_part, sizeof(double) * nvir, cudaMemcpyDeviceToHost, stream));
  MB_CUDA(cudaMemcpyAsync(&tb, tiny_bits, sizeof(tb), cudaMemcpyDeviceToHost, stream));
  MB_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, stream));
  MB_CUDA(cudaStreamSynchronize(stream));
  if (herr) return mb_set_error(MB_ERR_UNSUPPORTED, "mb_mz_diagg1_dev: a virtual LMO covers more than 512 atoms");
  double st = 0.0;
  for (int i = 0; i < nvir; ++i) st += sp[i];
  *sumt = st;
  double tnew;
  memcpy(&tnew, &tb, sizeof(tnew));
  tiny = tnew;
  const long long ijc = total;
  if (ijc == cap) safety = safety * 2.0;
  else safety = safety * 0.5 > 1.0 ? safety * 0.5 : 1.0;
  *nij = ijc;
  *eigs_done = 0;
  if (idiagg > 2 && idiagg % 4 != 0) {
    const double t2 = tiny * tiny;
    fref = t2 * t2;
  } else {
    mzd_occ_energy<<<(occ->nlmo + 127) / 128, 128, 0, stream>>>(*L, *occ, fao, p, aocc, cutoff, eigs);
    MB_LAUNCH_CHECK();
    oldlim = tiny * safety * 1.0e-3;
    const double t2 = tiny * tiny;
    fref = t2 * t2;
    *eigs_done = 1;
  }
  state[0] = fref;
  state[1] = safety;
  state[2] = oldlim;
  state[3] = tiny;
  return MB_OK;
}

// ------------------------------------------------------------------ diagg2
namespace {

struct D2Args {
  MbMzLmos occ, vir;
  const int* iorbs;
  const int* ifmo;
  const double* fmo;
  const double* eigs;
  const double* eigv;
  const long long* order;
  long long lo, hi;
  double cst, shift, thresh, tiny, biglim;
  int retry, nocc, nvir, norbs;
  double* beta_sum;
  int* rej;
};

// Offset of atom a's coefficients in LMO q's block (atoms nn .. nn+cnt), or -1.
__device__ __forceinline__ int find_atom(const int* ic, int nn, int cnt, const int* iorbs, int a) {
  int off = 0;
  for (int t = nn; t < nn + cnt; ++t) {
    const int b = ic[t] - 1;
    if (b == a) return off;
    off += iorbs[b];
  }
  return -1;
}

// Whether a rotation is rejected depends only on coefficients it has not yet
// touched (those of atoms in one LMO only), so a dry run decides it first;
// modifying and then restoring, as the reference does, leaves the same
// coefficients as not modifying.  The atom numbers it appends before a
// rejection stay in the LMOs' spare slots in the reference (it restores the
// counts, not the slots); the dry run writes them too.
// ---------------------------------------------------------- warp per rotation
// diagg2's 2x2 rotation (diagg2.F90:180-345), one warp per rotation: the atom lists of
// the two LMOs are walked 32 atoms at a time, one lane per atom, and what the
// sequential loop carries from atom to atom -- the running coefficient offset,
// the number of atoms appended so far and their coefficient count -- is a
// warp prefix sum, so every lane knows where its atom's coefficients sit and
// where an appended atom goes.  Membership ("is atom a in the other LMO, and
// at which offset") goes through a per-warp hash map in shared memory.  Each
// atom's own arithmetic (its squared-sum test over its orbitals, its 2x2
// rotations) is the sequential loop's, in the same order, and atoms touch
// disjoint coefficients, so the result is bit for bit the sequential loop's.  An
// overflow check fails first at the same atom as in the sequential loop:
// the running totals only grow.
constexpr int WMAP = 1024;            // slots per map; at most WMAP / 2 atoms mapped
constexpr int D2W = 4;                // warps (rotations) per CTA
constexpr unsigned FULLW = 0xffffffffu;
constexpr size_t D2_SMEM = sizeof(int) * 4 * WMAP * D2W;  // two maps (keys, values) per warp

struct WMap {
  int* key;
  int* val;
  bool ok;
};

__device__ __forceinline__ unsigned wmap_hash(int a) { return ((unsigned)a * 2654435761u) & (WMAP - 1); }

// Inclusive warp scan of x.
__device__ __forceinline__ long long warp_scan(long long x, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(FULLW, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// Map atom -> coefficient offset over the first cnt atoms of a list; returns
// the list's total coefficient count.
__device__ long long wmap_build(WMap& m, const int* ic, int nn, int cnt, const int* iorbs, int lane) {
  m.ok = cnt <= WMAP / 2;
  if (m.ok)
    for (int q = lane; q < WMAP; q += 32) { m.key[q] = -1; m.val[q] = 0x7fffffff; }
  __syncwarp();
  long long carry = 0;
  for (int base = 0; base < cnt; base += 32) {
    const int t = base + lane;
    int b = -1, no = 0;
    if (t < cnt) { b = ic[nn + t] - 1; no = iorbs[b]; }
    const long long inc = warp_scan(no, lane);
    const long long off = carry + inc - no;
    if (m.ok && t < cnt) {
      unsigned h = wmap_hash(b);
      for (;;) {
        const int prev = atomicCAS(&m.key[h], -1, b);
        if (prev == -1 || prev == b) break;
        h = (h + 1) & (WMAP - 1);
      }
      atomicMin(&m.val[h], (int)off);  // a repeated atom keeps its first slot
    }
    carry += __shfl_sync(FULLW, inc, 31);
  }
  __syncwarp();
  return carry;
}

__device__ __forceinline__ int wmap_find(const WMap& m, int a, const int* ic, int nn, int cnt, const int* iorbs) {
  if (m.ok) {
    unsigned h = wmap_hash(a);
    while (m.key[h] >= 0) {
      if (m.key[h] == a) return m.val[h];
      h = (h + 1) & (WMAP - 1);
    }
    return -1;
  }
  return find_atom(ic, nn, cnt, iorbs, a);
}

__global__ void __launch_bounds__(32 * D2W) mzd2_level_warp(D2Args A) {
  extern __shared__ int d2_smem[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long q = A.lo + (long long)blockIdx.x * D2W + wid;
  if (q >= A.hi) return;  // whole warp
  WMap mj, mi;
  mj.key = d2_smem + wid * 4 * WMAP;
  mj.val = mj.key + WMAP;
  mi.key = mj.val + WMAP;
  mi.val = mi.key + WMAP;
  const long long e = A.order[q];
  const int i = A.ifmo[2 * e] - 1, j = A.ifmo[2 * e + 1] - 1;
  const double fm = A.fmo[e];
  if (!(fabs(fm) >= A.tiny)) {
    if (lane == 0) { A.beta_sum[e] = 0.0; A.rej[e] = 0; }
    return;
  }
  const double c = DMUL(fm, A.cst);
  const double d = DSUB(DSUB(A.eigs[j], A.eigv[i]), A.shift);
  if (!(fabs(c / d) >= A.biglim)) {
    if (lane == 0) { A.beta_sum[e] = 0.0; A.rej[e] = 0; }
    return;
  }
  int* ncf = const_cast<int*>(A.occ.ncf);
  int* icocc = const_cast<int*>(A.occ.icocc);
  double* cocc = const_cast<double*>(A.occ.cocc);
  int* nce = const_cast<int*>(A.vir.ncf);
  int* icvir = const_cast<int*>(A.vir.icocc);
  double* cvir = const_cast<double*>(A.vir.cocc);
  const int* nncf = A.occ.nncf;
  const int* nnce = A.vir.nncf;
  const long long loopj = A.occ.ncocc[j], loopi = A.vir.ncocc[i];
  const long long jlr = loopj + 1, ilr = loopi + 1;
  long long jur = (j != A.nocc - 1) ? A.occ.ncocc[j + 1] : A.occ.ncoeff;
  const long long jncf = (j != A.nocc - 1) ? nncf[j + 1] : A.occ.nentries;
  long long iur = (i != A.nvir - 1) ? A.vir.ncocc[i + 1] : A.vir.ncoeff;
  const long long incv = (i != A.nvir - 1) ? nnce[i + 1] : A.vir.nentries;
  jur = jlr + A.norbs - 1 < jur ? jlr + A.norbs - 1 : jur;
  iur = ilr + A.norbs - 1 < iur ? ilr + A.norbs - 1 : iur;
  const int ncf0 = ncf[j], nce0 = nce[i];
  const int nnj = nncf[j], nni = nnce[i];
  const long long mlf0 = wmap_build(mj, icocc, nnj, ncf0, A.iorbs, lane);  // coefficients of LMO j
  const long long mle0 = wmap_build(mi, icvir, nni, nce0, A.iorbs, lane);  // coefficients of LMO i
  const double ee = copysign(sqrt(DADD(DMUL(DMUL(4.0, c), c), DMUL(d, d))), d);
  double alpha = sqrt(DMUL(0.5, DADD(1.0, d / ee)));
  double bs = 0.0;
  int rj = 0;
  const unsigned lt = (1u << lane) - 1u;
  double beta = 0.0;
  for (;;) {
    beta = -copysign(sqrt(DSUB(1.0, DMUL(alpha, alpha))), c);
    bs = DADD(bs, fabs(beta));
    // ---- dry run 1: atoms of LMO i that would join LMO j
    bool rejected = false;
    {
      long long nfj = ncf0, mlf = mlf0, moff = 0;
      for (int base = 0; base < nce0 && !rejected; base += 32) {
        const int t = base + lane;
        int mie = -1, no = 0;
        if (t < nce0) { mie = icvir[nni + t] - 1; no = A.iorbs[mie]; }
        const long long inc = warp_scan(no, lane);
        const long long off = moff + inc - no;
        bool cand = false;
        if (t < nce0 && wmap_find(mj, mie, icocc, nnj, ncf0, A.iorbs) < 0) {
          double sum = 0.0;
          for (int k = 0; k < no; ++k) {
            const double tt = DMUL(beta, cvir[loopi + off + k]);
            sum = DADD(sum, DMUL(tt, tt));
          }
          cand = sum > A.thresh;
        }
        const unsigned bal = __ballot_sync(FULLW, cand);
        const long long cno = warp_scan(cand ? no : 0, lane);
        const long long pos_n = nfj + __popc(bal & lt), pos_m = mlf + cno - (cand ? no : 0);
        const bool over = cand && (nnj + pos_n >= jncf || pos_m + no + loopj > jur);
        const unsigned ob = __ballot_sync(FULLW, over);
        const int first = ob ? __ffs(ob) - 1 : 32;
        if (cand && lane < first) icocc[nnj + pos_n] = mie + 1;  // as the reference leaves them
        if (ob) rejected = true;
        nfj += __popc(bal);
        mlf += __shfl_sync(FULLW, cno, 31);
        moff += __shfl_sync(FULLW, inc, 31);
      }
    }
    // ---- dry run 2: atoms of LMO j that would join LMO i
    if (!rejected) {
      long long nfi = nce0, mle = mle0, joff = 0;
      for (int base = 0; base < ncf0 && !rejected; base += 32) {
        const int t = base + lane;
        int ii = -1, no = 0;
        if (t < ncf0) { ii = icocc[nnj + t] - 1; no = A.iorbs[ii]; }
        const long long inc = warp_scan(no, lane);
        const long long off = joff + inc - no;
        bool cand = false;
        if (t < ncf0 && wmap_find(mi, ii, icvir, nni, nce0, A.iorbs) < 0) {
          double sum = 0.0;
          for (int k = 0; k < no; ++k) {
            const double tt = DMUL(beta, cocc[loopj + off + k]);
            sum = DADD(sum, DMUL(tt, tt));
          }
          cand = sum > A.thresh;
        }
        const unsigned bal = __ballot_sync(FULLW, cand);
        const long long cno = warp_scan(cand ? no : 0, lane);
        const long long pos_n = nfi + __popc(bal & lt), pos_m = mle + cno - (cand ? no : 0);
        const bool over = cand && (nni + pos_n >= incv || pos_m + no + loopi > iur);
        const unsigned ob = __ballot_sync(FULLW, over);
        const int first = ob ? __ffs(ob) - 1 : 32;
        if (cand && lane < first) icvir[nni + pos_n] = ii + 1;
        if (ob) rejected = true;
        nfi += __popc(bal);
        mle += __shfl_sync(FULLW, cno, 31);
        joff += __shfl_sync(FULLW, inc, 31);
      }
    }
    if (rejected) {
      ++rj;
      if (A.retry) { alpha = DMUL(0.5, DADD(alpha, 1.0)); continue; }
      break;
    }
    // ---- apply 1: LMO i's atoms -- rotate the shared ones, append the rest to j
    int addj = 0;
    {
      long long mlf = mlf0, moff = 0;
      for (int base = 0; base < nce0; base += 32) {
        const int t = base + lane;
        int mie = -1, no = 0;
        if (t < nce0) { mie = icvir[nni + t] - 1; no = A.iorbs[mie]; }
        const long long inc = warp_scan(no, lane);
        const long long off = moff + inc - no;
        const int uj = t < nce0 ? wmap_find(mj, mie, icocc, nnj, ncf0, A.iorbs) : 0;
        bool cand = false;
        if (t < nce0 && uj >= 0) {
          for (int k = 0; k < no; ++k) {
            const long long pj = loopj + uj + k, pi = loopi + off + k;
            const double a = cocc[pj], b = cvir[pi];
            cocc[pj] = DADD(DMUL(alpha, a), DMUL(beta, b));
            cvir[pi] = DSUB(DMUL(alpha, b), DMUL(beta, a));
          }
        } else if (t < nce0) {
          double sum = 0.0;
          for (int k = 0; k < no; ++k) {
            const double tt = DMUL(beta, cvir[loopi + off + k]);
            sum = DADD(sum, DMUL(tt, tt));
          }
          cand = sum > A.thresh;
        }
        const unsigned bal = __ballot_sync(FULLW, cand);
        const long long cno = warp_scan(cand ? no : 0, lane);
        if (cand) {
          const long long pos_m = mlf + cno - no;
          icocc[nnj + ncf0 + addj + __popc(bal & lt)] = mie + 1;
          for (int k = 0; k < no; ++k) {
            const long long pi = loopi + off + k;
            cocc[loopj + pos_m + k] = DMUL(beta, cvir[pi]);
            cvir[pi] = DMUL(alpha, cvir[pi]);
          }
        }
        addj += __popc(bal);
        mlf += __shfl_sync(FULLW, cno, 31);
        moff += __shfl_sync(FULLW, inc, 31);
      }
    }
    // ---- apply 2: LMO j's original atoms not in i join LMO i
    int addi = 0;
    {
      long long mle = mle0, joff = 0;
      for (int base = 0; base < ncf0; base += 32) {
        const int t = base + lane;
        int ii = -1, no = 0;
        if (t < ncf0) { ii = icocc[nnj + t] - 1; no = A.iorbs[ii]; }
        const long long inc = warp_scan(no, lane);
        const long long off = joff + inc - no;
        bool cand = false;
        if (t < ncf0 && wmap_find(mi, ii, icvir, nni, nce0, A.iorbs) < 0) {
          double sum = 0.0;
          for (int k = 0; k < no; ++k) {
            const double tt = DMUL(beta, cocc[loopj + off + k]);
            sum = DADD(sum, DMUL(tt, tt));
          }
          cand = sum > A.thresh;
        }
        const unsigned bal = __ballot_sync(FULLW, cand);
        const long long cno = warp_scan(cand ? no : 0, lane);
        if (cand) {
          const long long pos_m = mle + cno - no;
          icvir[nni + nce0 + addi + __popc(bal & lt)] = ii + 1;
          for (int k = 0; k < no; ++k) {
            const long long pj = loopj + off + k;
            cvir[loopi + pos_m + k] = DMUL(-beta, cocc[pj]);
            cocc[pj] = DMUL(alpha, cocc[pj]);
          }
        }
        addi += __popc(bal);
        mle += __shfl_sync(FULLW, cno, 31);
        joff += __shfl_sync(FULLW, inc, 31);
      }
    }
    if (lane == 0) {
      ncf[j] = ncf0 + addj;
      nce[i] = nce0 + addi;
    }
    break;
  }
  if (lane == 0) {
    A.beta_sum[e] = bs;
    A.rej[e] = rj;
  }
}
}  // namespace

extern "C" int mb_mz_diagg2_dev(const MbMzLayout* L, MbMzLmos* occ, MbMzLmos* vir, const int* ifmo, const double* fmo,
                                long long nij, const double* eigs, const double* eigv, int idiagg, const double* ctl,
                                int* nrejct, double* sumb, long long* nrej, cudaStream_t stream) {
  if (!L || !occ || !vir || !ctl || !nrejct || !sumb || !nrej || nij < 0)
    return mb_set_error(MB_ERR_ARG, "mb_mz_diagg2_dev: bad args");
  *sumb = 0.0;
  *nrej = 0;
  const int retry = (nrejct[0] == nrejct[1] && nrejct[0] != 0 && nrejct[0] < 20);
  double tiny, biglim;
  if (idiagg % 5 == 0 || idiagg <= 5) {
    tiny = -1.0;
    biglim = -1.0;
  } else {
    tiny = 0.01 * ctl[3];
    biglim = ctl[4];
  }
  if (nij == 0) {
    nrejct[1] = nrejct[0];
    nrejct[0] = 0;
    return MB_OK;
  }
  // dependency levels: an entry follows the last earlier entry of its virtual and of its occupied LMO
  std::vector<int> hl(2 * (size_t)nij);
  MB_CUDA(cudaMemcpyAsync(hl.data(), ifmo, sizeof(int) * 2 * (size_t)nij, cudaMemcpyDeviceToHost, stream));
  MB_CUDA(cudaStreamSynchronize(stream));
  std::vector<int> lastv(vir->nlmo, 0), lasto(occ->nlmo, 0), lvl(nij);
  int nlev = 0;
  for (long long e = 0; e < nij; ++e) {
    const int i = hl[2 * e] - 1, j = hl[2 * e + 1] - 1;
    if (i < 0 || i >= vir->nlmo || j < 0 || j >= occ->nlmo) return mb_set_error(MB_ERR_ARG, "diagg2: bad list entry");
    const int lv = 1 + (lastv[i] > lasto[j] ? lastv[i] : lasto[j]);
    lastv[i] = lasto[j] = lv;
    lvl[e] = lv;
    if (lv > nlev) nlev = lv;
  }
  std::vector<long long> start(nlev + 2, 0), order(nij);
  for (long long e = 0; e < nij; ++e) start[lvl[e] + 1]++;
  for (int v = 1; v <= nlev + 1; ++v) start[v] += start[v - 1];
  {
    std::vector<long long> fill(start.begin(), start.end());
    for (long long e = 0; e < nij; ++e) order[fill[lvl[e]]++] = e;
  }
  long long* d_order = nullptr;
  double* d_bs = nullptr;
  int* d_rej = nullptr;
  MB_CUDA(mb_malloc_async((void**)&d_order, sizeof(long long) * nij, stream));
  MB_CUDA(mb_malloc_async((void**)&d_bs, sizeof(double) * nij, stream));
  MB_CUDA(mb_malloc_async((void**)&d_rej, sizeof(int) * nij, stream));
  int rc = MB_OK;
  if (cudaMemcpyAsync(d_order, order.data(), sizeof(long long) * nij, cudaMemcpyHostToDevice, stream) != cudaSuccess)
    rc = mb_set_error(MB_ERR_CUDA, "diagg2: upload");
  D2Args A;
  A.occ = *occ;
  A.vir = *vir;
  A.iorbs = L->iorbs;
  A.ifmo = ifmo;
  A.fmo = fmo;
  A.eigs = eigs;
  A.eigv = eigv;
  A.order = d_order;
  A.cst = ctl[0];
  A.shift = ctl[1];
  A.thresh = ctl[2];
  A.tiny = tiny;
  A.biglim = biglim;
  A.retry = retry;
  A.nocc = occ->nlmo;
  A.nvir = vir->nlmo;
  A.norbs = L->norbs;
  A.beta_sum = d_bs;
  A.rej = d_rej;
  static bool d2_attr = false;
  if (!d2_attr) {
    MB_CUDA(cudaFuncSetAttribute(mzd2_level_warp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D2_SMEM));
    d2_attr = true;
  }
  for (int v = 1; v <= nlev && rc == MB_OK; ++v) {
    A.lo = start[v];
    A.hi = start[v + 1];
    const long long cnt = A.hi - A.lo;
    if (cnt <= 0) continue;
    mzd2_level_warp<<<(unsigned)((cnt + D2W - 1) / D2W), 32 * D2W, D2_SMEM, stream>>>(A);
    mb_count_launch();
    if (cudaGetLastError() != cudaSuccess) rc = mb_set_error(MB_ERR_CUDA, "diagg2: launch");
  }
  std::vector<double> bs(nij);
  std::vector<int> rj(nij);
  if (rc == MB_OK && (cudaMemcpyAsync(bs.data(), d_bs, sizeof(double) * nij, cudaMemcpyDeviceToHost, stream) !=
                          cudaSuccess ||
                      cudaMemcpyAsync(rj.data(), d_rej, sizeof(int) * nij, cudaMemcpyDeviceToHost, stream) !=
                          cudaSuccess ||
                      cudaStreamSynchronize(stream) != cudaSuccess))
    rc = mb_set_error(MB_ERR_CUDA, "diagg2: results");
  cudaFreeAsync(d_order, stream);
  cudaFreeAsync(d_bs, stream);
  cudaFreeAsync(d_rej, stream);
  if (rc != MB_OK) return rc;
  double sb = 0.0;
  long long nr = 0;
  for (long long e = 0; e < nij; ++e) {
    sb += bs[e];
    nr += rj[e];
  }
  *sumb = sb;
  *nrej = nr;
  nrejct[1] = nrejct[0];
  nrejct[0] = (int)nr;
  return MB_OK;
}
