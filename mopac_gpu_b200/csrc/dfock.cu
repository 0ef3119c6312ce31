// dfock2 on the device: the two-centre Fock-matrix derivative of one atom
// (forces/dfock2.F90:16-279, the itype = 3 path, the only one the routine
// reaches; called from forces/deri1.F90:107 with f holding the one-electron
// derivatives).  For every partner jj != nati in ascending order the pair's
// block of the derivative integrals w (100, 10 or 1 values for heavy-heavy,
// heavy-light or light-light pairs, packed in partner order) adds jab's
// Coulomb terms (integrals/jab.F90) and kab's exchange terms
// (integrals/kab.F90), or the light-atom forms of both, to f.
//
// Bit-identical to the reference: every sum runs in its term order, the
// file is compiled without FMA contraction, and each element of f gets its
// additions in the reference's sequence.  A partner's own diagonal block
// and the (nati, jj) off-diagonal block receive one pair's terms only, so a
// thread per partner writes them directly; nati's diagonal block receives
// one term per partner, which the partners stage and one pass folds in
// partner order (a light nati takes two additions per heavy partner,
// f + 2 sumoff + sumdia, and one per light partner, staged beside a -0.0
// that leaves the sum unchanged bit for bit).
#include <vector>

#include "mb_common.cuh"

namespace {

__host__ __device__ constexpr int pair1(int a, int b) {  // 1-based index of orbital pair (a, b), 1..4
  return a > b ? a * (a - 1) / 2 + b : b * (b - 1) / 2 + a;
}
// jab's density gather, kab's term order and dfock2's jindex(1..16):
// term m (0-based) uses the pair (m / 4 + 1, m % 4 + 1)
__host__ __device__ constexpr int pidx(int m) { return pair1(m / 4 + 1, m % 4 + 1); }

// 0-based packed index of 1-based orbitals i, j
__device__ __forceinline__ long long ix(int i, int j) {
  const long long hi = i > j ? i : j, lo = i > j ? j : i;
  return hi * (hi - 1) / 2 + lo - 1;
}

struct DfArgs {
  int numat, nati;              // nati 1-based
  const int* first;             // 1-based first orbital per atom (device)
  const int* last;              // 1-based last orbital per atom (device)
  const long long* woff;        // w offset per atom (device; nati's unused)
  double* f;
  const double* ptot;
  const double* p;
  const double* w;
  double* stage;                // numat * 10 (heavy nati) or numat * 2 (light nati)
};

__global__ void dfock2_pairs(DfArgs a) {
  const int jj = blockIdx.x * blockDim.x + threadIdx.x + 1;  // 1-based partner
  if (jj > a.numat || jj == a.nati) return;
  const int ia = a.first[a.nati - 1], ib = a.last[a.nati - 1];
  const int ja = a.first[jj - 1], jb = a.last[jj - 1];
  const double* w = a.w + a.woff[jj - 1];
  double* f = a.f;
  const double* pt = a.ptot;
  const bool hi = ib - ia >= 3, hj = jb - ja >= 3;
  if (hi && hj) {
    // jab (dfock2.F90:79-82): pja, pjb the two diagonal blocks
    double pja[16], pjb[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      pja[m] = pt[ix(ia + m / 4, ia + m % 4)];
      pjb[m] = pt[ix(ja + m / 4, ja + m % 4)];
    }
    double* st = a.stage + (long long)(jj - 1) * 10;
    int i = 0;
    for (int i5 = 1; i5 <= 4; ++i5)
      for (int i6 = 1; i6 <= i5; ++i6, ++i) {
        const int r = i + 1;  // jab's 1-based element of the block
        double sa = pja[0] * w[10 * (pidx(0) - 1) + r - 1];
        double sb = pjb[0] * w[10 * (r - 1) + pidx(0) - 1];
#pragma unroll
        for (int m = 1; m < 16; ++m) {
          sa = sa + pja[m] * w[10 * (pidx(m) - 1) + r - 1];
          sb = sb + pjb[m] * w[10 * (r - 1) + pidx(m) - 1];
        }
        st[i] = sb;                                       // nati's block: folded in partner order
        const long long jo = ix(ja + i5 - 1, ja + i6 - 1);
        f[jo] = f[jo] + sa;
      }
    // kab (dfock2.F90:83-104): pk(4 (i - ia) + (j - ja)) = P(i, j)
    double pk[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) pk[m] = a.p[ix(ia + m / 4, ja + m % 4)];
    for (int x = 0; x < 4; ++x)
      for (int y = 0; y < 4; ++y) {
        double s = pk[0] * w[10 * (pair1(x + 1, 1) - 1) + pair1(y + 1, 1) - 1];
#pragma unroll
        for (int k = 1; k < 16; ++k)
          s = s + pk[k] * w[10 * (pair1(x + 1, k / 4 + 1) - 1) + pair1(y + 1, k % 4 + 1) - 1];
        const long long e = ix(ia + x, ja + y);
        f[e] = f[e] - s;
      }
  } else if (hi || hj) {
    // dfock2.F90:106-203: one heavy atom h0, one light atom l0
    const int h0 = hi ? ia : ja, l0 = hi ? ja : ia;
    const long long ll = ix(l0, l0);
    const double pll = pt[ll];
    double sumdia = 0.0, sumoff = 0.0;
    double* st = a.stage + (long long)(jj - 1) * (hi ? 10 : 2);
    int k = 0;
    for (int i = 0; i < 4; ++i) {
      for (int j = 0; j < i; ++j, ++k) {
        const long long j1 = ix(h0 + i, h0 + j);
        const double t = pll * w[k];
        if (hi) st[k] = t;
        else f[j1] = f[j1] + t;
        sumoff = sumoff + pt[j1] * w[k];
      }
      const long long j1 = ix(h0 + i, h0 + i);
      const double t = pll * w[k];
      if (hi) st[k] = t;
      else f[j1] = f[j1] + t;
      sumdia = sumdia + pt[j1] * w[k];
      ++k;
    }
    if (hi) {  // the light partner's diagonal: f + 2 sumoff + sumdia
      f[ll] = f[ll] + sumoff * 2.0 + sumdia;
    } else {   // nati's: staged as the two additions
      st[0] = sumoff * 2.0;
      st[1] = sumdia;
    }
    // exchange: f(h0 + i, l0) -= sum_j p(h0 + j, l0) w(jindex(4 i + j + 1))
    for (int i = 0; i < 4; ++i) {
      double s = 0.0;
      for (int j = 0; j < 4; ++j) s = s + a.p[ix(h0 + j, l0)] * w[pidx(4 * i + j) - 1];
      const long long e = ix(h0 + i, l0);
      f[e] = f[e] - s;
    }
  } else {
    // dfock2.F90:204-215: two light atoms
    const long long i1 = ix(ia, ia), j1 = ix(ja, ja), ij = ix(ia, ja);
    double* st = a.stage + (long long)(jj - 1) * 2;
    st[0] = pt[j1] * w[0];
    st[1] = -0.0;
    f[j1] = f[j1] + pt[i1] * w[0];
    f[ij] = f[ij] - a.p[ij] * w[0];
  }
}

// nati's diagonal block: thread r folds its element's staged terms in
// partner order.
__global__ void dfock2_fold(DfArgs a) {
  const int ia = a.first[a.nati - 1], ib = a.last[a.nati - 1];
  const bool hi = ib - ia >= 3;
  const int r = threadIdx.x;
  if (hi) {
    if (r >= 10) return;
    int i5 = 1;
    while (i5 * (i5 + 1) / 2 <= r) ++i5;
    const int i6 = r - (i5 - 1) * i5 / 2 + 1;
    const long long e = ix(ia + i5 - 1, ia + i6 - 1);
    double v = a.f[e];
    for (int jj = 1; jj <= a.numat; ++jj)
      if (jj != a.nati) v = v + a.stage[(long long)(jj - 1) * 10 + r];
    a.f[e] = v;
  } else {
    if (r != 0) return;
    const long long e = ix(ia, ia);
    double v = a.f[e];
    for (int jj = 1; jj <= a.numat; ++jj) {
      if (jj == a.nati) continue;
      v = v + a.stage[(long long)(jj - 1) * 2];
      v = v + a.stage[(long long)(jj - 1) * 2 + 1];
    }
    a.f[e] = v;
  }
}

}  // namespace

// Size of dfock2's w for atom nati (1-based): sum over partners of 100, 10
// or 1; -1 on bad arguments or d orbitals.
extern "C" long long mb_dfock2_w_len(int numat, const int* nfirst, const int* nlast, int nati) {
  if (numat <= 0 || !nfirst || !nlast || nati < 1 || nati > numat) return -1;
  long long kk = 0;
  const bool hi = nlast[nati - 1] - nfirst[nati - 1] >= 3;
  for (int jj = 1; jj <= numat; ++jj) {
    const int no = nlast[jj - 1] - nfirst[jj - 1];
    if (no >= 6 || no < 0) return -1;
    if (jj == nati) continue;
    const bool hj = no >= 3;
    kk += (hi && hj) ? 100 : ((hi || hj) ? 10 : 1);
  }
  return kk;
}

// dfock2 (forces/dfock2.F90) on device arrays: f (in/out), ptot, p packed
// (mpack), w of mb_dfock2_w_len values; nfirst, nlast host, 1-based.
extern "C" int mb_dfock2_dev(int numat, const int* nfirst, const int* nlast, int nati, double* f, const double* ptot,
                             const double* p, const double* w, cudaStream_t s) {
  if (mb_dfock2_w_len(numat, nfirst, nlast, nati) < 0 || !f || !ptot || !p || !w)
    return mb_set_error(MB_ERR_ARG, "mb_dfock2_dev: bad arguments or an atom with d orbitals");
  for (int a = 0; a < numat; ++a) {
    const int no = nlast[a] - nfirst[a] + 1;
    if (no != 1 && no != 4) return mb_set_error(MB_ERR_UNSUPPORTED, "mb_dfock2_dev: s or sp atoms only");
  }
  if (numat == 1) return MB_OK;
  std::vector<long long> off(numat, 0);
  const bool hi = nlast[nati - 1] - nfirst[nati - 1] >= 3;
  long long kk = 0;
  for (int jj = 1; jj <= numat; ++jj) {
    if (jj == nati) continue;
    off[jj - 1] = kk;
    const bool hj = nlast[jj - 1] - nfirst[jj - 1] >= 3;
    kk += (hi && hj) ? 100 : ((hi || hj) ? 10 : 1);
  }
  const size_t b_idx = sizeof(int) * 2 * (size_t)numat, b_off = sizeof(long long) * (size_t)numat;
  const size_t b_stage = sizeof(double) * 10 * (size_t)numat;
  char* buf = nullptr;
  MB_CUDA(mb_malloc_async(&buf, b_idx + b_off + b_stage + 64, s));
  long long* d_off = (long long*)buf;
  double* d_stage = (double*)(buf + b_off);
  int* d_first = (int*)(buf + b_off + b_stage);
  int* d_last = d_first + numat;
  DfArgs a{numat, nati, d_first, d_last, d_off, f, ptot, p, w, d_stage};
  cudaError_t e = cudaMemcpyAsync(d_first, nfirst, sizeof(int) * numat, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_last, nlast, sizeof(int) * numat, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_off, off.data(), b_off, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    dfock2_pairs<<<(numat + 127) / 128, 128, 0, s>>>(a);
    e = cudaGetLastError();
    mb_count_launch();
  }
  if (e == cudaSuccess) {
    dfock2_fold<<<1, 32, 0, s>>>(a);
    e = cudaGetLastError();
    mb_count_launch();
  }
  // the host arrays above are read by the copies: finish before returning
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFreeAsync(buf, s);
  if (e != cudaSuccess) return mb_set_cuda_error(e, "mb_dfock2_dev", __FILE__, __LINE__);
  return MB_OK;
}
