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
#include <vector>

#include "mb_common.cuh"

namespace {

__device__ __forceinline__ int pair_elems(int io, int jo, bool diag) { return diag ? io * (io + 1) / 2 : io * jo; }

// One warp per stored block (grid-stride over pair entries).
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
    int a = Q.atom_ptr[i], ae = Q.atom_ptr[i + 1];
    int b = Q.atom_ptr[j], be = Q.atom_ptr[j + 1];
    while (a < ae && b < be) {  // warp-uniform merge of two ascending LMO lists
      const int la = Q.atom_lmo[a], lb = Q.atom_lmo[b];
      if (la == lb) {
        if (act) acc = DADD(acc, DMUL(Q.cocc[Q.atom_coff[b] + k1], Q.cocc[Q.atom_coff[a] + j1]));
        ++a;
        ++b;
      } else if (la < lb) {
        ++a;
      } else {
        ++b;
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

int grid_for(long long n) {
  long long b = (n + 255) / 256;
  return (int)(b > 148 * 8 ? 148 * 8 : (b < 1 ? 1 : b));
}

template <class T>
int upload(const std::vector<T>& v, const T** out) {
  T* d = nullptr;
  if (!v.empty()) {
    MB_CUDA(cudaMalloc(&d, sizeof(T) * v.size()));
    MB_CUDA(cudaMemcpy(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
  }
  *out = d;
  return MB_OK;
}

}  // namespace

extern "C" int mb_mz_layout_create(int numat, const int* iorbs, const double* coord, double cutof1, double cutof2,
                                   MbMzLayout* out, long long* nijbo) {
  if (numat <= 0 || !iorbs || !coord || !out) return mb_set_error(MB_ERR_ARG, "mb_mz_layout_create: bad args");
  memset(out, 0, sizeof(*out));
  for (int i = 0; i < numat; ++i)
    if (iorbs[i] < 0 || iorbs[i] > 4) return mb_set_error(MB_ERR_UNSUPPORTED, "MOZYME layout: s and p shells only");
  std::vector<int> pi, pj, ptr(numat + 1, 0);
  std::vector<long long> po;
  long long mpack = 0;
  for (int i = 0; i < numat; ++i) {
    ptr[i] = (int)pi.size();
    const int io = iorbs[i];
    for (int j = 0; j < i; ++j) {
      const double dx = coord[3 * i] - coord[3 * j], dy = coord[3 * i + 1] - coord[3 * j + 1],
                   dz = coord[3 * i + 2] - coord[3 * j + 2];
      const double r = dx * dx + dy * dy + dz * dz;
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
      if (nijbo) nijbo[(long long)i * numat + j] = nijbo[(long long)j * numat + i] = v;
    }
    pi.push_back(i);
    pj.push_back(i);
    po.push_back(mpack);
    if (nijbo) nijbo[(long long)i * numat + i] = mpack;
    mpack += (long long)io * (io + 1) / 2;
  }
  ptr[numat] = (int)pi.size();
  std::vector<int> io(iorbs, iorbs + numat);
  out->numat = numat;
  out->mpack = mpack;
  out->npairs = (long long)pi.size();
  int rc = upload(io, &out->iorbs);
  if (rc == MB_OK) rc = upload(ptr, &out->pair_ptr);
  if (rc == MB_OK) rc = upload(pi, &out->pair_i);
  if (rc == MB_OK) rc = upload(pj, &out->pair_j);
  if (rc == MB_OK) rc = upload(po, &out->pair_off);
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

extern "C" int mb_mz_lmos_create(int numat, const int* iorbs, int nlmo, const int* ncf, const int* nncf,
                                 const int* icocc, const int* ncocc, const double* cocc, long long ncocc_total,
                                 MbMzLmos* out) {
  if (numat <= 0 || nlmo < 0 || !out) return mb_set_error(MB_ERR_ARG, "mb_mz_lmos_create: bad args");
  memset(out, 0, sizeof(*out));
  std::vector<int> cnt(numat + 1, 0);
  for (int i = 0; i < nlmo; ++i)
    for (int jj = nncf[i]; jj < nncf[i] + ncf[i]; ++jj) {
      const int a = icocc[jj] - 1;
      if (a < 0 || a >= numat) return mb_set_error(MB_ERR_ARG, "mb_mz_lmos_create: atom number out of range");
      cnt[a + 1]++;
    }
  for (int a = 0; a < numat; ++a) cnt[a + 1] += cnt[a];
  std::vector<int> fill(cnt.begin(), cnt.end() - 1), lmo(cnt[numat]), coff(cnt[numat]);
  for (int i = 0; i < nlmo; ++i) {  // ascending LMO order per atom by construction
    int c = ncocc[i];
    for (int jj = nncf[i]; jj < nncf[i] + ncf[i]; ++jj) {
      const int a = icocc[jj] - 1;
      lmo[fill[a]] = i;
      coff[fill[a]] = c;
      fill[a]++;
      c += iorbs[a];
    }
    if (c > ncocc_total) return mb_set_error(MB_ERR_ARG, "mb_mz_lmos_create: cocc too short for the atom lists");
  }
  std::vector<double> cv(cocc, cocc + ncocc_total);
  out->nlmo = nlmo;
  int rc = upload(cnt, &out->atom_ptr);
  if (rc == MB_OK) rc = upload(lmo, &out->atom_lmo);
  if (rc == MB_OK) rc = upload(coff, &out->atom_coff);
  if (rc == MB_OK) rc = upload(cv, &out->cocc);
  if (rc != MB_OK) mb_mz_lmos_destroy(out);
  return rc;
}

extern "C" int mb_mz_lmos_destroy(MbMzLmos* Q) {
  if (!Q) return MB_OK;
  cudaFree((void*)Q->atom_ptr);
  cudaFree((void*)Q->atom_lmo);
  cudaFree((void*)Q->atom_coff);
  cudaFree((void*)Q->cocc);
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
