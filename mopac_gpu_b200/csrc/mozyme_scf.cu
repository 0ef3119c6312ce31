// The routines iter_for_MOZYME (MOZYME/iter_for_MOZYME.F90:218-630) calls
// between the sparse kernels, on the device:
//   * check (MOZYME/check.F90): renormalise every LMO over its atoms;
//   * eimp (MOZYME/eimp.F90): the first element of every stored off-diagonal
//     block of P becomes the block's sum of squared F elements (diagg1 reads
//     it as the pair's weight; the next density build overwrites it);
//   * hbonds (MOZYME/hbonds.F90), called by addhb: the (virtual, occupied)
//     LMO pairs around stored atom pairs that carry Fock coupling but no
//     density yet, the list diagg2 then rotates.
// Each sum runs in the reference's order (one thread per LMO or block), so the
// results are bit for bit the oracle's.  The hbonds list is assembled on the
// host from the device's per-pair flags and the LMOs' first two atoms: it is
// integer index work in the reference's loop order, a few times per SCF.
#include <math.h>
#include <string.h>

#include <vector>

#include "mb_common.cuh"

namespace {

int nblk(long long n, int t) { return (int)((n + t - 1) / t); }

__global__ void check_kernel(int nlmo, const int* __restrict__ iorbs, const int* __restrict__ ncf,
                             const int* __restrict__ nncf, const int* __restrict__ icocc,
                             const int* __restrict__ ncocc, double* __restrict__ cocc, double* __restrict__ norm2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nlmo) return;
  int n = 0;
  for (int j = 0; j < ncf[i]; ++j) n += iorbs[icocc[nncf[i] + j] - 1];
  double* c = cocc + ncocc[i];
  double s = 0.0;
  for (int m = 0; m < n; ++m) s = DADD(s, DMUL(c[m], c[m]));
  norm2[i] = s;
  const double sc = 1.0 / sqrt(s);
  for (int m = 0; m < n; ++m) c[m] = DMUL(c[m], sc);
}

__global__ void eimp_kernel(long long npairs, const int* __restrict__ pair_i, const int* __restrict__ pair_j,
                            const long long* __restrict__ pair_off, const int* __restrict__ iorbs,
                            const double* __restrict__ f, double* __restrict__ p) {
  long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= npairs) return;
  const int i = pair_i[e], j = pair_j[e];
  if (i == j) return;
  const long long k = pair_off[e];
  const int m = iorbs[i] * iorbs[j];
  double s = 0.0;
  for (int q = 0; q < m; ++q) s = DADD(s, DMUL(f[k + q], f[k + q]));
  p[k] = s;
}

__global__ void hbond_flags_kernel(long long npairs, const int* __restrict__ pair_i, const int* __restrict__ pair_j,
                                   const long long* __restrict__ pair_off, const int* __restrict__ iorbs,
                                   const double* __restrict__ f, const double* __restrict__ p, double cutoff,
                                   unsigned char* __restrict__ flag) {
  long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= npairs) return;
  const int i = pair_i[e], j = pair_j[e];
  unsigned char r = 0;
  if (i != j) {
    const long long k = pair_off[e];
    const int m = iorbs[i] * iorbs[j];
    double sf = 0.0, sp = 0.0;
    for (int q = 0; q < m; ++q) {
      sf = DADD(sf, DMUL(f[k + q], f[k + q]));
      sp = DADD(sp, DMUL(p[k + q], p[k + q]));
    }
    r = (sp < 1.0e-10 && sf > cutoff) ? 1 : 0;
  }
  flag[e] = r;
}

// First and second atom (1-based) of every LMO: icocc(l) and
// icocc(l + min(ncf - 1, 1)), l = nncf + 1 in the reference's indexing.
__global__ void heads_kernel(int nlmo, const int* __restrict__ ncf, const int* __restrict__ nncf,
                             const int* __restrict__ icocc, int* __restrict__ heads) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nlmo) return;
  if (ncf[q] <= 0) {  // an empty LMO touches no atom
    heads[2 * q] = heads[2 * q + 1] = 0;
    return;
  }
  const int kk = ncf[q] - 1 < 1 ? ncf[q] - 1 : 1;
  heads[2 * q] = icocc[nncf[q]];
  heads[2 * q + 1] = icocc[nncf[q] + kk];
}

}  // namespace

extern "C" int mb_mz_check_dev(const MbMzLmos* Q, const int* iorbs, double* norm2, double* error_out,
                               cudaStream_t s) {
  if (!Q || !iorbs || !norm2) return mb_set_error(MB_ERR_ARG, "mb_mz_check_dev: bad args");
  if (Q->nlmo == 0) {
    if (error_out) *error_out = 0.0;
    return MB_OK;
  }
  // the LMO coefficients are device-owned and updated in place (as diagg2 does)
  check_kernel<<<nblk(Q->nlmo, 128), 128, 0, s>>>(Q->nlmo, iorbs, Q->ncf, Q->nncf, Q->icocc, Q->ncocc,
                                                  const_cast<double*>(Q->cocc), norm2);
  MB_LAUNCH_CHECK();
  if (error_out) {
    std::vector<double> h((size_t)Q->nlmo);
    MB_CUDA(cudaMemcpyAsync(h.data(), norm2, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    double err = 0.0;
    for (double v : h) err += fabs(1.0 - v);
    *error_out = err;
  }
  return MB_OK;
}

extern "C" int mb_mz_eimp_dev(const MbMzLayout* L, double* p, const double* f, cudaStream_t s) {
  if (!L || !p || !f) return mb_set_error(MB_ERR_ARG, "mb_mz_eimp_dev: bad args");
  if (L->npairs == 0) return MB_OK;
  eimp_kernel<<<nblk(L->npairs, 256), 256, 0, s>>>(L->npairs, L->pair_i, L->pair_j, L->pair_off, L->iorbs, f, p);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

// hbonds: the list in diagg1's layout (ifmo[2e] virtual, ifmo[2e+1]
// occupied, 1-based; fmo[e] = 0.1), at most cap entries (MB_ERR_UNSUPPORTED
// beyond).  ifmo, fmo: device.  Synchronises the stream.
extern "C" int mb_mz_hbonds_dev(const MbMzLayout* L, const MbMzLmos* occ, const MbMzLmos* vir, const double* f,
                                const double* p, double cutoff, long long cap, int* ifmo, double* fmo,
                                long long* nij_out, cudaStream_t s) {
  if (!L || !occ || !vir || !f || !p || !ifmo || !fmo || !nij_out || cap <= 0)
    return mb_set_error(MB_ERR_ARG, "mb_mz_hbonds_dev: bad args");
  *nij_out = 0;
  const long long np = L->npairs;
  const int no = occ->nlmo, nv = vir->nlmo;
  unsigned char* dflag = nullptr;
  int* dheads = nullptr;
  MB_CUDA(cudaMallocAsync((void**)&dflag, (size_t)(np > 0 ? np : 1), s));
  cudaError_t e = cudaMallocAsync((void**)&dheads, sizeof(int) * 2 * (size_t)(no + nv + 1), s);
  if (e != cudaSuccess) {
    cudaFreeAsync(dflag, s);
    return mb_set_cuda_error(e, "mb_mz_hbonds_dev", __FILE__, __LINE__);
  }
  std::vector<unsigned char> flag((size_t)np);
  std::vector<int> pi((size_t)np), pj((size_t)np), heads(2 * (size_t)(no + nv));
  int rc = MB_OK;
  if (np > 0) {
    hbond_flags_kernel<<<nblk(np, 256), 256, 0, s>>>(np, L->pair_i, L->pair_j, L->pair_off, L->iorbs, f, p, cutoff,
                                                     dflag);
    if ((e = cudaGetLastError()) != cudaSuccess) rc = mb_set_cuda_error(e, "hbond flags", __FILE__, __LINE__);
    mb_count_launch();
  }
  if (rc == MB_OK && no > 0) {
    heads_kernel<<<nblk(no, 128), 128, 0, s>>>(no, occ->ncf, occ->nncf, occ->icocc, dheads);
    if ((e = cudaGetLastError()) != cudaSuccess) rc = mb_set_cuda_error(e, "hbond heads", __FILE__, __LINE__);
    mb_count_launch();
  }
  if (rc == MB_OK && nv > 0) {
    heads_kernel<<<nblk(nv, 128), 128, 0, s>>>(nv, vir->ncf, vir->nncf, vir->icocc, dheads + 2 * no);
    if ((e = cudaGetLastError()) != cudaSuccess) rc = mb_set_cuda_error(e, "hbond heads", __FILE__, __LINE__);
    mb_count_launch();
  }
  if (rc == MB_OK && np > 0) {
    e = cudaMemcpyAsync(flag.data(), dflag, (size_t)np, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(pi.data(), L->pair_i, sizeof(int) * np, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(pj.data(), L->pair_j, sizeof(int) * np, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) rc = mb_set_cuda_error(e, "hbond copies", __FILE__, __LINE__);
  }
  if (rc == MB_OK && no + nv > 0) {
    e = cudaMemcpyAsync(heads.data(), dheads, sizeof(int) * heads.size(), cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) rc = mb_set_cuda_error(e, "hbond copies", __FILE__, __LINE__);
  }
  // always wait: copies already queued write into the host vectors above
  e = cudaStreamSynchronize(s);
  if (rc == MB_OK && e != cudaSuccess) rc = mb_set_cuda_error(e, "hbond sync", __FILE__, __LINE__);
  cudaFreeAsync(dflag, s);
  cudaFreeAsync(dheads, s);
  if (rc != MB_OK) return rc;
  // the reference's loops: atoms i ascending, partners j < i ascending (the
  // layout's pair order), then virtual LMOs, then the occupied ones found
  std::vector<int> hi, hv;  // (virtual, occupied) 1-based
  std::vector<int> used;
  for (long long q = 0; q < np; ++q) {
    if (!flag[q]) continue;
    const int i = pi[q] + 1, j = pj[q] + 1;  // 1-based like icocc
    used.clear();
    for (int k = 0; k < no; ++k) {
      const int a = heads[2 * k], b = heads[2 * k + 1];
      if (a == i || b == i || a == j || b == j) used.push_back(k);
    }
    for (int k = 0; k < nv; ++k) {
      const int a = heads[2 * (no + k)], b = heads[2 * (no + k) + 1];
      if (a == i || b == i || a == j || b == j)
        for (int u : used) {
          hi.push_back(k + 1);
          hv.push_back(u + 1);
        }
    }
  }
  const long long nij = (long long)hi.size();
  if (nij > cap) return mb_set_error(MB_ERR_UNSUPPORTED, "mb_mz_hbonds_dev: list longer than cap");
  if (nij > 0) {
    std::vector<int> pairs(2 * (size_t)nij);
    std::vector<double> vals((size_t)nij, 0.1);
    for (long long t = 0; t < nij; ++t) {
      pairs[2 * t] = hi[t];
      pairs[2 * t + 1] = hv[t];
    }
    MB_CUDA(cudaMemcpyAsync(ifmo, pairs.data(), sizeof(int) * pairs.size(), cudaMemcpyHostToDevice, s));
    MB_CUDA(cudaMemcpyAsync(fmo, vals.data(), sizeof(double) * vals.size(), cudaMemcpyHostToDevice, s));
    MB_CUDA(cudaStreamSynchronize(s));  // the host vectors go out of scope
  }
  *nij_out = nij;
  return MB_OK;
}
