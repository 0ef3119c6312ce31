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

// tidy's compression step, one thread per LMO: drop the atoms whose squared
// coefficients sum to thresh or less, keeping the order of the rest, in place
// within the LMO's own storage (moves only to lower addresses).
__global__ void tidy_kernel(int nlmo, const int* __restrict__ iorbs, int* __restrict__ ncf,
                            const int* __restrict__ nncf, int* __restrict__ icocc, const int* __restrict__ ncocc,
                            double* __restrict__ cocc, double thresh) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nlmo) return;
  long long mm = ncocc[i], mn = ncocc[i];
  int kept = 0;
  const int n = ncf[i];
  for (int j1 = 0; j1 < n; ++j1) {
    const int a = icocc[nncf[i] + j1];
    const int no = iorbs[a - 1];
    double s = 0.0;
    for (int k = 0; k < no; ++k) s = DADD(s, DMUL(cocc[mm + k], cocc[mm + k]));
    if (s > thresh) {
      for (int k = 0; k < no; ++k) cocc[mn + k] = cocc[mm + k];
      icocc[nncf[i] + kept] = a;
      mn += no;
      ++kept;
    }
    mm += no;
  }
  ncf[i] = kept;
}

}  // namespace

extern "C" int mb_mz_tidy_dev(MbMzLmos* Q, const int* iorbs, double thresh, cudaStream_t s) {
  if (!Q || !iorbs) return mb_set_error(MB_ERR_ARG, "mb_mz_tidy_dev: bad args");
  if (Q->nlmo <= 0) return MB_OK;
  tidy_kernel<<<nblk(Q->nlmo, 128), 128, 0, s>>>(Q->nlmo, iorbs, const_cast<int*>(Q->ncf), Q->nncf,
                                                 const_cast<int*>(Q->icocc), Q->ncocc, const_cast<double*>(Q->cocc),
                                                 thresh);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

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
  MB_CUDA(mb_malloc_async((void**)&dflag, (size_t)(np > 0 ? np : 1), s));
  cudaError_t e = mb_malloc_async((void**)&dheads, sizeof(int) * 2 * (size_t)(no + nv + 1), s);
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

// ------------------------------------------------------------ the SCF loop
// iter_for_MOZYME (MOZYME/iter_for_MOZYME.F90:218-630) for a whole
// closed-shell system behind one C entry: density, Fock and energy of the
// starting LMOs (:439-473); per iteration tidy's compression (:221, :326),
// check (:482-484), eimp (:495),
// diagg = diagg1 + diagg2 + density (diagg.F90), addhb every third iteration
// while fewer than four were made (:529-538), cnvgz while the three-point
// extrapolation is on (:549), buildf and helecz (:558-567), isitsc's 1SCF
// test (isitsc.F90:34-44: ovmax below 5 selcon and |dE| below selcon on two
// consecutive iterations; ovmax is diagg1's tiny) and the shift control
// (:615-628).  The host sees a few scalars per iteration.
extern "C" size_t mb_mz_fock_ws_bytes(const MbMzLayout* layout);
extern "C" int mb_mz_fock_nat_dev(const MbMzLayout* layout, const int* nat, const double* coord, const double* w,
                                  const double* ptot, const double* h, double* f, void* ws, cudaStream_t stream);
extern "C" int mb_mz_fock_dev(const MbMzLayout* layout, const double* coord, const double* w, const double* ptot,
                              const double* h, double* f, void* ws, cudaStream_t stream);
extern "C" int mb_mz_density_dev(const MbMzLayout* layout, const MbMzLmos* lmos, int mode, const double* partp,
                                 double* p, cudaStream_t stream);
extern "C" size_t mb_mz_diagg1_ws_bytes(const MbMzLayout* layout, const MbMzLmos* occ, const MbMzLmos* vir);
extern "C" int mb_mz_diagg1_dev(const MbMzLayout* layout, const MbMzLmos* occ, const MbMzLmos* vir, const double* fao,
                                const double* p, int idiagg, double* state, int* nfmo, int* ifmo, double* fmo,
                                long long* nij, double* eigv, double* eigs, int* eigs_done, double* sumt, void* ws,
                                cudaStream_t stream);
extern "C" int mb_mz_diagg2_dev(const MbMzLayout* layout, MbMzLmos* occ, MbMzLmos* vir, const int* ifmo,
                                const double* fmo, long long nij, const double* eigs, const double* eigv, int idiagg,
                                const double* ctl, int* nrejct, double* sumb, long long* nrej, cudaStream_t stream);
extern "C" size_t mb_mz_helecz_ws_bytes(void);
extern "C" int mb_mz_helecz_ws(long long mpack, int norbs, const long long* idiag, const double* p, const double* h,
                               const double* f, double* out, double* ws, cudaStream_t stream);
extern "C" size_t mb_mz_cnvgz_ws_bytes(void);
extern "C" int mb_mz_cnvgz_ws(int norbs, long long mpack, double* pnew, double* p, double* p1, double* p2, double* p3,
                              int niter, const long long* idiag, int use3, double* pmax_out, void* ws,
                              cudaStream_t stream);
extern "C" int mb_mz_idiag(const MbMzLayout* layout, long long* idiag);
extern "C" int mb_mz_lmos_refresh(int numat, const int* iorbs_host, MbMzLmos* lmos);
extern "C" int mb_mz_lmos_refresh_dev(int numat, const int* iorbs_dev, MbMzLmos* lmos, cudaStream_t stream);

extern "C" void mb_mz_scf_opts_default(mb_mz_scf_opts* o) {
  o->scfcrt = 1.0e-2;
  o->itrmax = 2000;
  o->cap = 0;
  o->verbose = 0;
  o->nat = nullptr;
}

namespace {
// device buffers of one MOZYME SCF, freed together
struct MzScfBufs {
  std::vector<void*> ptrs;
  template <typename T>
  int get(T** out, size_t count) {
    void* p = nullptr;
    MB_CUDA(cudaMalloc(&p, sizeof(T) * (count > 0 ? count : 1)));
    ptrs.push_back(p);
    *out = (T*)p;
    return MB_OK;
  }
  ~MzScfBufs() {
    for (void* p : ptrs) cudaFree(p);
  }
};
}  // namespace

extern "C" int mb_mz_scf_run(const MbMzLayout* L, const int* iorbs_host, MbMzLmos* occ, MbMzLmos* vir,
                             const double* coord, const double* w, const double* h, double enuclr, double atheat,
                             const mb_mz_scf_opts* opts_in, double* p, double* f, mb_mz_scf_result* res,
                             cudaStream_t s) {
  if (!L || !iorbs_host || !occ || !vir || !coord || !w || !h || !p || !f || !res)
    return mb_set_error(MB_ERR_ARG, "mb_mz_scf_run: bad args");
  mb_mz_scf_opts opts;
  if (opts_in) opts = *opts_in; else mb_mz_scf_opts_default(&opts);
  memset(res, 0, sizeof(*res));
  const double fpc9 = 23.060547830619029;
  const int n = L->norbs, numat = L->numat;
  const long long mpack = L->mpack;
  const long long cap = opts.cap > 0 ? opts.cap : 300LL * n;
  const double selcon = opts.scfcrt;
  const double const_damp = 1.0, thresh = 1.0e-13, bigeps = 50.0 * sqrt(1.0e-39);
  const double hb_limits[4] = {1.0, 0.1, 0.01, 0.001};  // addhb's cutoffs on its first four calls
  cudaEvent_t e0, e1;
  MB_CUDA(cudaEventCreate(&e0));
  MB_CUDA(cudaEventCreate(&e1));
  MB_CUDA(cudaEventRecord(e0, s));
  MzScfBufs B;
  long long* idiag;
  double *pold, *p1, *p2, *p3, *norm_o, *norm_v, *eigv, *eigs, *fmo, *hb_fmo, *scal, *hws, *cws;
  int *nfmo, *ifmo, *hb_ifmo;
  void *fws, *dws;
  const int nocc = occ->nlmo, nvir = vir->nlmo;
  MB_TRY(B.get(&idiag, n));
  MB_TRY(B.get(&pold, mpack));
  MB_TRY(B.get(&p1, n));
  MB_TRY(B.get(&p2, n));
  MB_TRY(B.get(&p3, n));
  MB_TRY(B.get(&norm_o, nocc));
  MB_TRY(B.get(&norm_v, nvir));
  MB_TRY(B.get(&eigv, nvir));
  MB_TRY(B.get(&eigs, nocc));
  MB_TRY(B.get(&nfmo, nvir));
  MB_TRY(B.get(&ifmo, 2 * cap));
  MB_TRY(B.get(&fmo, cap));
  MB_TRY(B.get(&hb_ifmo, 2 * cap));
  MB_TRY(B.get(&hb_fmo, cap));
  MB_TRY(B.get(&scal, 8));
  MB_TRY(B.get(&hws, mb_mz_helecz_ws_bytes() / 8 + 1));
  MB_TRY(B.get(&cws, mb_mz_cnvgz_ws_bytes() / 8 + 1));
  MB_TRY(B.get((char**)&fws, mb_mz_fock_ws_bytes(L) + 256));
  MB_TRY(B.get((char**)&dws, mb_mz_diagg1_ws_bytes(L, occ, vir) + 256));
  void* dws_al = (void*)(((uintptr_t)dws + 255) & ~(uintptr_t)255);
  {
    std::vector<long long> idg(n);
    MB_TRY(mb_mz_idiag(L, idg.data()));
    MB_CUDA(cudaMemcpyAsync(idiag, idg.data(), sizeof(long long) * n, cudaMemcpyHostToDevice, s));
    MB_CUDA(cudaStreamSynchronize(s));
  }
  MB_CUDA(cudaMemsetAsync(pold, 0, sizeof(double) * mpack, s));
  MB_CUDA(cudaMemsetAsync(p1, 0, sizeof(double) * n, s));
  MB_CUDA(cudaMemsetAsync(p2, 0, sizeof(double) * n, s));
  MB_CUDA(cudaMemsetAsync(p3, 0, sizeof(double) * n, s));
  MB_CUDA(cudaMemsetAsync(nfmo, 0, sizeof(int) * (nvir > 0 ? nvir : 1), s));
  MB_CUDA(cudaMemsetAsync(eigv, 0, sizeof(double) * (nvir > 0 ? nvir : 1), s));
  MB_CUDA(cudaMemsetAsync(eigs, 0, sizeof(double) * (nocc > 0 ? nocc : 1), s));
  auto energy = [&](double* ee_out) -> int {
    MB_TRY(mb_mz_helecz_ws(mpack, n, idiag, p, h, f, scal, hws, s));
    MB_CUDA(cudaMemcpyAsync(ee_out, scal, sizeof(double), cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    return MB_OK;
  };
  // the starting LMOs' density, Fock matrix and energy (iter_for_MOZYME.F90:439-473)
  MB_TRY(mb_mz_density_dev(L, occ, 0, nullptr, p, s));
  MB_TRY(mb_mz_fock_nat_dev(L, opts.nat, coord, w, p, h, f, fws, s));
  double ee = 0.0;
  MB_TRY(energy(&ee));
  double escf = (ee + enuclr) * fpc9 + atheat;
  double state[4] = {10.0, 1.0, 0.0, 0.0};  // diagg1's fref, safety, oldlim, tiny
  int nrejct[2] = {0, 0};
  double eold = 0.0, shift = 0.0;
  int niter = 0, idiagg = 0, lstart = 0, nhb = 0;
  bool use3 = true, scf1 = false, converged = false;
  long long nrej_total = 0;
  for (;;) {
    // tidy's compression (iter_for_MOZYME.F90:221, :326), then the index
    MB_TRY(mb_mz_tidy_dev(occ, L->iorbs, thresh, s));
    MB_TRY(mb_mz_tidy_dev(vir, L->iorbs, thresh, s));
    MB_TRY(mb_mz_lmos_refresh_dev(numat, L->iorbs, occ, s));
    MB_TRY(mb_mz_lmos_refresh_dev(numat, L->iorbs, vir, s));
    double eo = 0.0, ev = 0.0;
    MB_TRY(mb_mz_check_dev(occ, L->iorbs, norm_o, &eo, s));
    MB_TRY(mb_mz_check_dev(vir, L->iorbs, norm_v, &ev, s));
    if (eo > 0.1 || ev > 0.1) return mb_set_error(MB_ERR_NUMERIC, "ERROR DETECTED IN SUBROUTINE CHECK");
    MB_TRY(mb_mz_eimp_dev(L, p, f, s));
    long long nij = cap;
    int done = 0;
    double sumt = 0.0;
    MB_TRY(mb_mz_diagg1_dev(L, occ, vir, f, p, idiagg, state, nfmo, ifmo, fmo, &nij, eigv, eigs, &done, &sumt,
                            dws_al, s));
    const double ovmax = state[3];
    double ctl[5] = {const_damp, shift, thresh, state[3], bigeps};
    double sumb = 0.0;
    long long nrej = 0;
    MB_TRY(mb_mz_diagg2_dev(L, occ, vir, ifmo, fmo, nij, eigs, eigv, idiagg, ctl, nrejct, &sumb, &nrej, s));
    nrej_total += nrej;
    MB_TRY(mb_mz_lmos_refresh_dev(numat, L->iorbs, occ, s));
    MB_TRY(mb_mz_lmos_refresh_dev(numat, L->iorbs, vir, s));
    MB_TRY(mb_mz_density_dev(L, occ, 0, nullptr, p, s));
    ++idiagg;
    ++niter;
    long long nhb_ij = 0;
    if (niter % 3 == 0 && nhb < 4) {  // addhb
      ++nhb;
      MB_TRY(mb_mz_hbonds_dev(L, occ, vir, f, p, hb_limits[nhb - 1], cap, hb_ifmo, hb_fmo, &nhb_ij, s));
      if (nhb_ij) {
        double ctl2[5] = {const_damp, shift, thresh, state[3], bigeps};
        MB_TRY(mb_mz_diagg2_dev(L, occ, vir, hb_ifmo, hb_fmo, nhb_ij, eigs, eigv, idiagg, ctl2, nrejct, &sumb, &nrej,
                                s));
        nrej_total += nrej;
        MB_TRY(mb_mz_lmos_refresh_dev(numat, L->iorbs, occ, s));
        MB_TRY(mb_mz_lmos_refresh_dev(numat, L->iorbs, vir, s));
        if (idiagg % 2 == 1) ++idiagg;
      }
    }
    if (use3) MB_TRY(mb_mz_cnvgz_ws(n, mpack, p, pold, p1, p2, p3, niter, idiag, 1, scal + 1, cws, s));
    MB_TRY(mb_mz_fock_nat_dev(L, opts.nat, coord, w, p, h, f, fws, s));
    MB_TRY(energy(&ee));
    if (!isfinite(ee)) return mb_set_error(MB_ERR_NUMERIC, "mb_mz_scf_run: non-finite energy");
    escf = (ee + enuclr) * fpc9 + atheat;
    double de = escf - eold;
    eold = escf;
    if (fabs(de) > 9999.0) de = 0.0;
    if (opts.verbose)
      fprintf(stderr, " MOZYME ITERATION %4d ENERGY %16.6f DELTAE %13.7f OVMAX %10.3e PAIRS %lld HB %lld\n", niter,
              escf, de, ovmax, nij, nhb_ij);
    const bool ok = ovmax < 5.0 * selcon && fabs(de) < selcon;
    if ((ok && scf1) || niter > opts.itrmax) {
      if (niter > 3) {
        converged = niter <= opts.itrmax;
        break;
      }
    }
    scf1 = ok;
    if (use3) {
      if (niter % 3 == 2 && fabs(de) < 0.1) {
        use3 = false;
        lstart = niter;
        shift = 0.0;
      }
    } else if (de > 0.0 && shift < 11.0 && niter > lstart + 2) {
      shift += 2.0;
      lstart = niter;
    }
  }
  MB_CUDA(cudaEventRecord(e1, s));
  MB_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  MB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  res->escf = escf;
  res->ee = ee;
  res->niter = niter;
  res->converged = converged ? 1 : 0;
  res->t_total_ms = ms;
  res->nrejected = nrej_total;
  if (!converged) return mb_set_error(MB_ERR_NOCONV, "MOZYME: UNABLE TO ACHIEVE SELF-CONSISTENCE");
  return MB_OK;
}
