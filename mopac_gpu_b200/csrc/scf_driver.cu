// Device-resident SCF context and driver.
//
// mb_scf_run restates the control flow of iter (SCF/iter.F90:16-1107) for
// closed-shell RHF with default keywords and 1SCF settings: the level-shift
// logic (:273-325), Fock build (:553), energy and heat (:641-659), the
// convergence test (:675-690), the newdg/oknewd switches (:1022-1041), full
// diagonalisation (:849) or -- with opts.pseudo -- the pseudo-diagonalisation
// the reference comments out (:847-861), the density (:897), cnvg (:899-901)
// or -- with opts.pulay, the PULAY keyword -- Pulay's converger (:815-831),
// and the exit diagonalisation (:1052-1106).  All matrices stay in HBM; the
// host only sees the scalars the control flow branches on (energy, max|dP|,
// HOMO/LUMO eigenvalues), a handful of bytes per iteration.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "mb_common.cuh"
#include "pm7_params.h"

// kernels defined in other translation units
extern "C" int mb_helect_ws(int n, const double* p, const double* h, const double* f, double* out, double* ws,
                            cudaStream_t stream);
extern "C" int mb_cnvg_ws(int norbs, double* pnew, double* p, double* p1, int niter, double* pl_out, double* ws,
                          cudaStream_t stream);
extern "C" size_t mb_eigh_ws_bytes(int n);
extern "C" int mb_eigh_ws(int n, double* fpacked, int perturb, double* c, double* eigs, void* ws, int* status_dev,
                          cudaStream_t stream);
extern "C" size_t mb_pseudo_ws_bytes(int n, int nocc);
extern "C" int mb_dgemm_dev(char transa, char transb, int m, int n, int k, double alpha, const double* a, int lda,
                            const double* b, int ldb, double beta, double* c, int ldc, cudaStream_t stream);
extern "C" int mb_unpack_dev(int n, const double* pk, double* a, int lda, int perturb, double* pk_mut,
                             cudaStream_t stream);
extern "C" size_t mb_fock2_ws_bytes(int numat);
extern "C" int mb_fock2_ws(const MbAtomsDev* atoms, double* f, const double* h, const double* ptot, const double* pa,
                           const double* w, double shift, int use_shift, void* ws, size_t ws_bytes,
                           cudaStream_t stream);
extern "C" int mb_pseudo_diag_ws(int n, int nocc, const double* fpacked, double* c, const double* eigs,
                                 unsigned long long* nrot_dev, void* ws, cudaStream_t stream);
extern "C" int mb_pseudo_diag_ex(int n, int nocc, const double* fpacked, double* c, const double* eigs,
                                 unsigned long long* nrot_dev, void* ws, void* split_ws, size_t split_ws_bytes,
                                 int* split_err, double bigeps, double tiny_direct, cudaStream_t stream);
extern "C" int mb_orbital_energies_ws(int n, const double* fpacked, const double* c, double* eigs, void* ws,
                                      cudaStream_t stream);
extern "C" size_t mb_gemm_split_ws_bytes(int m, int n, int k);
extern "C" size_t mb_density_split_ws_bytes(int n, int nocc);
extern "C" int mb_density_split_ws(int n, int nocc, double occ, const double* c, int ldc, double* p, void* ws,
                                   size_t ws_bytes, int* err_dev, cudaStream_t stream);
extern "C" size_t mb_pulay_ws_bytes(int n);
extern "C" int mb_pulay_ws(int n, double* f, const double* p, double* fppf, double* fock, int mfock, double* emat,
                           int ldemat, int* lfock, int* nfock, int* start, double* pl, void* ws, cudaStream_t stream);
struct mb_campking;
extern "C" int mb_campking_create(int n, mb_campking** out);
extern "C" void mb_campking_destroy(mb_campking* ck);
extern "C" int mb_campking_interp(mb_campking* ck, int np_, int mode, double e, const double* fp, double* cp,
                                  void* eig_ws, int* status, cudaStream_t s, int* mode_out, int* rotated);
extern "C" int mb_hcore_dev(const int* nat_d, const double* coord_d, const MbAtomsDev* at, int numat, double* h,
                            double* w, double* enuc_pairs, cudaStream_t stream);
extern "C" int mb_hcore_finish(int numat, const MbAtomsDev* at, const int* nat_d, double* h, const double* e1b,
                               double* enuclr_dev, const double* enuc_pairs, cudaStream_t stream);

// ------------------------------------------------------------------ errors
static thread_local std::string g_last_error;

int mb_set_error(int code, const char* msg) {
  g_last_error = msg ? msg : "";
  return code;
}

int mb_set_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
  g_last_error = buf;
  if (e == cudaErrorMemoryAllocation) return MB_ERR_NOMEM;
  return MB_ERR_CUDA;
}

extern "C" const char* mb_last_error(void) { return g_last_error.c_str(); }

static unsigned long long g_launches = 0;
void mb_count_launch() { __atomic_add_fetch(&g_launches, 1ull, __ATOMIC_RELAXED); }
extern "C" long long mb_launch_count(void) { return (long long)__atomic_load_n(&g_launches, __ATOMIC_RELAXED); }
extern "C" int mb_version(void) { return 100; }

// ------------------------------------------------------------ atom layout
static int build_layout(int numat, const int* nfirst, const int* nlast, std::vector<int>& first,
                        std::vector<int>& nor, std::vector<int>& lim, std::vector<long long>& wrow,
                        std::vector<int>& cum, long long* n2elec) {
  first.resize(numat); nor.resize(numat); lim.resize(numat); wrow.resize(numat); cum.resize(numat);
  long long off = 0;
  int c = 0;
  for (int a = 0; a < numat; ++a) {
    first[a] = nfirst[a] - 1;
    nor[a] = nlast[a] - nfirst[a] + 1;
    if (nor[a] != 1 && nor[a] != 4) return mb_set_error(MB_ERR_UNSUPPORTED, "only s and sp atoms are supported");
    lim[a] = nor[a] * (nor[a] + 1) / 2;
    cum[a] = c;
    wrow[a] = off;
    off += (long long)lim[a] * c + (long long)lim[a] * lim[a];
    c += lim[a];
  }
  *n2elec = off;
  return MB_OK;
}

extern "C" int mb_atoms_create(int numat, const int* nfirst, const int* nlast, MbAtomsDev* out) {
  if (numat <= 0 || !nfirst || !nlast || !out) return mb_set_error(MB_ERR_ARG, "mb_atoms_create: bad args");
  std::vector<int> first, nor, lim, cum;
  std::vector<long long> wrow;
  long long n2 = 0;
  MB_TRY(build_layout(numat, nfirst, nlast, first, nor, lim, wrow, cum, &n2));
  int *d_first, *d_nor, *d_lim, *d_cum;
  long long* d_wrow;
  MB_CUDA(cudaMalloc(&d_first, sizeof(int) * numat));
  MB_CUDA(cudaMalloc(&d_nor, sizeof(int) * numat));
  MB_CUDA(cudaMalloc(&d_lim, sizeof(int) * numat));
  MB_CUDA(cudaMalloc(&d_cum, sizeof(int) * numat));
  MB_CUDA(cudaMalloc(&d_wrow, sizeof(long long) * numat));
  MB_CUDA(cudaMemcpy(d_first, first.data(), sizeof(int) * numat, cudaMemcpyHostToDevice));
  MB_CUDA(cudaMemcpy(d_nor, nor.data(), sizeof(int) * numat, cudaMemcpyHostToDevice));
  MB_CUDA(cudaMemcpy(d_lim, lim.data(), sizeof(int) * numat, cudaMemcpyHostToDevice));
  MB_CUDA(cudaMemcpy(d_cum, cum.data(), sizeof(int) * numat, cudaMemcpyHostToDevice));
  MB_CUDA(cudaMemcpy(d_wrow, wrow.data(), sizeof(long long) * numat, cudaMemcpyHostToDevice));
  out->numat = numat;
  out->first = d_first;
  out->nor = d_nor;
  out->lim = d_lim;
  out->cum = d_cum;
  out->wrow = d_wrow;
  return MB_OK;
}

extern "C" int mb_atoms_destroy(MbAtomsDev* a) {
  if (!a) return MB_OK;
  cudaFree((void*)a->first);
  cudaFree((void*)a->nor);
  cudaFree((void*)a->lim);
  cudaFree((void*)a->cum);
  cudaFree((void*)a->wrow);
  memset(a, 0, sizeof(*a));
  return MB_OK;
}

// ------------------------------------------------------------------ context
struct mb_ctx {
  int numat = 0, norbs = 0, nclose = 0;
  long long mpack = 0, n2elec = 0;
  std::vector<int> nat, nfirst, nlast;
  std::vector<double> coord, pdiag;
  double atheat = 0.0, enuclr = 0.0;
  bool have_hw = false;
  MbAtomsDev atoms{};
  int* d_nat = nullptr;
  double* d_coord = nullptr;
  double* d_pdiag = nullptr;  // the diagonal guess on the device (norbs)
  double *h = nullptr, *w = nullptr, *f = nullptr, *p = nullptr, *pa = nullptr, *pold = nullptr, *pold2 = nullptr,
         *c = nullptr, *eigs = nullptr, *fdiag = nullptr;
  double* scal = nullptr;   // device scalars: [0] ee, [1] pl, [8..] scratch
  double* hws = nullptr;    // helect workspace (2n)
  int* status = nullptr;
  unsigned long long* nrot = nullptr;
  void* eig_ws = nullptr;
  void* pseudo_ws = nullptr;
  void* fock_ws = nullptr;  // the Fock build's staging (mb_fock2_ws_bytes(numat)), allocated on the first SCF
  // Pulay histories (npulay * mpack each), allocated on the first Pulay run
  double *fppf_hist = nullptr, *fock_hist = nullptr;
  // BF16 plane buffers of the split-precision GEMMs, allocated on first use
  void* tc_ws_raw = nullptr;
  void* tc_ws = nullptr;     // 1024-byte aligned inside tc_ws_raw
  size_t tc_ws_bytes = 0;
  // starting density for opts.guess (mb_ctx_set_guess / mb_ctx_guess)
  double* pguess = nullptr;
  bool have_guess = false;
  double* pprev = nullptr;          // previous density for the FP64 finish's max|dP|
  mb_guess_ws* guess_ws = nullptr;  // the prediction's grow-only workspace
  void* purify_ws = nullptr;        // McWeeny matrices when eig_ws is too small
  mb_campking* ck = nullptr;        // Camp-King's state, made on its first use
  double* exit_ws = nullptr;        // the split exit diagonalisation's matrices, made on its first use
  cudaStream_t stream = nullptr;
};

// History length of Pulay's converger: molkst_C.F90:114-115 sets npulay = 10.
static const int kNpulay = 10;

static void ctx_free(mb_ctx* c) {
  if (!c) return;
  mb_atoms_destroy(&c->atoms);
  mb_guess_ws_destroy(c->guess_ws);
  mb_campking_destroy(c->ck);
  void* ptrs[] = {c->d_nat, c->d_coord, c->d_pdiag, c->h, c->w, c->f, c->p, c->pa, c->pold, c->pold2, c->c, c->eigs,
                  c->fdiag, c->scal, c->hws, c->status, c->nrot, c->eig_ws, c->pseudo_ws,
                  c->fock_ws, c->fppf_hist, c->fock_hist, c->tc_ws_raw, c->pguess, c->purify_ws, c->pprev,
                  c->exit_ws};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

extern "C" void mb_scf_opts_default(mb_scf_opts* o) {
  o->pseudo = 0;
  o->itrmax = 2000;
  o->scfcrt = 1.0e-4;
  o->precision = 0;
  o->switch_pl = 1.0e-4;
  o->verbose = 0;
  o->pulay = 0;
  o->guess = 0;
  o->finish_dp = -1.0;
  o->finish_max = 40;
  o->bshift = -80.0;
  o->camp = 0;
}

extern "C" int mb_ctx_create(int numat, const int* nat, const double* coord, mb_ctx** out) {
  if (numat <= 0 || !nat || !out) return mb_set_error(MB_ERR_ARG, "mb_ctx_create: bad args");
  *out = nullptr;
  static Pm7Params P;
  static bool pinit = false;
  if (!pinit) { pm7_init(&P); pinit = true; }
  mb_ctx* c = new mb_ctx();
  c->numat = numat;
  c->nat.assign(nat, nat + numat);
  if (coord) c->coord.assign(coord, coord + 3 * (size_t)numat);
  else c->coord.assign(3 * (size_t)numat, 0.0);
  c->nfirst.resize(numat);
  c->nlast.resize(numat);
  int ia = 1, nelec = 0;
  for (int a = 0; a < numat; ++a) {
    if (!pm7_supported(nat[a])) { delete c; return mb_set_error(MB_ERR_UNSUPPORTED, "element outside H, C, O"); }
    const Pm7Elem& e = P.el[nat[a]];
    c->nfirst[a] = ia;
    c->nlast[a] = ia + e.natorb - 1;
    ia += e.natorb;
    nelec += (int)e.tore;
  }
  if (nelec % 2) { delete c; return mb_set_error(MB_ERR_UNSUPPORTED, "closed-shell RHF needs an even electron count"); }
  c->norbs = ia - 1;
  c->nclose = nelec / 2;
  c->mpack = (long long)c->norbs * (c->norbs + 1) / 2;
  // diagonal guess (moldat.F90:731-760) and atomic heat (mopac_api_initialize.F90:340-350)
  c->pdiag.resize(c->norbs);
  double atheat = 0.0, eat = 0.0;
  for (int a = 0; a < numat; ++a) {
    const Pm7Elem& e = P.el[nat[a]];
    for (int q = c->nfirst[a] - 1; q < c->nlast[a]; ++q) c->pdiag[q] = e.natorb == 1 ? e.tore : e.tore * 0.25;
    atheat += e.eheat;
  }
  for (int a = 0; a < numat; ++a) eat += P.el[nat[a]].eisol;
  c->atheat = atheat - eat * PM7_FPC9;
  int rc = mb_atoms_create(numat, c->nfirst.data(), c->nlast.data(), &c->atoms);
  if (rc != MB_OK) { ctx_free(c); return rc; }
  {
    std::vector<int> first, nor, lim, cum;
    std::vector<long long> wrow;
    build_layout(numat, c->nfirst.data(), c->nlast.data(), first, nor, lim, wrow, cum, &c->n2elec);
  }
  const int n = c->norbs;
  const size_t mp = (size_t)c->mpack, nn = (size_t)n * n;
  cudaError_t e = cudaSuccess;
#define ALLOC(ptr, bytes) if (e == cudaSuccess) e = cudaMalloc((void**)&(ptr), (bytes))
  ALLOC(c->d_nat, sizeof(int) * numat);
  ALLOC(c->d_coord, sizeof(double) * 3 * numat);
  ALLOC(c->d_pdiag, sizeof(double) * n);
  ALLOC(c->h, sizeof(double) * mp);
  ALLOC(c->w, sizeof(double) * (size_t)c->n2elec);
  ALLOC(c->f, sizeof(double) * mp);
  ALLOC(c->p, sizeof(double) * mp);
  ALLOC(c->pa, sizeof(double) * mp);
  ALLOC(c->pold, sizeof(double) * mp);
  ALLOC(c->pold2, sizeof(double) * n);
  ALLOC(c->c, sizeof(double) * nn);
  ALLOC(c->eigs, sizeof(double) * n);
  ALLOC(c->fdiag, sizeof(double) * mp);
  ALLOC(c->scal, sizeof(double) * 64);
  ALLOC(c->hws, sizeof(double) * 2 * n);
  ALLOC(c->status, sizeof(int) * 4);
  ALLOC(c->nrot, sizeof(unsigned long long) * 2);
  ALLOC(c->eig_ws, mb_eigh_ws_bytes(n));
#undef ALLOC
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMemcpy(c->d_nat, nat, sizeof(int) * numat, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(c->d_coord, c->coord.data(), sizeof(double) * 3 * numat, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(c->d_pdiag, c->pdiag.data(), sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(c->c, 0, sizeof(double) * nn);
  if (e == cudaSuccess) e = cudaMemset(c->eigs, 0, sizeof(double) * n);
  if (e != cudaSuccess) {
    int r = mb_set_cuda_error(e, "mb_ctx_create", __FILE__, __LINE__);
    ctx_free(c);
    return r;
  }
  *out = c;
  return MB_OK;
}

extern "C" double mb_atheat(int numat, const int* nat) {
  static Pm7Params P;
  static bool pinit = false;
  if (!pinit) { pm7_init(&P); pinit = true; }
  if (numat <= 0 || !nat) return 0.0;
  double atheat = 0.0, eat = 0.0;
  for (int a = 0; a < numat; ++a) {
    if (!pm7_supported(nat[a])) return NAN;
    atheat += P.el[nat[a]].eheat;
    eat += P.el[nat[a]].eisol;
  }
  return atheat - eat * PM7_FPC9;
}

extern "C" int mb_ctx_destroy(mb_ctx* c) {
  if (c) {
    cudaStreamSynchronize(c->stream);
    ctx_free(c);
  }
  return MB_OK;
}

extern "C" int mb_ctx_norbs(const mb_ctx* c) { return c ? c->norbs : 0; }
extern "C" long long mb_ctx_n2elec(const mb_ctx* c) { return c ? c->n2elec : 0; }
extern "C" int mb_ctx_nclose(const mb_ctx* c) { return c ? c->nclose : 0; }

extern "C" int mb_ctx_set_hw(mb_ctx* c, const double* h, const double* w, double enuclr) {
  if (!c || !h || !w) return mb_set_error(MB_ERR_ARG, "mb_ctx_set_hw: bad args");
  MB_CUDA(cudaMemcpyAsync(c->h, h, sizeof(double) * (size_t)c->mpack, cudaMemcpyHostToDevice, c->stream));
  MB_CUDA(cudaMemcpyAsync(c->w, w, sizeof(double) * (size_t)c->n2elec, cudaMemcpyHostToDevice, c->stream));
  MB_CUDA(cudaStreamSynchronize(c->stream));
  c->enuclr = enuclr;
  c->have_hw = true;
  return MB_OK;
}

extern "C" int mb_ctx_get_hw(mb_ctx* c, double* h, double* w, double* enuclr) {
  if (!c || !c->have_hw) return mb_set_error(MB_ERR_ARG, "mb_ctx_get_hw: no integrals yet");
  if (h) MB_CUDA(cudaMemcpyAsync(h, c->h, sizeof(double) * (size_t)c->mpack, cudaMemcpyDeviceToHost, c->stream));
  if (w) MB_CUDA(cudaMemcpyAsync(w, c->w, sizeof(double) * (size_t)c->n2elec, cudaMemcpyDeviceToHost, c->stream));
  MB_CUDA(cudaStreamSynchronize(c->stream));
  if (enuclr) *enuclr = c->enuclr;
  return MB_OK;
}

extern "C" int mb_ctx_hcore(mb_ctx* c) {
  if (!c) return mb_set_error(MB_ERR_ARG, "mb_ctx_hcore: null context");
  // pair energies and e1b/e2a staging live in the eigensolver workspace (idle here)
  double* enuc_pairs = (double*)c->eig_ws;
  MB_TRY(mb_hcore_dev(c->d_nat, c->d_coord, &c->atoms, c->numat, c->h, c->w, enuc_pairs, c->stream));
  MB_TRY(mb_hcore_finish(c->numat, &c->atoms, c->d_nat, c->h, nullptr, c->scal + 16, enuc_pairs, c->stream));
  double en = 0.0;
  MB_CUDA(cudaMemcpyAsync(&en, c->scal + 16, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  MB_CUDA(cudaStreamSynchronize(c->stream));
  c->enuclr = en;
  c->have_hw = true;
  return MB_OK;
}

extern "C" int mb_ctx_get_density(mb_ctx* c, double* p) {
  if (!c || !p) return mb_set_error(MB_ERR_ARG, "mb_ctx_get_density: bad args");
  MB_CUDA(cudaMemcpyAsync(p, c->p, sizeof(double) * (size_t)c->mpack, cudaMemcpyDeviceToHost, c->stream));
  MB_CUDA(cudaStreamSynchronize(c->stream));
  return MB_OK;
}

extern "C" int mb_ctx_get_vectors(mb_ctx* c, double* cv, double* eigs) {
  if (!c) return mb_set_error(MB_ERR_ARG, "mb_ctx_get_vectors: null context");
  if (cv) MB_CUDA(cudaMemcpyAsync(cv, c->c, sizeof(double) * (size_t)c->norbs * c->norbs, cudaMemcpyDeviceToHost, c->stream));
  if (eigs) MB_CUDA(cudaMemcpyAsync(eigs, c->eigs, sizeof(double) * (size_t)c->norbs, cudaMemcpyDeviceToHost, c->stream));
  MB_CUDA(cudaStreamSynchronize(c->stream));
  return MB_OK;
}

extern "C" int mb_ctx_get_fock(mb_ctx* c, double* f) {
  if (!c || !f) return mb_set_error(MB_ERR_ARG, "mb_ctx_get_fock: bad args");
  MB_CUDA(cudaMemcpyAsync(f, c->f, sizeof(double) * (size_t)c->mpack, cudaMemcpyDeviceToHost, c->stream));
  MB_CUDA(cudaStreamSynchronize(c->stream));
  return MB_OK;
}

extern "C" int mb_ctx_device_ptrs(mb_ctx* c, double** h, double** w, double** f, double** p, double** cv,
                                  double** eigs) {
  if (!c) return mb_set_error(MB_ERR_ARG, "null context");
  if (h) *h = c->h;
  if (w) *w = c->w;
  if (f) *f = c->f;
  if (p) *p = c->p;
  if (cv) *cv = c->c;
  if (eigs) *eigs = c->eigs;
  return MB_OK;
}

extern "C" size_t mb_dcart_ws_bytes(int numat);
extern "C" int mb_dcart_dev(const int* nat_d, const double* coord_d, const MbAtomsDev* at, int numat, const double* p,
                            double* dxyz_dev, void* ws, size_t ws_bytes, cudaStream_t stream);

extern "C" int mb_ctx_gradient(mb_ctx* c, double* dxyz) {
  if (!c || !dxyz) return mb_set_error(MB_ERR_ARG, "mb_ctx_gradient: bad args");
  if (!c->have_hw) return mb_set_error(MB_ERR_ARG, "mb_ctx_gradient: call mb_ctx_hcore or mb_ctx_set_hw first");
  const size_t wsb = mb_dcart_ws_bytes(c->numat), outb = sizeof(double) * 3 * (size_t)c->numat;
  char* ws = nullptr;
  MB_CUDA(mb_malloc_async((void**)&ws, wsb + outb + 256, c->stream));
  double* out = (double*)(ws + ((wsb + 255) & ~(size_t)255));
  int rc = mb_dcart_dev(c->d_nat, c->d_coord, &c->atoms, c->numat, c->p, out, ws, wsb, c->stream);
  if (rc == MB_OK && cudaMemcpyAsync(dxyz, out, outb, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
    rc = mb_set_error(MB_ERR_CUDA, "mb_ctx_gradient: copy");
  cudaFreeAsync(ws, c->stream);
  if (rc == MB_OK) MB_CUDA(cudaStreamSynchronize(c->stream));
  return rc;
}

extern "C" int mb_ctx_atoms_dev(mb_ctx* c, MbAtomsDev* out) {
  if (!c || !out) return mb_set_error(MB_ERR_ARG, "null context");
  *out = c->atoms;
  return MB_OK;
}

extern "C" int mb_guess_predict_density_ws(const mb_guess_model* m, int numat, const int* nat, const double* xyz,
                                           const int* first, const int* nor, int norbs, double* p, mb_guess_ws* w,
                                           cudaStream_t s);
extern "C" int mb_guess_ws_create(mb_guess_ws** out);
extern "C" int mb_guess_ws_destroy(mb_guess_ws* w);

static int ensure_guess_buffer(mb_ctx* c) {
  if (!c->pguess) MB_CUDA(cudaMalloc(&c->pguess, sizeof(double) * (size_t)c->mpack));
  return MB_OK;
}

extern "C" int mb_ctx_set_guess(mb_ctx* c, const double* p) {
  if (!c || !p) return mb_set_error(MB_ERR_ARG, "mb_ctx_set_guess: bad args");
  MB_TRY(ensure_guess_buffer(c));
  MB_CUDA(cudaMemcpyAsync(c->pguess, p, sizeof(double) * (size_t)c->mpack, cudaMemcpyHostToDevice, c->stream));
  MB_CUDA(cudaStreamSynchronize(c->stream));
  c->have_guess = true;
  return MB_OK;
}

extern "C" size_t mb_guess_purify_ws_bytes(int n);
extern "C" int mb_guess_purify_dev(int n, double* p, int steps, void* ws, cudaStream_t s);
extern "C" int mb_guess_purify_split_dev(int n, double* p, int steps, void* ws, void* tc_ws, size_t tc_ws_bytes,
                                         int* err_dev, cudaStream_t s);

extern "C" int mb_ctx_guess(mb_ctx* c, const mb_guess_model* m, int purify_steps) {
  if (!c || !m || purify_steps < 0) return mb_set_error(MB_ERR_ARG, "mb_ctx_guess: bad args");
  for (int a = 0; a < c->numat; ++a)
    if (c->nat[a] != 1 && c->nat[a] != 8)
      return mb_set_error(MB_ERR_UNSUPPORTED, "mb_ctx_guess: the network is trained on H and O only");
  MB_TRY(ensure_guess_buffer(c));
  if (!c->guess_ws) MB_TRY(mb_guess_ws_create(&c->guess_ws));
  c->have_guess = false;
  MB_TRY(mb_guess_predict_density_ws(m, c->numat, c->d_nat, c->d_coord, c->atoms.first, c->atoms.nor, c->norbs,
                                     c->pguess, c->guess_ws, c->stream));
  if (purify_steps > 0) {
    // the purification's three n x n matrices: the eigensolver workspace when
    // it is large enough (idle before the SCF), else a buffer the context keeps
    void* ws = c->eig_ws;
    if (mb_guess_purify_ws_bytes(c->norbs) > mb_eigh_ws_bytes(c->norbs)) {
      if (!c->purify_ws) MB_CUDA(cudaMalloc(&c->purify_ws, mb_guess_purify_ws_bytes(c->norbs)));
      ws = c->purify_ws;
    }
    // the two products per step on the tensor cores, in the split GEMM
    // workspace the SCF uses afterwards (grown here if it is smaller)
    const int n = c->norbs;
    const size_t need = mb_gemm_split_ws_bytes(n, n, n);
    if (need > c->tc_ws_bytes) {
      if (c->tc_ws_raw) cudaFree(c->tc_ws_raw);
      c->tc_ws_raw = c->tc_ws = nullptr;
      c->tc_ws_bytes = 0;
      MB_CUDA(cudaMalloc(&c->tc_ws_raw, need + 1024));
      c->tc_ws = (void*)(((uintptr_t)c->tc_ws_raw + 1023) & ~(uintptr_t)1023);
      c->tc_ws_bytes = need;
    }
    MB_CUDA(cudaMemsetAsync(c->status + 1, 0, sizeof(int), c->stream));
    MB_TRY(mb_guess_purify_split_dev(n, c->pguess, purify_steps, ws, c->tc_ws, c->tc_ws_bytes, c->status + 1,
                                     c->stream));
    int terr = 0;
    MB_CUDA(cudaMemcpyAsync(&terr, c->status + 1, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    MB_CUDA(cudaStreamSynchronize(c->stream));
    if (terr) return mb_set_error(MB_ERR_CUDA, "mb_ctx_guess: tensor-core GEMM pipeline wait expired");
  }
  MB_CUDA(cudaStreamSynchronize(c->stream));
  c->have_guess = true;
  return MB_OK;
}

// ---------------------------------------------------------------- kernels
namespace {
__global__ void half_kernel(long long n, const double* __restrict__ p, double* __restrict__ pa) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    pa[i] = p[i] * 0.5;
}
__global__ void add_tail_kernel(int n, int from, double* e, double s) {
  int i = from + blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) e[i] = e[i] + s;
}
// Starting state from a supplied density, as iter sets it up after reading
// one with OLDENS (iter.F90:151-158, RHF): pa = p/2 and pold = 2*pa.  That
// branch leaves pold2 as allocated; here it starts as the diagonal of p.
__global__ void diag_start_kernel(int n, const double* __restrict__ pdiag, double w1, double* __restrict__ p,
                                  double* __restrict__ pa, double* __restrict__ pold, double* __restrict__ pold2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long j = (long long)i * (i + 1) / 2 + i;
  const double d = pdiag[i], da = (d * w1) * 1.0;
  p[j] = d;
  pa[j] = da;
  pold[j] = da;
  pold2[i] = da;
}
__global__ void guess_start_kernel(int n, long long mpack, const double* __restrict__ g, double* __restrict__ p,
                                   double* __restrict__ pa, double* __restrict__ pold, double* __restrict__ pold2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < mpack; i += (long long)gridDim.x * blockDim.x) {
    double v = g[i];
    p[i] = v;
    pa[i] = v * 0.5;
    pold[i] = (v * 0.5) * 2.0;
  }
  for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r < n; r += (long long)gridDim.x * blockDim.x)
    pold2[r] = g[r * (r + 1) / 2 + r];
}
// out = max|p - prev| over the packed matrix (out zeroed by the caller; the
// values are >= 0, so their bit patterns order like the values), then
// prev <- p for the next iteration.
__global__ void maxdiff_copy_kernel(long long n, const double* __restrict__ p, double* __restrict__ prev,
                                    unsigned long long* __restrict__ out) {
  double m = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = p[i];
    m = fmax(m, fabs(v - prev[i]));
    prev[i] = v;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// The m x m diagonal block of M (column-major, leading dimension ld) that
// starts at (r0, r0), symmetrised and packed by rows as the eigensolver reads
// it: pk[i(i+1)/2 + j] = (M(i, j) + M(j, i)) / 2 for i >= j.  Grid (x over j,
// y = row i).
__global__ void pack_block_kernel(int m, int r0, const double* __restrict__ M, int ld, double* __restrict__ pk) {
  const int i = blockIdx.y;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m || j > i) return;
  const double a = M[(size_t)(r0 + i) + (size_t)(r0 + j) * ld];
  const double b = M[(size_t)(r0 + j) + (size_t)(r0 + i) * ld];
  pk[(long long)i * (i + 1) / 2 + j] = 0.5 * (a + b);
}

// Per-block partial sums of squares of the rows x cols block of M starting
// at M[0] (leading dimension ld); a fixed grid and a fixed tree, so the sum
// below is the same in every run.
__global__ void __launch_bounds__(256) block_sumsq_partials(int rows, int cols, const double* __restrict__ M, int ld,
                                                            double* __restrict__ part) {
  __shared__ double red[256];
  double s = 0.0;
  const long long total = (long long)rows * cols;
  for (long long q = blockIdx.x * 256LL + threadIdx.x; q < total; q += (long long)gridDim.x * 256) {
    const long long col = q / rows, row = q - col * rows;
    const double x = M[row + col * ld];
    s += x * x;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void sum_partials_kernel(int nb, const double* __restrict__ part, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double s = 0.0;
    for (int b = 0; b < nb; ++b) s += part[b];
    *out = s;
  }
}

// X(a, i) = B'(a, i) / (e_i - e_(no + a)) in place over the nv x no coupling
// in the two blocks' eigenbases: the first-order rotation between occupied
// orbital i and virtual orbital a that removes it.
__global__ void coupling_rotation_kernel(int nv, int no, const double* __restrict__ eigs, double* __restrict__ b) {
  const long long total = (long long)nv * no;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q / nv), a = (int)(q - (long long)i * nv);
    b[q] = b[q] / (eigs[i] - eigs[no + a]);
  }
}
}  // namespace

static int d2h(mb_ctx* c, double* dst, const double* src, int count) {
  MB_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * count, cudaMemcpyDeviceToHost, c->stream));
  MB_CUDA(cudaStreamSynchronize(c->stream));
  return MB_OK;
}

struct PhaseTimer {
  cudaEvent_t a, b;
  float total = 0.f;
  cudaStream_t s;
  explicit PhaseTimer(cudaStream_t st) : s(st) { cudaEventCreate(&a); cudaEventCreate(&b); }
  ~PhaseTimer() { cudaEventDestroy(a); cudaEventDestroy(b); }
  void start() { cudaEventRecord(a, s); }
  void stop() {
    cudaEventRecord(b, s);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    total += ms;
  }
};

static int full_diag(mb_ctx* c, double* fpacked, double* eig_homo, double* eig_lumo, int ihomo, int perturb = 1) {
  mb_kstat_mark(MB_KSTAT_EIGH, c->stream, true);
  MB_TRY(mb_eigh_ws(c->norbs, fpacked, perturb, c->c, c->eigs, c->eig_ws, c->status, c->stream));
  mb_kstat_mark(MB_KSTAT_EIGH, c->stream, false);
  int st = 0;
  MB_CUDA(cudaMemcpyAsync(&st, c->status, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  double hl[2] = {0.0, 0.0};
  const int n = c->norbs;
  MB_CUDA(cudaMemcpyAsync(hl, c->eigs + (ihomo - 1), sizeof(double) * (ihomo < n ? 2 : 1), cudaMemcpyDeviceToHost,
                          c->stream));
  MB_CUDA(cudaStreamSynchronize(c->stream));
  if (st != 0) return mb_set_error(MB_ERR_NUMERIC, "eigensolver failed (inverse iteration)");
  *eig_homo = hl[0];
  *eig_lumo = hl[1];
  return MB_OK;
}

static inline size_t pad32(size_t x) { return (x + 31) & ~(size_t)31; }  // doubles, to 256 bytes

// The exit diagonalisation of an SCF that ended in the FP64 finish of the
// pseudo-diagonalisation.  There the current vectors C split F into its
// occupied and virtual invariant subspaces up to a small coupling
// B = C_v^T F C_o (the finish has rotated it down with every pair active), so
// the eigenproblem of F is solved as the two diagonal blocks of M = C^T F C,
// nclose and n - nclose orbitals, on this library's eigensolver, and the
// first-order rotation X = B' / (e_o - e_v) (B' = B in the blocks'
// eigenbases) then takes the coupling out of the vectors.  The eigenvalues
// differ from those of the whole matrix by at most ||B||_2^2 / gap <=
// ||B||_F^2 / gap (the gap between the highest occupied and lowest virtual
// block eigenvalue); the split is used only when that bound is below
// 1e-8 eV, otherwise *done stays 0 and the caller runs the full eigensolve on
// fpacked, which then already carries the perturbation.  F gets the
// reference's perturbation i * 1e-10 on its diagonal first
// (eigenvectors_LAPACK.F90:53-121), in place, as the full eigensolve does.
// *coupling receives ||B||_F (eV).
static int exit_block_diag(mb_ctx* c, double* fpacked, double* eig_homo, double* eig_lumo, int* done,
                           double* coupling) {
  *done = 0;
  *coupling = -1.0;
  const int n = c->norbs, no = c->nclose, nv = n - no;
  cudaStream_t s = c->stream;
  const size_t nn = (size_t)n * n;
  const size_t o_m = 0, o_g = o_m + pad32(nn), o_ap = o_g + pad32(nn),
               o_dp = o_ap + pad32((size_t)no * (no + 1) / 2), o_qa = o_dp + pad32((size_t)nv * (nv + 1) / 2),
               o_qd = o_qa + pad32((size_t)no * no), o_t = o_qd + pad32((size_t)nv * nv),
               o_x = o_t + pad32((size_t)nv * no), o_part = o_x + pad32((size_t)nv * no), total = o_part + 1024;
  if (!c->exit_ws) MB_CUDA(cudaMalloc(&c->exit_ws, sizeof(double) * total));
  double* M = c->exit_ws + o_m;   // F full, then C^T F C
  double* G = c->exit_ws + o_g;   // F C, then the block vectors C Q
  double* Ap = c->exit_ws + o_ap;
  double* Dp = c->exit_ws + o_dp;
  double* Qa = c->exit_ws + o_qa;
  double* Qd = c->exit_ws + o_qd;
  double* T = c->exit_ws + o_t;
  double* X = c->exit_ws + o_x;
  double* part = c->exit_ws + o_part;
  mb_kstat_mark(MB_KSTAT_EIGH, s, true);
  MB_TRY(mb_unpack_dev(n, fpacked, M, n, 1, fpacked, s));
  MB_TRY(mb_dgemm_dev('N', 'N', n, n, n, 1.0, M, n, c->c, n, 0.0, G, n, s));
  MB_TRY(mb_dgemm_dev('T', 'N', n, n, n, 1.0, c->c, n, G, n, 0.0, M, n, s));
  const int nb = 148 * 4;
  block_sumsq_partials<<<nb, 256, 0, s>>>(nv, no, M + no, n, part);
  MB_LAUNCH_CHECK();
  sum_partials_kernel<<<1, 32, 0, s>>>(nb, part, part + nb);
  MB_LAUNCH_CHECK();
  double b2 = 0.0;
  MB_TRY(d2h(c, &b2, part + nb, 1));
  *coupling = sqrt(b2);
  const double tol_ev = 1.0e-8;
  // the gap is at least 1 eV wherever the split can pass the test below
  if (!(b2 <= tol_ev * 1.0e3)) {
    mb_kstat_mark(MB_KSTAT_EIGH, s, false);
    return MB_OK;
  }
  {
    dim3 ga((no + 255) / 256, no), gd((nv + 255) / 256, nv);
    pack_block_kernel<<<ga, 256, 0, s>>>(no, 0, M, n, Ap);
    MB_LAUNCH_CHECK();
    pack_block_kernel<<<gd, 256, 0, s>>>(nv, no, M, n, Dp);
    MB_LAUNCH_CHECK();
  }
  int st[2] = {0, 0};
  MB_TRY(mb_eigh_ws(no, Ap, 0, Qa, c->eigs, c->eig_ws, c->status, s));
  MB_CUDA(cudaMemcpyAsync(&st[0], c->status, sizeof(int), cudaMemcpyDeviceToHost, s));
  MB_TRY(mb_eigh_ws(nv, Dp, 0, Qd, c->eigs + no, c->eig_ws, c->status, s));
  MB_CUDA(cudaMemcpyAsync(&st[1], c->status, sizeof(int), cudaMemcpyDeviceToHost, s));
  double hl[2] = {0.0, 0.0};
  MB_CUDA(cudaMemcpyAsync(hl, c->eigs + (no - 1), sizeof(double) * 2, cudaMemcpyDeviceToHost, s));
  MB_CUDA(cudaStreamSynchronize(s));
  const double gap = hl[1] - hl[0];
  if (st[0] != 0 || st[1] != 0 || !(gap > 0.0) || !(b2 <= tol_ev * gap)) {
    mb_kstat_mark(MB_KSTAT_EIGH, s, false);
    return MB_OK;  // the full eigensolve takes over (c->c is untouched)
  }
  // B' = Qd^T B Qa (nv x no), then X = B' / (e_o - e_v)
  MB_TRY(mb_dgemm_dev('N', 'N', nv, no, no, 1.0, M + no, n, Qa, no, 0.0, T, nv, s));
  MB_TRY(mb_dgemm_dev('T', 'N', nv, no, nv, 1.0, Qd, nv, T, nv, 0.0, X, nv, s));
  {
    const long long kv = (long long)nv * no;
    int blocks = (int)((kv + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    coupling_rotation_kernel<<<blocks, 256, 0, s>>>(nv, no, c->eigs, X);
    MB_LAUNCH_CHECK();
  }
  // block vectors [C_o Qa | C_v Qd], then C_o' = C_o Qa + C_v Qd X and
  // C_v' = C_v Qd - C_o Qa X^T
  MB_TRY(mb_dgemm_dev('N', 'N', n, no, no, 1.0, c->c, n, Qa, no, 0.0, G, n, s));
  MB_TRY(mb_dgemm_dev('N', 'N', n, nv, nv, 1.0, c->c + (size_t)no * n, n, Qd, nv, 0.0, G + (size_t)no * n, n, s));
  MB_CUDA(cudaMemcpyAsync(c->c, G, sizeof(double) * nn, cudaMemcpyDeviceToDevice, s));
  MB_TRY(mb_dgemm_dev('N', 'N', n, no, nv, 1.0, G + (size_t)no * n, n, X, nv, 1.0, c->c, n, s));
  MB_TRY(mb_dgemm_dev('N', 'T', n, nv, no, -1.0, G, n, X, nv, 1.0, c->c + (size_t)no * n, n, s));
  mb_kstat_mark(MB_KSTAT_EIGH, s, false);
  *eig_homo = hl[0];
  *eig_lumo = hl[1];
  *done = 1;
  return MB_OK;
}

extern "C" int mb_scf_run(mb_ctx* c, const mb_scf_opts* opts_in, mb_scf_result* res) {
  if (!c || !res) return mb_set_error(MB_ERR_ARG, "mb_scf_run: bad args");
  if (!c->have_hw) return mb_set_error(MB_ERR_ARG, "mb_scf_run: call mb_ctx_hcore or mb_ctx_set_hw first");
  mb_scf_opts opts;
  if (opts_in) opts = *opts_in; else mb_scf_opts_default(&opts);
  memset(res, 0, sizeof(*res));
  const int n = c->norbs;
  const long long mpack = c->mpack;
  const int nclose = c->nclose;
  cudaStream_t s = c->stream;
  if (opts.pseudo && !c->pseudo_ws) MB_CUDA(cudaMalloc(&c->pseudo_ws, mb_pseudo_ws_bytes(n, nclose)));
  if (!c->fock_ws) MB_CUDA(cudaMalloc(&c->fock_ws, mb_fock2_ws_bytes(c->numat)));
  if (c->ck) {  // interp's saved state belongs to one SCF
    mb_campking_destroy(c->ck);
    c->ck = nullptr;
  }
  bool okpuly = opts.pulay != 0;
  if (okpuly) {
    if (!c->fppf_hist) MB_CUDA(cudaMalloc(&c->fppf_hist, sizeof(double) * kNpulay * (size_t)mpack));
    if (!c->fock_hist) MB_CUDA(cudaMalloc(&c->fock_hist, sizeof(double) * kNpulay * (size_t)mpack));
    // the commutator work runs in the eigensolver workspace, idle before the diagonalisation
    if (mb_pulay_ws_bytes(n) > mb_eigh_ws_bytes(n))
      return mb_set_error(MB_ERR_ARG, "mb_scf_run: Pulay workspace exceeds the eigensolver workspace");
  }
  // In the reference pold and pold2 are the heads of pulay's history arrays
  // (setup_mopac_arrays.F90:148, iter.F90:826-831): keep that aliasing.
  double* pold = okpuly ? c->fppf_hist : c->pold;
  double* pold2 = okpuly ? c->fock_hist : c->pold2;
  int modea = opts.camp ? 1 : 0;  // interp's mode (iter.F90:322-330)
  std::vector<double> emat((size_t)(kNpulay + 1) * (kNpulay + 1), 0.0);
  int lfock = 0, nfock = 0, frst = 1;
  // Split precision: density and Fmo GEMMs on the tensor cores until pl falls
  // below switch_pl; convergence is only accepted once FP64 has taken over.
  bool use_split = opts.precision != 0 && nclose > 0 && nclose < n;
  if (use_split) {
    const int nv = n - nclose, kmin = nclose < nv ? nclose : nv;
    size_t need = mb_density_split_ws_bytes(n, nclose);
    size_t g1 = mb_gemm_split_ws_bytes(n, kmin, n), g2 = mb_gemm_split_ws_bytes(nv, nclose, n);
    if (g1 > need) need = g1;
    if (g2 > need) need = g2;
    if (need > c->tc_ws_bytes) {
      if (c->tc_ws_raw) cudaFree(c->tc_ws_raw);
      c->tc_ws_raw = c->tc_ws = nullptr;
      c->tc_ws_bytes = 0;
      MB_CUDA(cudaMalloc(&c->tc_ws_raw, need + 1024));
      c->tc_ws = (void*)(((uintptr_t)c->tc_ws_raw + 1023) & ~(uintptr_t)1023);
      c->tc_ws_bytes = need;
    }
  }
  // the device wait flag of the split GEMMs and the rotation sweep
  MB_CUDA(cudaMemsetAsync(c->status + 1, 0, sizeof(int), s));
  // FP64 finish: automatic (< 0) means on for the split precision only
  const double finish_dp = opts.finish_dp < 0.0 ? (opts.precision != 0 ? 1.0e-7 : 0.0) : opts.finish_dp;
  const int finish_max = opts.finish_max > 0 ? opts.finish_max : 0;
  const bool finishing = finish_dp > 0.0 && finish_max > 0;
  double dp = finishing ? INFINITY : -1.0;  // max|P_k - P_(k-1)| of the last update
  bool refreshed = false;                   // orbital energies refreshed for the finish
  if (finishing && !c->pprev) MB_CUDA(cudaMalloc(&c->pprev, sizeof(double) * (size_t)mpack));
  PhaseTimer t_fock(s), t_diag(s), t_dens(s);
  cudaEvent_t ev_begin, ev_end;
  MB_CUDA(cudaEventCreate(&ev_begin));
  MB_CUDA(cudaEventCreate(&ev_end));
  MB_CUDA(cudaEventRecord(ev_begin, s));

  // ---- first-call setup (iter.F90:123-221)
  const double enrgy = PM7_FPC9;
  // bshift: -80 by default, -n with SHIFT=n (iter.F90:119, :131-132)
  double bshift = opts.bshift;
  double shift = 1.0, shfmax = 20.0, pl = 1.0, ten = fabs(bshift) > 1.0e-20 ? bshift : 0.0, shfto = 0.0,
         shftbo = 0.0, shiftb = 0.0;
  const double plchek = 0.005, trans = 0.2;
  bool newdg = false, oknewd = fabs(bshift) < 0.001;
  const bool halfe = false;
  bool camkin = opts.camp != 0;
  bool allcon = okpuly || camkin;  // iter.F90:142
  const int na1el = nclose, nb1el = nclose;
  const int ihomo = nclose > 1 ? nclose : 1;
  {
    // the diagonal guess: P = diag(pdiag), alpha and old densities scaled by
    // w1 (iter.F90:168-189; the reference's `random` factor alternates
    // between 1 and 1/1, so it is 1 for every orbital)
    const double w1 = na1el / (na1el + 1.0e-6 + nb1el);
    MB_CUDA(cudaMemsetAsync(c->p, 0, sizeof(double) * mpack, s));
    MB_CUDA(cudaMemsetAsync(c->pa, 0, sizeof(double) * mpack, s));
    MB_CUDA(cudaMemsetAsync(pold, 0, sizeof(double) * mpack, s));
    diag_start_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, c->d_pdiag, w1, c->p, c->pa, pold, pold2);
    MB_LAUNCH_CHECK();
  }
  if (opts.guess) {
    if (!c->have_guess) return mb_set_error(MB_ERR_ARG, "mb_scf_run: opts.guess needs mb_ctx_set_guess or mb_ctx_guess");
    guess_start_kernel<<<148, 256, 0, s>>>(n, mpack, c->pguess, c->p, c->pa, pold, pold2);
    MB_LAUNCH_CHECK();
  }
  if (finishing) MB_CUDA(cudaMemcpyAsync(c->pprev, c->p, sizeof(double) * mpack, cudaMemcpyDeviceToDevice, s));
  const double gnorm = 0.0;
  double selcon = opts.scfcrt;
  selcon = fmin(fmin(opts.scfcrt * 100.0, 0.1), fmax(opts.scfcrt * gnorm * gnorm * gnorm, opts.scfcrt));
  const double pltest = 0.05 * sqrt(fabs(selcon));
  int iredy = 1, niter = 0;
  double eold = 1.0e2, diff = 0.0, escf = 0.0, ee = 0.0, sellim = 0.0;
  const double scorr = 0.0;
  bool ready = false, converged = false;
  double eig_homo = 0.0, eig_lumo = 0.0;  // host copies of eigs(ihomo), eigs(ihomo+1)
  const int hblocks = (int)((mpack + 255) / 256 > 148 * 16 ? 148 * 16 : (mpack + 255) / 256);

  for (;;) {  // label 250
    const bool incitr = modea != 3;  // an interpolated pass is not an iteration (iter.F90:342-343)
    if (incitr) ++niter;
    if (niter > opts.itrmax) break;
    if (niter > opts.itrmax - 10 && !allcon) {
      // SWITCH ON ALL CONVERGERS (iter.F90:351-372): Pulay and Camp-King on,
      // a constant shift, and the iteration count restarts (label 180)
      if (!c->fppf_hist || !c->fock_hist) {
        if (mb_pulay_ws_bytes(n) > mb_eigh_ws_bytes(n))
          return mb_set_error(MB_ERR_ARG, "mb_scf_run: Pulay workspace exceeds the eigensolver workspace");
        if (!c->fppf_hist) MB_CUDA(cudaMalloc(&c->fppf_hist, sizeof(double) * kNpulay * (size_t)mpack));
        if (!c->fock_hist) MB_CUDA(cudaMalloc(&c->fock_hist, sizeof(double) * kNpulay * (size_t)mpack));
      }
      if (pold != c->fppf_hist) {
        // pulay's histories start at pold and pold2 (one pair of arrays in
        // the reference): carry cnvg's heads over
        MB_CUDA(cudaMemcpyAsync(c->fppf_hist, pold, sizeof(double) * mpack, cudaMemcpyDeviceToDevice, s));
        MB_CUDA(cudaMemcpyAsync(c->fock_hist, pold2, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        pold = c->fppf_hist;
        pold2 = c->fock_hist;
      }
      okpuly = true;
      camkin = !halfe;
      allcon = true;
      bshift = 4.44;
      iredy = -4;
      eold = 100.0;
      newdg = false;
      frst = 1;
      niter = 0;
      modea = camkin ? 1 : 0;
      res->forced_on = 1;
      continue;
    }
    bool use_shift = false;
    if (fabs(shift) > 1.0e-10 && bshift != 0.0) {
      if (niter > 1) {
        if (newdg && !(halfe || camkin)) {
          if (diff > 0.0) {
            shift = 1.0;
            if (diff > 1) newdg = false;
          } else {
            shift = -0.1;
          }
        } else {
          shift = (ihomo < n) ? ten + eig_lumo - eig_homo + shift : 0.0;
        }
        if (diff > 0.0) {
          if (shift > 4.0) shfmax = 4.5;
          if (shift > shfmax) shfmax = fmax(shfmax - 0.5, 0.0);
        }
        shift = fmax(-20.0, fmin(shfmax, shift));
        if (fabs(shift - shfmax) < 1.0e-5) shfmax = shfmax + 0.01;
        if (okpuly || fabs(bshift - 4.44) < 1.0e-5) {
          shift = -8.0;
          if (newdg) shift = 0.0;
        }
      }
      if (pl > plchek) {
        shftbo = shiftb;
        shfto = shift;
      } else {
        shiftb = shftbo;
        shift = shfto;
      }
      if (ihomo < n) {
        add_tail_kernel<<<(n - ihomo + 255) / 256, 256, 0, s>>>(n, ihomo, c->eigs, shift);
        MB_LAUNCH_CHECK();
        eig_lumo = eig_lumo + shift;
      }
      use_shift = true;
    }
    double cur_shift = shift;
    for (;;) {  // label 320
      t_fock.start();
      MB_TRY(mb_fock2_ws(&c->atoms, c->f, c->h, c->p, c->pa, c->w, cur_shift, use_shift ? 1 : 0, c->fock_ws,
                         mb_fock2_ws_bytes(c->numat), s));
      t_fock.stop();
      MB_TRY(mb_helect_ws(n, c->pa, c->h, c->f, c->scal, c->hws, s));
      double hee = 0.0;
      MB_TRY(d2h(c, &hee, c->scal, 1));
      ee = hee * 2.0;
      // a NaN or Inf in H, W or the density shows in the energy first: stop
      // before the eigensolver sees the Fock matrix
      if (!isfinite(ee)) return mb_set_error(MB_ERR_NUMERIC, "non-finite electronic energy (H, W or P)");
      escf = (ee + c->enuclr) * enrgy + c->atheat + scorr;
      if (!incitr) break;  // an interpolated point: no energy test (iter.F90:662)
      diff = escf - eold;
      if (diff > 0) ten = ten - 1.0;
      else ten = ten * 0.975 + 0.05;
      sellim = fmax(selcon, 1.0e-15 * fmax(fabs(ee), 1.0));
      bool conv = niter > 4 && (pl == 0.0 || (pl < pltest && fabs(diff) < sellim)) && ready;
      if (conv && use_split) {  // finish in FP64 before accepting convergence
        use_split = false;
        conv = false;
      }
      if (conv && finishing && dp > finish_dp && res->n_finish < finish_max) {
        res->n_finish++;  // FP64 finish: go on until the density stops moving
        conv = false;
      }
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
    if (incitr) {
      ready = iredy > 0 && (fabs(diff) < sellim * 10.0 || pl == 0.0);
      ++iredy;
      eold = escf;
    }
    if (opts.verbose)
      fprintf(stderr, " ITERATION %4d PLS=%10.3e ENERGY %14.6f DELTAE %13.7f shift %8.3f %s%s\n", niter, pl, escf,
              diff, shift, newdg ? "newdg" : "", incitr ? "" : " (interpolated)");
    if (niter > 2 && camkin) {  // Camp-King on the alpha vectors (iter.F90:781-798; makea is always set for RHF)
      if (!c->ck) MB_TRY(mb_campking_create(n, &c->ck));
      int mnew = modea, rot = 0;
      MB_TRY(mb_campking_interp(c->ck, na1el, modea, escf / enrgy, c->f, c->c, c->eig_ws, c->status, s, &mnew, &rot));
      modea = mnew;
      if (rot) res->n_interp++;
    }
    const bool interpolated = modea == 3;  // no Pulay, no diagonalisation, no cnvg (iter.F90:800, :888)
    if (!interpolated && newdg && okpuly && iredy > 1) {  // iter.F90:815-831
      MB_TRY(mb_pulay_ws(n, c->f, c->pa, c->fppf_hist, c->fock_hist, kNpulay, emat.data(), kNpulay + 1, &lfock,
                         &nfock, &frst, &pl, c->eig_ws, s));
      res->n_pulay++;
    }
    t_diag.start();
    if (interpolated) {
      // the density of the interpolated vectors
    } else if (newdg && opts.pseudo && !(halfe || camkin)) {
      if (res->n_finish > 0 && !refreshed) {
        // the finish's rotation angles use the energies of the current vectors
        MB_TRY(mb_orbital_energies_ws(n, c->f, c->c, c->eigs, c->eig_ws, s));
        refreshed = true;
      }
      mb_kstat_mark(MB_KSTAT_PSEUDO, s, true);
      // the finish rotates every occupied-virtual pair: neither the relative
      // threshold bigeps nor the absolute 0.05 max|Fmo| skips any (fewer
      // finish iterations to the same fixed point)
      const bool fin = res->n_finish > 0;
      MB_TRY(mb_pseudo_diag_ex(n, na1el, c->f, c->c, c->eigs, c->nrot, c->pseudo_ws, use_split ? c->tc_ws : nullptr,
                               c->tc_ws_bytes, c->status + 1, fin ? 0.0 : 1.5e-7, fin ? 0.0 : -1.0, s));
      mb_kstat_mark(MB_KSTAT_PSEUDO, s, false);
      res->n_pseudo_diag++;
    } else {
      MB_TRY(full_diag(c, c->f, &eig_homo, &eig_lumo, ihomo));
      res->n_full_diag++;
    }
    t_diag.stop();
    t_dens.start();
    if (use_split) {
      MB_TRY(mb_density_split_ws(n, nclose, 2.0, c->c, n, c->p, c->tc_ws, c->tc_ws_bytes, c->status + 1, s));
      res->n_split++;
    } else {
      MB_TRY(mb_density_dev(n, nclose, 2.0, c->c, n, c->p, s));
    }
    const bool do_cnvg = !interpolated && !(newdg && okpuly);  // iter.F90:899
    if (do_cnvg) MB_TRY(mb_cnvg_ws(n, c->p, pold, pold2, niter, c->scal + 1, c->scal + 8, s));
    half_kernel<<<hblocks, 256, 0, s>>>(mpack, c->p, c->pa);
    MB_LAUNCH_CHECK();
    if (finishing) {
      unsigned long long* dpbits = (unsigned long long*)(c->scal + 2);
      MB_CUDA(cudaMemsetAsync(dpbits, 0, sizeof(unsigned long long), s));
      maxdiff_copy_kernel<<<hblocks, 256, 0, s>>>(mpack, c->p, c->pprev, dpbits);
      MB_LAUNCH_CHECK();
    }
    t_dens.stop();
    if (do_cnvg) MB_TRY(d2h(c, &pl, c->scal + 1, 1));
    if (finishing) MB_TRY(d2h(c, &dp, c->scal + 2, 1));
    if (res->n_pseudo_diag > 0 || (opts.precision != 0 && res->n_split > 0)) {
      int terr = 0;
      MB_CUDA(cudaMemcpyAsync(&terr, c->status + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
      MB_CUDA(cudaStreamSynchronize(s));
      if (terr & 4) return mb_set_error(MB_ERR_CUDA, "rotation sweep: a dependency wait expired");
      if (terr) return mb_set_error(MB_ERR_CUDA, "tensor-core GEMM pipeline wait expired");
    }
    if (use_split && pl < opts.switch_pl) use_split = false;
    if (!isfinite(pl)) return mb_set_error(MB_ERR_NUMERIC, "non-finite density change");
    oknewd = pl < sellim || oknewd;
    newdg = (pl < trans && oknewd) || newdg;
    if (pl < trans * 0.3333) oknewd = true;
  }
  // ---- label 600: final energy and exit diagonalisation
  MB_TRY(mb_helect_ws(n, c->pa, c->h, c->f, c->scal, c->hws, s));
  double hee = 0.0;
  MB_TRY(d2h(c, &hee, c->scal, 1));
  ee = hee * 2.0;
  MB_CUDA(cudaMemcpyAsync(c->fdiag, c->f, sizeof(double) * mpack, cudaMemcpyDeviceToDevice, s));
  t_diag.start();
  int split_exit = 0;
  bool split_tried = false;
  res->exit_coupling = -1.0;
  if (converged && finishing && res->n_finish > 0 && newdg && opts.pseudo && !camkin && nclose > 0 && nclose < n) {
    split_tried = true;
    MB_TRY(exit_block_diag(c, c->fdiag, &eig_homo, &eig_lumo, &split_exit, &res->exit_coupling));
  }
  if (split_exit) {
    res->exit_split = 1;
  } else {
    // a declined split has perturbed fdiag already
    MB_TRY(full_diag(c, c->fdiag, &eig_homo, &eig_lumo, ihomo, split_tried ? 0 : 1));
    res->n_full_diag++;
  }
  t_diag.stop();
  escf = (ee + c->enuclr) * enrgy + c->atheat;
  res->escf = escf;
  res->ee = ee;
  res->niter = niter;
  res->converged = converged ? 1 : 0;
  res->pl = pl;
  res->dp = finishing ? dp : -1.0;
  res->t_fock_ms = t_fock.total;
  res->t_diag_ms = t_diag.total;
  res->t_density_ms = t_dens.total;
  MB_CUDA(cudaEventRecord(ev_end, s));
  MB_CUDA(cudaEventSynchronize(ev_end));
  float tot = 0.f;
  MB_CUDA(cudaEventElapsedTime(&tot, ev_begin, ev_end));
  cudaEventDestroy(ev_begin);
  cudaEventDestroy(ev_end);
  res->t_total_ms = tot;
  res->t_other_ms = tot - res->t_fock_ms - res->t_diag_ms - res->t_density_ms;
  if (!converged) return mb_set_error(MB_ERR_NOCONV, "UNABLE TO ACHIEVE SELF-CONSISTENCE");
  return MB_OK;
}
