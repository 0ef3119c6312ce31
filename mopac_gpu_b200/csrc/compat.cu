// Reference-facing entry points.
//
// (1) The bind(C) symbols of the reference's src/gpu/cuda_wrappers.cu with
//     identical signatures (host pointers, synchronous, void return), so a
//     Fortran build that links the reference's wrappers links this library
//     instead.  Device buffers are cached grow-only, like the reference's
//     DevBuf (cuda_wrappers.cu:11-28); errors, which the reference ignores,
//     are reported through mb_last_error() and, for the eigensolver, info.
// (2) Fortran-callable shims (gfortran mangling, by-reference arguments) for
//     the routines iter calls, so a gfortran-built iter can link them.
#include <string.h>

#include <mutex>
#include <vector>

#include "mb_common.cuh"

extern "C" int mb_eigh_ws(int n, double* fpacked, int perturb, double* c, double* eigs, void* ws, int* status_dev,
                          cudaStream_t stream);
extern "C" size_t mb_eigh_ws_bytes(int n);
extern "C" int mb_density_occ_dev(int n, int ndubl, int nsingl, double occ, double fract, int mode, int iopc,
                                  const double* c, int ldc, double* p, cudaStream_t stream);
extern "C" size_t mb_pseudo_ws_bytes(int n, int nocc);
extern "C" int mb_pseudo_diag_ws(int n, int nocc, const double* fpacked, double* c, const double* eigs,
                                 unsigned long long* nrot_dev, void* ws, cudaStream_t stream);
extern "C" int mb_rot_sweep_ws(int n, int nocc, const double* fmo, const double* eigs, double* c, double bigeps,
                               double tiny, unsigned long long* nrot_dev, void* ws, cudaStream_t stream);
extern "C" int mb_cnvg_ws(int norbs, double* pnew, double* p, double* p1, int niter, double* pl_out, double* ws,
                          cudaStream_t stream);
extern "C" int mb_helect_ws(int n, const double* p, const double* h, const double* f, double* out, double* ws,
                            cudaStream_t stream);
extern "C" size_t mb_pulay_ws_bytes(int n);
extern "C" int mb_pulay_ws(int n, double* f, const double* p, double* fppf, double* fock, int mfock, double* emat,
                           int ldemat, int* lfock, int* nfock, int* start, double* pl, void* ws, cudaStream_t stream);

namespace {

// Grow-only device buffer cache (one set per process, serialised by a mutex;
// the reference layer is not thread-safe at all).
struct Buf {
  void* p = nullptr;
  size_t cap = 0;
  int get(size_t bytes) {
    if (bytes <= cap) return MB_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    MB_CUDA(cudaMalloc(&p, bytes));
    cap = bytes;
    return MB_OK;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

std::mutex g_mu;
Buf g_a, g_b, g_c, g_d, g_ws;
cudaStream_t g_stream = nullptr;
int g_norbs_fortran = 0;
int g_npulay_fortran = 10;  // molkst_C.F90:114-115
int g_mfock_fortran = 0;    // pulay's saved mfock (pulay.F90:40, :57-59)

int ensure_stream() {
  if (!g_stream) MB_CUDA(cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking));
  return MB_OK;
}

// copy a (rows x cols, leading dim ld) host matrix to a dense device one (ld = rows)
int h2d_mat(double* dst, const double* src, int rows, int cols, int ld) {
  if (rows <= 0 || cols <= 0) return MB_OK;
  MB_CUDA(cudaMemcpy2DAsync(dst, sizeof(double) * rows, src, sizeof(double) * ld, sizeof(double) * rows, cols,
                            cudaMemcpyHostToDevice, g_stream));
  return MB_OK;
}
int d2h_mat(double* dst, const double* src, int rows, int cols, int ld) {
  if (rows <= 0 || cols <= 0) return MB_OK;
  MB_CUDA(cudaMemcpy2DAsync(dst, sizeof(double) * ld, src, sizeof(double) * rows, sizeof(double) * rows, cols,
                            cudaMemcpyDeviceToHost, g_stream));
  return MB_OK;
}

bool is_t(char c) { return c == 'T' || c == 't' || c == 'C' || c == 'c'; }

int gemm_host(char tra, char trb, int m, int n, int k, double alpha, const double* A, int lda, const double* B,
              int ldb, double beta, double* C, int ldc) {
  if (m <= 0 || n <= 0) return MB_OK;
  MB_TRY(ensure_stream());
  const int ar = is_t(tra) ? k : m, ac = is_t(tra) ? m : k;
  const int br = is_t(trb) ? n : k, bc = is_t(trb) ? k : n;
  MB_TRY(g_a.get(sizeof(double) * (size_t)ar * ac + 8));
  MB_TRY(g_b.get(sizeof(double) * (size_t)br * bc + 8));
  MB_TRY(g_c.get(sizeof(double) * (size_t)m * n));
  MB_TRY(h2d_mat((double*)g_a.p, A, ar, ac, lda));
  MB_TRY(h2d_mat((double*)g_b.p, B, br, bc, ldb));
  if (beta != 0.0) MB_TRY(h2d_mat((double*)g_c.p, C, m, n, ldc));
  MB_TRY(mb_dgemm_dev(tra, trb, m, n, k, alpha, (const double*)g_a.p, ar > 0 ? ar : 1, (const double*)g_b.p,
                      br > 0 ? br : 1, beta, (double*)g_c.p, m, g_stream));
  MB_TRY(d2h_mat(C, (const double*)g_c.p, m, n, ldc));
  MB_CUDA(cudaStreamSynchronize(g_stream));
  return MB_OK;
}

__global__ void keep_triangle(int n, const double* __restrict__ full, double* __restrict__ c, int upper) {
  const int col = blockIdx.y;
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x)
    if (upper ? row <= col : row >= col) c[(long long)col * n + row] = full[(long long)col * n + row];
}

int syrk_host(char uplo, char tra, int n, int k, double alpha, const double* A, int lda, double beta, double* C,
              int ldc) {
  if (n <= 0) return MB_OK;
  MB_TRY(ensure_stream());
  const bool t = is_t(tra);
  const int ar = t ? k : n, ac = t ? n : k;
  MB_TRY(g_a.get(sizeof(double) * (size_t)ar * ac + 8));
  MB_TRY(g_c.get(sizeof(double) * (size_t)n * n));
  MB_TRY(g_d.get(sizeof(double) * (size_t)n * n));
  MB_TRY(h2d_mat((double*)g_a.p, A, ar, ac, lda));
  MB_TRY(h2d_mat((double*)g_c.p, C, n, n, ldc));
  MB_CUDA(cudaMemcpyAsync(g_d.p, g_c.p, sizeof(double) * (size_t)n * n, cudaMemcpyDeviceToDevice, g_stream));
  // full product into d (both triangles), then keep only the requested one
  MB_TRY(mb_dgemm_dev(t ? 'T' : 'N', t ? 'N' : 'T', n, n, k, alpha, (const double*)g_a.p, ar > 0 ? ar : 1,
                      (const double*)g_a.p, ar > 0 ? ar : 1, beta, (double*)g_d.p, n, g_stream));
  dim3 grid((n + 255) / 256, n);
  keep_triangle<<<grid, 256, 0, g_stream>>>(n, (const double*)g_d.p, (double*)g_c.p,
                                            (uplo == 'U' || uplo == 'u') ? 1 : 0);
  MB_LAUNCH_CHECK();
  MB_TRY(d2h_mat(C, (const double*)g_c.p, n, n, ldc));
  MB_CUDA(cudaStreamSynchronize(g_stream));
  return MB_OK;
}

__global__ void pack_upper(int n, const double* __restrict__ a, int lda, double* __restrict__ pk) {
  const int col = blockIdx.y;
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row <= col; row += gridDim.x * blockDim.x)
    pk[mb_tri(col, row)] = a[(long long)col * lda + row];
}

int eigh_host(int n, const double* A_upper, int lda, double* vecs, int ldv, double* w, double* fpacked_host,
              int perturb) {
  MB_TRY(ensure_stream());
  const size_t mp = (size_t)n * (n + 1) / 2, nn = (size_t)n * n;
  MB_TRY(g_a.get(sizeof(double) * (nn > mp ? nn : mp)));
  MB_TRY(g_b.get(sizeof(double) * mp));
  MB_TRY(g_c.get(sizeof(double) * (nn + n)));
  MB_TRY(g_ws.get(mb_eigh_ws_bytes(n) + 64));
  double* pk = (double*)g_b.p;
  if (fpacked_host) {
    MB_CUDA(cudaMemcpyAsync(pk, fpacked_host, sizeof(double) * mp, cudaMemcpyHostToDevice, g_stream));
  } else {
    MB_TRY(h2d_mat((double*)g_a.p, A_upper, n, n, lda));
    dim3 grid((n + 255) / 256, n);
    pack_upper<<<grid, 256, 0, g_stream>>>(n, (const double*)g_a.p, n, pk);
    MB_LAUNCH_CHECK();
  }
  double* cv = (double*)g_c.p;
  double* ev = cv + nn;
  int* st = (int*)((char*)g_ws.p + mb_eigh_ws_bytes(n));
  MB_TRY(mb_eigh_ws(n, pk, perturb, cv, ev, g_ws.p, st, g_stream));
  int hst = 0;
  MB_CUDA(cudaMemcpyAsync(&hst, st, sizeof(int), cudaMemcpyDeviceToHost, g_stream));
  MB_TRY(d2h_mat(vecs, cv, n, n, ldv));
  MB_CUDA(cudaMemcpyAsync(w, ev, sizeof(double) * n, cudaMemcpyDeviceToHost, g_stream));
  if (fpacked_host && perturb)
    MB_CUDA(cudaMemcpyAsync(fpacked_host, pk, sizeof(double) * mp, cudaMemcpyDeviceToHost, g_stream));
  MB_CUDA(cudaStreamSynchronize(g_stream));
  if (hst != 0) return mb_set_error(MB_ERR_NUMERIC, "eigensolver: inverse iteration failed");
  return MB_OK;
}

void report(int rc, const char* where) {
  if (rc != MB_OK) fprintf(stderr, "mopac_b200 %s: %s\n", where, mb_last_error());
}

}  // namespace

// ============================================================ (1) bind(C)
extern "C" void call_gemm_cublas(char tra, char trb, int m, int n, int k, double alpha, const double* A, int lda,
                                 const double* B, int ldb, double beta, double* C, int ldc) {
  std::lock_guard<std::mutex> lk(g_mu);
  report(gemm_host(tra, trb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc), "call_gemm_cublas");
}

extern "C" void call_syrk_cublas(char uplo, char tra, int n, int k, double alpha, const double* A, int lda,
                                 double beta, double* C, int ldc) {
  std::lock_guard<std::mutex> lk(g_mu);
  report(syrk_host(uplo, tra, n, k, alpha, A, lda, beta, C, ldc), "call_syrk_cublas");
}

extern "C" void call_gemm_cublas_2gpu(char tra, char trb, int m, int n, int k, double alpha, const double* A,
                                      int lda, const double* B, int ldb, double beta, double* C, int ldc) {
  call_gemm_cublas(tra, trb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
}

extern "C" void call_syrk_cublas_2gpu(char uplo, char tra, int n, int k, double alpha, const double* A, int lda,
                                      double beta, double* C, int ldc) {
  call_syrk_cublas(uplo, tra, n, k, alpha, A, lda, beta, C, ldc);
}

extern "C" void mopac_cuda_dsyevd(int n, double* A, int lda, double* W, int* info) {
  std::lock_guard<std::mutex> lk(g_mu);
  int rc = (n <= 0 || lda < n) ? mb_set_error(MB_ERR_ARG, "mopac_cuda_dsyevd: bad size")
                               : eigh_host(n, A, lda, A, lda, W, nullptr, 0);
  report(rc, "mopac_cuda_dsyevd");
  if (info) *info = rc == MB_OK ? 0 : -rc;
}

extern "C" void call_rot_cuda_gpu(const double* fmo, const double* eig, double* vector, const double* ci0,
                                  const double* ca0, int nocc, int lumo, int n, double bigeps, double tiny) {
  (void)ci0; (void)ca0;
  std::lock_guard<std::mutex> lk(g_mu);
  int rc = MB_OK;
  const int nv = n - (lumo - 1);
  if (nocc <= 0 || nv <= 0 || lumo - 1 != nocc) {
    rc = (nocc <= 0 || nv <= 0) ? MB_OK : mb_set_error(MB_ERR_ARG, "call_rot_cuda_gpu: lumo must be nocc + 1");
  } else {
    rc = ensure_stream();
    if (rc == MB_OK) rc = g_a.get(sizeof(double) * (size_t)nocc * nv);
    if (rc == MB_OK) rc = g_b.get(sizeof(double) * (size_t)n + 64);
    if (rc == MB_OK) rc = g_c.get(sizeof(double) * (size_t)n * n);
    if (rc == MB_OK) rc = g_ws.get(mb_pseudo_ws_bytes(n, nocc) + 64);
    unsigned long long* nr = (unsigned long long*)((char*)g_b.p + sizeof(double) * (size_t)n);
    if (rc == MB_OK && cudaMemcpyAsync(g_a.p, fmo, sizeof(double) * (size_t)nocc * nv, cudaMemcpyHostToDevice, g_stream) != cudaSuccess) rc = MB_ERR_CUDA;
    if (rc == MB_OK && cudaMemcpyAsync(g_b.p, eig, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, g_stream) != cudaSuccess) rc = MB_ERR_CUDA;
    if (rc == MB_OK && cudaMemcpyAsync(g_c.p, vector, sizeof(double) * (size_t)n * n, cudaMemcpyHostToDevice, g_stream) != cudaSuccess) rc = MB_ERR_CUDA;
    if (rc == MB_OK)
      rc = mb_rot_sweep_ws(n, nocc, (const double*)g_a.p, (const double*)g_b.p, (double*)g_c.p, bigeps, tiny, nr,
                           g_ws.p, g_stream);
    if (rc == MB_OK && cudaMemcpyAsync(vector, g_c.p, sizeof(double) * (size_t)n * n, cudaMemcpyDeviceToHost, g_stream) != cudaSuccess) rc = MB_ERR_CUDA;
    if (rc == MB_OK && cudaStreamSynchronize(g_stream) != cudaSuccess) rc = MB_ERR_CUDA;
  }
  report(rc, "call_rot_cuda_gpu");
}

extern "C" void call_rot_cuda_2gpu_gpu(const double* fmo, const double* eig, double* vector, const double* ci0,
                                       const double* ca0, int nocc, int lumo, int n, double bigeps, double tiny) {
  call_rot_cuda_gpu(fmo, eig, vector, ci0, ca0, nocc, lumo, n, bigeps, tiny);
}

extern "C" void getGPUInfo(bool* hasGpu, bool* hasDouble, int* nDevices, char (*name)[256], int* name_size,
                           size_t* totalMem, int* clockRate, int* major, int* minor) {
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess) nd = 0;
  if (hasGpu) *hasGpu = nd > 0;
  if (nDevices) *nDevices = nd;
  for (int i = 0; i < nd && i < 6; ++i) {
    cudaDeviceProp pr;
    if (cudaGetDeviceProperties(&pr, i) != cudaSuccess) continue;
    if (hasDouble) hasDouble[i] = pr.major >= 2;
    if (name) {
      strncpy(name[i], pr.name, 255);
      name[i][255] = 0;
    }
    if (name_size) name_size[i] = (int)strlen(pr.name);
    if (totalMem) totalMem[i] = pr.totalGlobalMem;
    int clk = 0;
    cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, i);
    if (clockRate) clockRate[i] = clk;
    if (major) major[i] = pr.major;
    if (minor) minor[i] = pr.minor;
  }
}

extern "C" void setDevice(int idevice, bool* stat) {
  cudaError_t e = cudaSetDevice(idevice);
  if (stat) *stat = e == cudaSuccess;
}

extern "C" void set_mozyme_gpu_pair(int dev0, int dev1) { (void)dev0; (void)dev1; }
extern "C" void create_handle(void) {}
extern "C" void destroy_handle(void) {}

void mz_release_bound();  // the MOZYME shims' registered system (below)

extern "C" void mopac_cuda_destroy_resources(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_a.release(); g_b.release(); g_c.release(); g_d.release(); g_ws.release();
  mz_release_bound();
  if (g_stream) { cudaStreamDestroy(g_stream); g_stream = nullptr; }
}

// ====================================================== (2) Fortran shims
// molkst_C's norbs for cnvg_, which takes it from the module, not an argument.
extern "C" void mb_set_norbs_(const int* norbs) { g_norbs_fortran = norbs ? *norbs : 0; }

extern "C" void fock2_(double* f, const double* ptot, const double* p, const double* w, const double* wj,
                       const double* wk, const int* numat, const int* nfirst, const int* nlast, const int* mode) {
  (void)wj; (void)wk;
  std::lock_guard<std::mutex> lk(g_mu);
  int rc = MB_OK;
  const int na = numat ? *numat : 0;
  if (na <= 0 || !mode || *mode != 2) {
    report(mb_set_error(MB_ERR_UNSUPPORTED, "fock2_: numat > 0 and mode 2 only"), "fock2_");
    return;
  }
  MbAtomsDev at{};
  rc = mb_atoms_create(na, nfirst, nlast, &at);
  const int norbs = nlast[na - 1];
  const size_t mp = (size_t)norbs * (norbs + 1) / 2;
  long long n2 = 0;
  for (int a = 0; a < na; ++a) {
    long long li = (long long)(nlast[a] - nfirst[a] + 1) * (nlast[a] - nfirst[a] + 2) / 2, s = 0;
    for (int b = 0; b < a; ++b) s += (long long)(nlast[b] - nfirst[b] + 1) * (nlast[b] - nfirst[b] + 2) / 2;
    n2 += li * s + li * li;
  }
  if (rc == MB_OK) rc = ensure_stream();
  if (rc == MB_OK) rc = g_a.get(sizeof(double) * mp * 3);
  if (rc == MB_OK) rc = g_b.get(sizeof(double) * (size_t)n2);
  double *df = (double*)g_a.p, *dpt = df + mp, *dpa = dpt + mp;
  if (rc == MB_OK && (cudaMemcpyAsync(df, f, sizeof(double) * mp, cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(dpt, ptot, sizeof(double) * mp, cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(dpa, p, sizeof(double) * mp, cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(g_b.p, w, sizeof(double) * (size_t)n2, cudaMemcpyHostToDevice, g_stream) != cudaSuccess))
    rc = MB_ERR_CUDA;
  // F arrives holding the start value; use_shift = 0 with h = f reproduces "f += ..."
  if (rc == MB_OK) rc = mb_fock2_dev(&at, df, df, dpt, dpa, (const double*)g_b.p, 0.0, 0, g_stream);
  if (rc == MB_OK && cudaMemcpyAsync(f, df, sizeof(double) * mp, cudaMemcpyDeviceToHost, g_stream) != cudaSuccess)
    rc = MB_ERR_CUDA;
  if (rc == MB_OK && cudaStreamSynchronize(g_stream) != cudaSuccess) rc = MB_ERR_CUDA;
  mb_atoms_destroy(&at);
  report(rc, "fock2_");
}

extern "C" long long mb_dfock2_w_len(int numat, const int* nfirst, const int* nlast, int nati);
extern "C" int mb_dfock2_dev(int numat, const int* nfirst, const int* nlast, int nati, double* f, const double* ptot,
                             const double* p, const double* w, cudaStream_t s);

extern "C" void dfock2_(double* f, const double* ptot, const double* p, const double* w, const int* numat,
                        const int* nfirst, const int* nlast, const int* nati) {
  std::lock_guard<std::mutex> lk(g_mu);
  const int na = numat ? *numat : 0;
  const long long nw = (na > 0 && nati) ? mb_dfock2_w_len(na, nfirst, nlast, *nati) : -1;
  if (nw < 0 || !f || !ptot || !p || !w) {
    report(mb_set_error(MB_ERR_ARG, "dfock2_: bad arguments or an atom with d orbitals"), "dfock2_");
    return;
  }
  const int norbs = nlast[na - 1];
  const size_t mp = (size_t)norbs * (norbs + 1) / 2;
  int rc = ensure_stream();
  if (rc == MB_OK) rc = g_a.get(sizeof(double) * mp * 3);
  if (rc == MB_OK) rc = g_b.get(sizeof(double) * (size_t)(nw > 0 ? nw : 1));
  double *df = (double*)g_a.p, *dpt = df + mp, *dp = dpt + mp;
  if (rc == MB_OK && (cudaMemcpyAsync(df, f, sizeof(double) * mp, cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(dpt, ptot, sizeof(double) * mp, cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(dp, p, sizeof(double) * mp, cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
                      (nw > 0 && cudaMemcpyAsync(g_b.p, w, sizeof(double) * (size_t)nw, cudaMemcpyHostToDevice,
                                                 g_stream) != cudaSuccess)))
    rc = MB_ERR_CUDA;
  if (rc == MB_OK) rc = mb_dfock2_dev(na, nfirst, nlast, *nati, df, dpt, dp, (const double*)g_b.p, g_stream);
  if (rc == MB_OK && cudaMemcpyAsync(f, df, sizeof(double) * mp, cudaMemcpyDeviceToHost, g_stream) != cudaSuccess)
    rc = MB_ERR_CUDA;
  if (rc == MB_OK && cudaStreamSynchronize(g_stream) != cudaSuccess) rc = MB_ERR_CUDA;
  report(rc, "dfock2_");
}

extern "C" double helect_(const int* n, const double* p, const double* h, const double* f) {
  std::lock_guard<std::mutex> lk(g_mu);
  const int nn = *n;
  const size_t mp = (size_t)nn * (nn + 1) / 2;
  double out = 0.0;
  int rc = ensure_stream();
  if (rc == MB_OK) rc = g_a.get(sizeof(double) * (mp * 3 + 2 * (size_t)nn + 2));
  double* d = (double*)g_a.p;
  if (rc == MB_OK && (cudaMemcpyAsync(d, p, sizeof(double) * mp, cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(d + mp, h, sizeof(double) * mp, cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(d + 2 * mp, f, sizeof(double) * mp, cudaMemcpyHostToDevice, g_stream) != cudaSuccess))
    rc = MB_ERR_CUDA;
  if (rc == MB_OK) rc = mb_helect_ws(nn, d, d + mp, d + 2 * mp, d + 3 * mp + 2 * nn, d + 3 * mp, g_stream);
  if (rc == MB_OK && cudaMemcpyAsync(&out, d + 3 * mp + 2 * nn, sizeof(double), cudaMemcpyDeviceToHost, g_stream) != cudaSuccess)
    rc = MB_ERR_CUDA;
  if (rc == MB_OK && cudaStreamSynchronize(g_stream) != cudaSuccess) rc = MB_ERR_CUDA;
  report(rc, "helect_");
  return out;
}

extern "C" void cnvg_(double* pnew, double* p, double* p1, const int* niter, double* pl) {
  std::lock_guard<std::mutex> lk(g_mu);
  const int n = g_norbs_fortran;
  if (n <= 0) {
    report(mb_set_error(MB_ERR_ARG, "cnvg_: call mb_set_norbs_ first"), "cnvg_");
    return;
  }
  const size_t mp = (size_t)n * (n + 1) / 2;
  int rc = ensure_stream();
  if (rc == MB_OK) rc = g_a.get(sizeof(double) * (2 * mp + (size_t)n + 8));
  double* d = (double*)g_a.p;
  double *dpn = d, *dp = d + mp, *dp1 = d + 2 * mp, *ws = dp1 + n;
  if (rc == MB_OK && (cudaMemcpyAsync(dpn, pnew, sizeof(double) * mp, cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(dp, p, sizeof(double) * mp, cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(dp1, p1, sizeof(double) * n, cudaMemcpyHostToDevice, g_stream) != cudaSuccess))
    rc = MB_ERR_CUDA;
  if (rc == MB_OK) rc = mb_cnvg_ws(n, dpn, dp, dp1, *niter, ws + 4, ws, g_stream);
  if (rc == MB_OK && (cudaMemcpyAsync(pnew, dpn, sizeof(double) * mp, cudaMemcpyDeviceToHost, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(p, dp, sizeof(double) * mp, cudaMemcpyDeviceToHost, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(p1, dp1, sizeof(double) * n, cudaMemcpyDeviceToHost, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(pl, ws + 4, sizeof(double), cudaMemcpyDeviceToHost, g_stream) != cudaSuccess))
    rc = MB_ERR_CUDA;
  if (rc == MB_OK && cudaStreamSynchronize(g_stream) != cudaSuccess) rc = MB_ERR_CUDA;
  report(rc, "cnvg_");
}

extern "C" void density_for_gpu_(const double* c, const double* fract, const int* ndubl, const int* nsingl,
                                 const double* occ, const int* mpack, const int* norbs, const int* mode, double* pp,
                                 const int* iopc) {
  (void)mpack;
  std::lock_guard<std::mutex> lk(g_mu);
  const int n = *norbs;
  const size_t mp = (size_t)n * (n + 1) / 2;
  int rc = ensure_stream();
  if (rc == MB_OK) rc = g_a.get(sizeof(double) * (size_t)n * n);
  if (rc == MB_OK) rc = g_b.get(sizeof(double) * mp);
  if (rc == MB_OK && cudaMemcpyAsync(g_a.p, c, sizeof(double) * (size_t)n * n, cudaMemcpyHostToDevice, g_stream) != cudaSuccess)
    rc = MB_ERR_CUDA;
  if (rc == MB_OK)
    rc = mb_density_occ_dev(n, *ndubl, *nsingl, *occ, *fract, *mode, *iopc, (const double*)g_a.p, n, (double*)g_b.p,
                            g_stream);
  if (rc == MB_OK && cudaMemcpyAsync(pp, g_b.p, sizeof(double) * mp, cudaMemcpyDeviceToHost, g_stream) != cudaSuccess)
    rc = MB_ERR_CUDA;
  if (rc == MB_OK && cudaStreamSynchronize(g_stream) != cudaSuccess) rc = MB_ERR_CUDA;
  report(rc, "density_for_gpu_");
}

extern "C" void eigenvectors_lapack_(double* eigenvecs, double* xmat, double* eigvals, const int* ndim) {
  std::lock_guard<std::mutex> lk(g_mu);
  const int n = *ndim;
  report(eigh_host(n, nullptr, n, eigenvecs, n, eigvals, xmat, 1), "eigenvectors_lapack_");
}

extern "C" void diag_for_gpu_(const double* fao, double* vector, const int* nocc, const double* eig, const int* norbs,
                              const int* mpack) {
  (void)mpack;
  std::lock_guard<std::mutex> lk(g_mu);
  const int n = *norbs, k = *nocc;
  if (k == n || k == 0) return;
  const size_t mp = (size_t)n * (n + 1) / 2;
  int rc = ensure_stream();
  if (rc == MB_OK) rc = g_a.get(sizeof(double) * mp);
  if (rc == MB_OK) rc = g_b.get(sizeof(double) * (size_t)n + 64);
  if (rc == MB_OK) rc = g_c.get(sizeof(double) * (size_t)n * n);
  if (rc == MB_OK) rc = g_ws.get(mb_pseudo_ws_bytes(n, k) + 64);
  unsigned long long* nr = (unsigned long long*)((char*)g_b.p + sizeof(double) * (size_t)n);
  if (rc == MB_OK && (cudaMemcpyAsync(g_a.p, fao, sizeof(double) * mp, cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(g_b.p, eig, sizeof(double) * n, cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(g_c.p, vector, sizeof(double) * (size_t)n * n, cudaMemcpyHostToDevice, g_stream) != cudaSuccess))
    rc = MB_ERR_CUDA;
  if (rc == MB_OK)
    rc = mb_pseudo_diag_ws(n, k, (const double*)g_a.p, (double*)g_c.p, (const double*)g_b.p, nr, g_ws.p, g_stream);
  if (rc == MB_OK && cudaMemcpyAsync(vector, g_c.p, sizeof(double) * (size_t)n * n, cudaMemcpyDeviceToHost, g_stream) != cudaSuccess)
    rc = MB_ERR_CUDA;
  if (rc == MB_OK && cudaStreamSynchronize(g_stream) != cudaSuccess) rc = MB_ERR_CUDA;
  report(rc, "diag_for_gpu_");
}

extern "C" void mb_set_npulay_(const int* npulay) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (npulay && *npulay > 0) g_npulay_fortran = *npulay;
}

extern "C" void pulay_(double* f, const double* p, const int* n, double* fppf, double* fock, double* emat,
                       int* lfock, int* nfock, const int* msize, int* start, double* pl) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!n || *n <= 0 || !msize) {
    report(mb_set_error(MB_ERR_ARG, "pulay_: bad size"), "pulay_");
    return;
  }
  const int nn = *n;
  const size_t lin = (size_t)nn * (nn + 1) / 2;
  if (*start) {
    int mf = (int)((size_t)*msize / lin);
    g_mfock_fortran = mf < g_npulay_fortran ? mf : g_npulay_fortran;
  }
  const int mfock = g_mfock_fortran;
  if (mfock < 1) {
    report(mb_set_error(MB_ERR_ARG, "pulay_: msize holds no history entry"), "pulay_");
    return;
  }
  const size_t hist = lin * (size_t)mfock;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  int rc = ensure_stream();
  if (rc == MB_OK) rc = g_a.get(al(sizeof(double) * lin) * 2 + al(sizeof(double) * hist) * 2);
  if (rc == MB_OK) rc = g_ws.get(mb_pulay_ws_bytes(nn));
  if (rc != MB_OK) { report(rc, "pulay_"); return; }
  char* b = (char*)g_a.p;
  double* df = (double*)b; b += al(sizeof(double) * lin);
  double* dp = (double*)b; b += al(sizeof(double) * lin);
  double* dfppf = (double*)b; b += al(sizeof(double) * hist);
  double* dfock = (double*)b;
  if (cudaMemcpyAsync(df, f, sizeof(double) * lin, cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
      cudaMemcpyAsync(dp, p, sizeof(double) * lin, cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
      cudaMemcpyAsync(dfppf, fppf, sizeof(double) * hist, cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
      cudaMemcpyAsync(dfock, fock, sizeof(double) * hist, cudaMemcpyHostToDevice, g_stream) != cudaSuccess)
    rc = MB_ERR_CUDA;
  if (rc == MB_OK)
    rc = mb_pulay_ws(nn, df, dp, dfppf, dfock, mfock, emat, g_npulay_fortran + 1, lfock, nfock, start, pl, g_ws.p,
                     g_stream);
  if (rc == MB_OK && (cudaMemcpyAsync(f, df, sizeof(double) * lin, cudaMemcpyDeviceToHost, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(fppf, dfppf, sizeof(double) * hist, cudaMemcpyDeviceToHost, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(fock, dfock, sizeof(double) * hist, cudaMemcpyDeviceToHost, g_stream) != cudaSuccess))
    rc = MB_ERR_CUDA;
  if (rc == MB_OK && cudaStreamSynchronize(g_stream) != cudaSuccess) rc = MB_ERR_CUDA;
  report(rc, "pulay_");
}

// ====================================================== (2) MOZYME shims
// The reference's MOZYME routines read their LMOs and storage tables from
// module MOZYME_C and common_arrays_C.  A C library cannot see Fortran
// module variables, so the host registers them once (mb_mz_bind_system_ after
// fillij / hcore_for_MOZYME, mb_mz_bind_lmos_ whenever the arrays are
// (re)allocated, e.g. after tidy repacks them) and the three shims then take
// the reference's own argument lists.  Every call stages the registered host
// arrays through the device kernels and writes the results back to them, as
// the reference's own GPU layer stages its matrices: the host arrays stay the
// truth between calls.
extern "C" int mb_mz_layout_create(int numat, const int* iorbs, const double* coord, double cutof1, double cutof2,
                                   MbMzLayout* out, long long* nijbo);
extern "C" int mb_mz_layout_destroy(MbMzLayout* layout);
extern "C" int mb_mz_lmos_create(int numat, const int* iorbs, int nlmo, const int* ncf, const int* nncf,
                                 const int* icocc, const int* ncocc, const double* cocc, long long icocc_dim,
                                 long long cocc_dim, MbMzLmos* out);
extern "C" int mb_mz_lmos_refresh(int numat, const int* iorbs_host, MbMzLmos* lmos);
extern "C" int mb_mz_lmos_destroy(MbMzLmos* lmos);
extern "C" int mb_mz_density_dev(const MbMzLayout* layout, const MbMzLmos* lmos, int mode, const double* partp,
                                 double* p, cudaStream_t stream);
extern "C" size_t mb_mz_fock_ws_bytes(const MbMzLayout* layout);
extern "C" int mb_mz_fock_dev(const MbMzLayout* layout, const double* coord, const double* w, const double* ptot,
                              const double* h, double* f, void* ws, cudaStream_t stream);
extern "C" size_t mb_mz_diagg1_ws_bytes(const MbMzLayout* layout, const MbMzLmos* occ, const MbMzLmos* vir);
extern "C" int mb_mz_diagg1_dev(const MbMzLayout* layout, const MbMzLmos* occ, const MbMzLmos* vir, const double* fao,
                                const double* p, int idiagg, double* state, int* nfmo, int* ifmo, double* fmo,
                                long long* nij, double* eigv, double* eigs, int* eigs_done, double* sumt, void* ws,
                                cudaStream_t stream);
extern "C" int mb_mz_diagg2_dev(const MbMzLayout* layout, MbMzLmos* occ, MbMzLmos* vir, const int* ifmo,
                                const double* fmo, long long nij, const double* eigs, const double* eigv, int idiagg,
                                const double* ctl, int* nrejct, double* sumb, long long* nrej, cudaStream_t stream);

namespace {
struct MzBound {
  bool have_system = false, have_lmos = false;
  int numat = 0, norbs = 0;
  long long mpack = 0, nw = 0;
  std::vector<int> iorbs;
  MbMzLayout L{};
  double *coord = nullptr, *h = nullptr, *w = nullptr;  // device copies
  // host arrays of MOZYME_C / common_arrays_C (the caller's, not copied)
  int nocc = 0, nvir = 0;
  int *ncf = nullptr, *nncf = nullptr, *icocc = nullptr, *ncocc = nullptr;
  int *nce = nullptr, *nnce = nullptr, *icvir = nullptr, *ncvir = nullptr;
  double *cocc = nullptr, *cvir = nullptr, *p = nullptr, *eigs = nullptr;
  long long icocc_dim = 0, cocc_dim = 0, icvir_dim = 0, cvir_dim = 0;
  double thresh = 1.0e-13, cst = 1.0;
  const double* shift = nullptr;         // MOZYME_C's shift, read at every diagg
  const double* thresh_p = nullptr;      // MOZYME_C's thresh
  // diagg1's and diagg2's saved variables (the Fortran save state)
  double state[4] = {10.0, 1.0, 0.0, 0.0};
  int nrejct[2] = {0, 0};
  long long cap = 0;
  Buf nfmo, ifmo, fmo;
};
MzBound g_mz;

void mz_release_system() {
  if (g_mz.have_system) mb_mz_layout_destroy(&g_mz.L);
  cudaFree(g_mz.coord);
  cudaFree(g_mz.h);
  cudaFree(g_mz.w);
  g_mz.coord = g_mz.h = g_mz.w = nullptr;
  g_mz.have_system = false;
}

}  // namespace

void mz_release_bound() {
  mz_release_system();
  g_mz.nfmo.release();
  g_mz.ifmo.release();
  g_mz.fmo.release();
  g_mz.have_lmos = false;
}

namespace {
int mz_upload(double** dst, const double* src, size_t count) {
  MB_CUDA(cudaMalloc(dst, sizeof(double) * (count > 0 ? count : 1)));
  if (count) MB_CUDA(cudaMemcpy(*dst, src, sizeof(double) * count, cudaMemcpyHostToDevice));
  return MB_OK;
}

// device copies of the registered LMOs (occupied first nocc_use of them)
int mz_lmos(int nocc_use, MbMzLmos* occ, MbMzLmos* vir) {
  MB_TRY(mb_mz_lmos_create(g_mz.numat, g_mz.iorbs.data(), nocc_use, g_mz.ncf, g_mz.nncf, g_mz.icocc, g_mz.ncocc,
                           g_mz.cocc, g_mz.icocc_dim, g_mz.cocc_dim, occ));
  if (vir) {
    int rc = mb_mz_lmos_create(g_mz.numat, g_mz.iorbs.data(), g_mz.nvir, g_mz.nce, g_mz.nnce, g_mz.icvir, g_mz.ncvir,
                               g_mz.cvir, g_mz.icvir_dim, g_mz.cvir_dim, vir);
    if (rc != MB_OK) { mb_mz_lmos_destroy(occ); return rc; }
  }
  return MB_OK;
}

int mz_download(const MbMzLmos* Q, int nlmo, int* ncf, int* ic, long long icdim, double* c, long long cdim) {
  MB_CUDA(cudaMemcpy(ncf, Q->ncf, sizeof(int) * nlmo, cudaMemcpyDeviceToHost));
  MB_CUDA(cudaMemcpy(ic, Q->icocc, sizeof(int) * icdim, cudaMemcpyDeviceToHost));
  MB_CUDA(cudaMemcpy(c, Q->cocc, sizeof(double) * cdim, cudaMemcpyDeviceToHost));
  return MB_OK;
}
}  // namespace

extern "C" int mb_mz_bind_system_(const int* numat, const int* iorbs, const double* coord, const double* cutof1,
                                  const double* cutof2, const double* h, const double* w, const long long* nw) {
  std::lock_guard<std::mutex> lk(g_mu);
  mz_release_system();
  const int n = *numat;
  g_mz.numat = n;
  g_mz.iorbs.assign(iorbs, iorbs + n);
  MB_TRY(mb_mz_layout_create(n, iorbs, coord, *cutof1, *cutof2, &g_mz.L, nullptr));
  g_mz.have_system = true;
  if (*nw != g_mz.L.nw) return mb_set_error(MB_ERR_ARG, "mb_mz_bind_system_: w length differs from the layout's");
  g_mz.norbs = g_mz.L.norbs;
  g_mz.mpack = g_mz.L.mpack;
  g_mz.nw = *nw;
  MB_TRY(mz_upload(&g_mz.coord, coord, 3 * (size_t)n));
  MB_TRY(mz_upload(&g_mz.h, h, (size_t)g_mz.mpack));
  MB_TRY(mz_upload(&g_mz.w, w, (size_t)g_mz.nw));
  g_mz.state[0] = 10.0; g_mz.state[1] = 1.0; g_mz.state[2] = 0.0; g_mz.state[3] = 0.0;
  g_mz.nrejct[0] = g_mz.nrejct[1] = 0;
  return MB_OK;
}

extern "C" int mb_mz_bind_lmos_(const int* nocc, int* ncf, int* nncf, int* icocc, int* ncocc, double* cocc,
                                const long long* icocc_dim, const long long* cocc_dim, const int* nvir, int* nce,
                                int* nnce, int* icvir, int* ncvir, double* cvir, const long long* icvir_dim,
                                const long long* cvir_dim, double* p, double* eigs, const long long* fmo_dim) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_mz.nocc = *nocc; g_mz.ncf = ncf; g_mz.nncf = nncf; g_mz.icocc = icocc; g_mz.ncocc = ncocc; g_mz.cocc = cocc;
  g_mz.icocc_dim = *icocc_dim; g_mz.cocc_dim = *cocc_dim;
  g_mz.nvir = *nvir; g_mz.nce = nce; g_mz.nnce = nnce; g_mz.icvir = icvir; g_mz.ncvir = ncvir; g_mz.cvir = cvir;
  g_mz.icvir_dim = *icvir_dim; g_mz.cvir_dim = *cvir_dim;
  g_mz.p = p;
  g_mz.eigs = eigs;
  g_mz.cap = *fmo_dim;
  g_mz.have_lmos = true;
  return MB_OK;
}

extern "C" int mb_mz_bind_controls_(const double* shift, const double* thresh) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_mz.shift = shift;
  g_mz.thresh_p = thresh;
  return MB_OK;
}

extern "C" void density_for_mozyme_(double* p, const int* mode, const int* nclose_loc, const double* partp) {
  std::lock_guard<std::mutex> lk(g_mu);
  int rc = (!g_mz.have_system || !g_mz.have_lmos)
               ? mb_set_error(MB_ERR_ARG, "density_for_mozyme_: call mb_mz_bind_system_ and mb_mz_bind_lmos_ first")
               : ensure_stream();
  MbMzLmos occ{};
  bool have = false;
  if (rc == MB_OK) rc = mz_lmos(*nclose_loc, &occ, nullptr);
  have = rc == MB_OK;
  const size_t mp = (size_t)g_mz.mpack;
  if (rc == MB_OK) rc = g_a.get(sizeof(double) * 2 * mp);
  double* dp = (double*)g_a.p;
  if (rc == MB_OK && *mode != 0 &&
      cudaMemcpyAsync(dp + mp, partp, sizeof(double) * mp, cudaMemcpyHostToDevice, g_stream) != cudaSuccess)
    rc = MB_ERR_CUDA;
  if (rc == MB_OK) rc = mb_mz_density_dev(&g_mz.L, &occ, *mode, *mode != 0 ? dp + mp : nullptr, dp, g_stream);
  if (rc == MB_OK && cudaMemcpyAsync(p, dp, sizeof(double) * mp, cudaMemcpyDeviceToHost, g_stream) != cudaSuccess)
    rc = MB_ERR_CUDA;
  if (rc == MB_OK && cudaStreamSynchronize(g_stream) != cudaSuccess) rc = MB_ERR_CUDA;
  if (have) mb_mz_lmos_destroy(&occ);
  report(rc, "density_for_mozyme_");
}

extern "C" void buildf_(double* f, const double* partf, const int* mode) {
  (void)partf;
  std::lock_guard<std::mutex> lk(g_mu);
  int rc = (!g_mz.have_system || !g_mz.have_lmos)
               ? mb_set_error(MB_ERR_ARG, "buildf_: call mb_mz_bind_system_ and mb_mz_bind_lmos_ first")
               : (*mode != 0 ? mb_set_error(MB_ERR_UNSUPPORTED, "buildf_: whole-F mode 0 only") : ensure_stream());
  const size_t mp = (size_t)g_mz.mpack;
  if (rc == MB_OK) rc = g_a.get(sizeof(double) * 2 * mp);
  if (rc == MB_OK) rc = g_ws.get(mb_mz_fock_ws_bytes(&g_mz.L) + 256);
  double* dp = (double*)g_a.p;
  double* df = dp + mp;
  if (rc == MB_OK && cudaMemcpyAsync(dp, g_mz.p, sizeof(double) * mp, cudaMemcpyHostToDevice, g_stream) != cudaSuccess)
    rc = MB_ERR_CUDA;
  if (rc == MB_OK) rc = mb_mz_fock_dev(&g_mz.L, g_mz.coord, g_mz.w, dp, g_mz.h, df, g_ws.p, g_stream);
  if (rc == MB_OK && cudaMemcpyAsync(f, df, sizeof(double) * mp, cudaMemcpyDeviceToHost, g_stream) != cudaSuccess)
    rc = MB_ERR_CUDA;
  if (rc == MB_OK && cudaStreamSynchronize(g_stream) != cudaSuccess) rc = MB_ERR_CUDA;
  report(rc, "buildf_");
}

extern "C" void diagg_(const double* fao, const int* nocc, const int* nvir, const int* idiagg, double* partp,
                       const int* indi) {
  std::lock_guard<std::mutex> lk(g_mu);
  int rc = (!g_mz.have_system || !g_mz.have_lmos)
               ? mb_set_error(MB_ERR_ARG, "diagg_: call mb_mz_bind_system_ and mb_mz_bind_lmos_ first")
               : ensure_stream();
  if (rc == MB_OK && (*nocc != g_mz.nocc || *nvir != g_mz.nvir))
    rc = mb_set_error(MB_ERR_ARG, "diagg_: nocc / nvir differ from the bound LMOs");
  MbMzLmos occ{}, vir{};
  bool have = false;
  if (rc == MB_OK) rc = mz_lmos(g_mz.nocc, &occ, &vir);
  have = rc == MB_OK;
  const size_t mp = (size_t)g_mz.mpack;
  const long long cap = g_mz.cap > 0 ? g_mz.cap : 300LL * g_mz.norbs;
  if (rc == MB_OK) rc = g_a.get(sizeof(double) * 3 * mp);
  if (rc == MB_OK) rc = g_b.get(sizeof(double) * ((size_t)g_mz.nocc + g_mz.nvir + 2));
  if (rc == MB_OK) rc = g_ws.get(mb_mz_diagg1_ws_bytes(&g_mz.L, &occ, &vir) + 256);
  if (rc == MB_OK) rc = g_mz.nfmo.get(sizeof(int) * ((size_t)g_mz.nvir + 1));
  if (rc == MB_OK) rc = g_mz.ifmo.get(sizeof(int) * 2 * (size_t)cap);
  if (rc == MB_OK) rc = g_mz.fmo.get(sizeof(double) * (size_t)cap);
  double *dfao = (double*)g_a.p, *dp = dfao + mp, *dpart = dp + mp;
  double *deigs = (double*)g_b.p, *deigv = deigs + g_mz.nocc;
  if (rc == MB_OK && (cudaMemcpyAsync(dfao, fao, sizeof(double) * mp, cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(dp, g_mz.p, sizeof(double) * mp, cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
                      cudaMemcpyAsync(deigs, g_mz.eigs, sizeof(double) * ((size_t)g_mz.nocc + g_mz.nvir),
                                      cudaMemcpyHostToDevice, g_stream) != cudaSuccess ||
                      (*indi != 0 && cudaMemcpyAsync(dpart, partp, sizeof(double) * mp, cudaMemcpyHostToDevice,
                                                     g_stream) != cudaSuccess)))
    rc = MB_ERR_CUDA;
  // diagg.F90: diagg1 (list, energies), diagg2 (rotations), density_for_MOZYME
  long long nij = cap;
  int done = 0;
  double sumt = 0.0, sumb = 0.0;
  long long nrej = 0;
  void* ws = (void*)(((uintptr_t)g_ws.p + 255) & ~(uintptr_t)255);
  if (rc == MB_OK)
    rc = mb_mz_diagg1_dev(&g_mz.L, &occ, &vir, dfao, dp, *idiagg, g_mz.state, (int*)g_mz.nfmo.p, (int*)g_mz.ifmo.p,
                          (double*)g_mz.fmo.p, &nij, deigv, deigs, &done, &sumt, ws, g_stream);
  // diagg2's controls as iter_for_MOZYME sets them: damping, the current
  // shift and thresh (registered by mb_mz_bind_controls_; 0 and 1e-13
  // otherwise), diagg1's tiny and bigeps (diagg2.F90:56-63,
  // iter_for_MOZYME.F90:86-97)
  const double ctl[5] = {g_mz.cst, g_mz.shift ? *g_mz.shift : 0.0, g_mz.thresh_p ? *g_mz.thresh_p : g_mz.thresh,
                         g_mz.state[3], 50.0 * sqrt(1.0e-39)};
  if (rc == MB_OK)
    rc = mb_mz_diagg2_dev(&g_mz.L, &occ, &vir, (const int*)g_mz.ifmo.p, (const double*)g_mz.fmo.p, nij, deigs, deigv,
                          *idiagg, ctl, g_mz.nrejct, &sumb, &nrej, g_stream);
  if (rc == MB_OK) rc = mb_mz_lmos_refresh(g_mz.numat, g_mz.iorbs.data(), &occ);
  if (rc == MB_OK) rc = mb_mz_density_dev(&g_mz.L, &occ, *indi, *indi != 0 ? dpart : nullptr, dp, g_stream);
  if (rc == MB_OK && cudaStreamSynchronize(g_stream) != cudaSuccess) rc = MB_ERR_CUDA;
  if (rc == MB_OK) rc = mz_download(&occ, g_mz.nocc, g_mz.ncf, g_mz.icocc, g_mz.icocc_dim, g_mz.cocc, g_mz.cocc_dim);
  if (rc == MB_OK) rc = mz_download(&vir, g_mz.nvir, g_mz.nce, g_mz.icvir, g_mz.icvir_dim, g_mz.cvir, g_mz.cvir_dim);
  if (rc == MB_OK && (cudaMemcpy(g_mz.p, dp, sizeof(double) * mp, cudaMemcpyDeviceToHost) != cudaSuccess ||
                      cudaMemcpy(g_mz.eigs, deigs, sizeof(double) * ((size_t)g_mz.nocc + g_mz.nvir),
                                 cudaMemcpyDeviceToHost) != cudaSuccess))
    rc = MB_ERR_CUDA;
  if (have) {
    mb_mz_lmos_destroy(&occ);
    mb_mz_lmos_destroy(&vir);
  }
  report(rc, "diagg_");
}
