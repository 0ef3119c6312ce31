// Camp-King interpolation converger on the device: interp
// (matrix/interp.F90:16-346; R. N. Camp and H. F. King, J. Chem. Phys. 75,
// 268 (1981)) with spline (interp.F90:349-484), schmit / schmib
// (matrix/schmit.F90, matrix/schmib.F90) and rsp (matrix/rsp.F90), for the
// closed-shell alpha call iter makes (SCF/iter.F90:781-798).
//
// The n x n matrices of interp (vec_interp, fock_interp, p_interp) stay on
// the device; every product is a DMMA GEMM, rsp is this library's
// eigensolver (with eigenvectors_LAPACK's perturbation), and the
// Gram-Schmidt steps run right-looking: once column k is final, one launch
// projects it out of every later column, which applies to each column the
// same updates in the same order as the reference's left-looking loop;
// the re-orthogonalisation passes and the unit-vector fallback run for the
// one column in a single CTA.  The spline and the control flow are host
// code on a few scalars.
//
// As in this version of the reference, emin stays 0 (spline's minimum is
// local to spline), so interp rotates the vectors only while
// eold - e <= 0.9 eold, i.e. for a positive heat of formation.
#include <cmath>
#include <cstring>

#include "mb_common.cuh"

extern "C" int mb_unpack_dev(int n, const double* pk, double* a, int lda, int perturb, double* pk_mut,
                             cudaStream_t stream);
extern "C" int mb_dgemm_ws(char transa, char transb, int m, int n, int k, double alpha, const double* a, int lda,
                           const double* b, int ldb, double beta, double* c, int ldc, double* ws, size_t ws_elems,
                           cudaStream_t stream);
extern "C" int mb_eigh_ws(int n, double* fpacked, int perturb, double* c, double* eigs, void* ws, int* status_dev,
                          cudaStream_t stream);

namespace {

constexpr int kFinThreads = 512;  // the finishing CTA of a Gram-Schmidt column

__device__ __forceinline__ int phys(int k, int nb, int rev) { return rev ? nb - 1 - k : k; }

// Lower triangle of a column-major matrix packed by rows (MOPAC's layout).
__global__ void pack_lower_rows(int n, const double* __restrict__ a, int lda, double* __restrict__ pk) {
  const long long mp = (long long)n * (n + 1) / 2;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < mp; q += (long long)gridDim.x * blockDim.x) {
    int r = (int)((sqrt(8.0 * (double)q + 1.0) - 1.0) * 0.5);
    while ((long long)r * (r + 1) / 2 > q) --r;
    while ((long long)(r + 1) * (r + 2) / 2 <= q) ++r;
    const int c = (int)(q - (long long)r * (r + 1) / 2);
    pk[q] = a[r + (long long)c * lda];
  }
}

// interp.F90:156-174: eigenpairs in descending order into theta and the
// first np columns of vec; theta(i) = asin(sqrt(min(max(theta(i), 0), 1)))
// for i < m.
__global__ void reverse_eigen(int np_, int m, const double* __restrict__ w, const double* __restrict__ vl,
                              double* __restrict__ theta, double* __restrict__ vec, int ldv) {
  const long long tot = (long long)np_ * np_;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(q % np_), i = (int)(q / np_);
    vec[r + (long long)i * ldv] = vl[r + (long long)(np_ - 1 - i) * np_];
    if (r == 0) {
      double t = w[np_ - 1 - i];
      if (i < m) t = asin(sqrt(fmin(fmax(t, 0.0), 1.0)));
      theta[i] = t;
    }
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// CTA-wide sum (every thread gets it); sh: 32 doubles.
__device__ double block_sum(double v, double* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < nw; ++w) t += sh[w];
  return t;
}

// schmit.F90:19-25 for every column at once: u_k <- u_k / |u_k| (as a
// product with the reciprocal), or a flag when |u_k|^2 < 1e-20.  One warp
// per column.
__global__ void mgs_prenorm(int nb, double* __restrict__ u, int ld, int* __restrict__ flag) {
  const int lane = threadIdx.x & 31;
  const int col = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (col >= nb) return;
  double* uc = u + (long long)col * ld;
  double d = 0.0;
  for (int r = lane; r < nb; r += 32) d += uc[r] * uc[r];
  d = warp_sum(d);
  if (fabs(d) < 1.0e-20) {
    if (lane == 0) flag[col] = 1;
    return;
  }
  if (lane == 0) flag[col] = 0;
  const double s = 1.0 / sqrt(d);
  for (int r = lane; r < nb; r += 32) uc[r] = s * uc[r];
}

// Column k (logical order) after the projections of the earlier columns:
// schmit.F90:26-59, the norm test, the extra passes (each a left-looking
// projection on all earlier columns, in order) and the fallback to the next
// unit vector.  One CTA.
__global__ void __launch_bounds__(kFinThreads) mgs_finish(int k, int nb, double* __restrict__ u, int ld, int rev,
                                                          const int* __restrict__ flag, int* __restrict__ ii) {
  __shared__ double sh[32];
  const double small = 0.01;
  double* uk = u + (long long)phys(k, nb, rev) * ld;
  int state = flag[phys(k, nb, rev)] ? 100 : 50;  // 50: test the norm (pass 1 done)
  int npass = 1;
  if (k == 0 && state == 50) return;              // schmit.F90:30: nothing to project on
  for (int guard = 0; guard < 64; ++guard) {
    if (state == 100) {                           // schmit.F90:55-58
      __syncthreads();
      const int idx = *ii;                        // read by all threads before thread 0 moves it
      __syncthreads();
      if (threadIdx.x == 0) *ii = idx + 1;
      if (idx < nb && threadIdx.x == 0) uk[idx] = 1.0;
      __syncthreads();
      if (k == 0) return;
      npass = 0;
      state = 40;
    }
    if (state == 40) {                            // schmit.F90:33-39: one more pass
      ++npass;
      for (int j = 0; j < k; ++j) {
        const double* uj = u + (long long)phys(j, nb, rev) * ld;
        double p = 0.0;
        for (int r = threadIdx.x; r < nb; r += blockDim.x) p += uj[r] * uk[r];
        const double d = block_sum(p, sh);
        __syncthreads();
        for (int r = threadIdx.x; r < nb; r += blockDim.x) uk[r] = uk[r] - d * uj[r];
        __syncthreads();
      }
      state = 50;
    }
    // state 50: schmit.F90:40-47
    double p = 0.0;
    for (int r = threadIdx.x; r < nb; r += blockDim.x) p += uk[r] * uk[r];
    const double dot = block_sum(p, sh);
    __syncthreads();
    if (fabs(dot) < 1.0e-20 || (dot < small && npass > 2)) {
      state = 100;
      continue;
    }
    const double s = 1.0 / sqrt(dot);
    for (int r = threadIdx.x; r < nb; r += blockDim.x) uk[r] = s * uk[r];
    __syncthreads();
    if (dot < small) {
      state = 40;
      continue;
    }
    return;
  }
}

// Right-looking step: once column k is final, u_j <- u_j - (u_k . u_j) u_k
// for every later column j (one warp each).
__global__ void mgs_project(int k, int nb, double* __restrict__ u, int ld, int rev) {
  const int lane = threadIdx.x & 31;
  const int j = k + 1 + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (j >= nb) return;
  const double* uk = u + (long long)phys(k, nb, rev) * ld;
  double* uj = u + (long long)phys(j, nb, rev) * ld;
  double d = 0.0;
  for (int r = lane; r < nb; r += 32) d += uk[r] * uj[r];
  d = warp_sum(d);
  for (int r = lane; r < nb; r += 32) uj[r] = uj[r] - d * uk[r];
}

// sum over i < np, k < m of theta_k a(i, k) b(i, k) (lda = ldb = ld), one CTA;
// out[slot].
__global__ void __launch_bounds__(1024) theta_dot(int np_, int m, const double* __restrict__ theta,
                                                  const double* __restrict__ a, const double* __restrict__ b, int ld,
                                                  double* __restrict__ out, int slot) {
  __shared__ double sh[32];
  double s = 0.0;
  const long long tot = (long long)np_ * m;
  for (long long q = threadIdx.x; q < tot; q += blockDim.x) {
    const int i = (int)(q % np_), k = (int)(q / np_);
    s += theta[k] * a[i + (long long)k * ld] * b[i + (long long)k * ld];
  }
  const double t = block_sum(s, sh);
  if (threadIdx.x == 0) out[slot] = t;
}

// sum over k < m of theta_k fk(k, k); out[slot].
__global__ void __launch_bounds__(1024) theta_diag(int m, const double* __restrict__ theta,
                                                   const double* __restrict__ fk, int ld, double* __restrict__ out,
                                                   int slot) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int k = threadIdx.x; k < m; k += blockDim.x) s += theta[k] * fk[k + (long long)k * ld];
  const double t = block_sum(s, sh);
  if (threadIdx.x == 0) out[slot] = t;
}

// interp.F90:317-325: cp = vec, then columns k and np + k rotated by
// x theta_k for k < m.
__global__ void rotate_pairs(int n, int np_, int m, double x, const double* __restrict__ theta,
                             const double* __restrict__ vec, double* __restrict__ cp) {
  const long long tot = (long long)n * n;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(q % n), col = (int)(q / n);
    double v = vec[q];
    if (col < m) {
      const double ck = cos(x * theta[col]), sk = sin(x * theta[col]);
      v = ck * vec[q] - sk * vec[r + (long long)(np_ + col) * n];
    } else if (col >= np_ && col < np_ + m) {
      const int k = col - np_;
      const double ck = cos(x * theta[k]), sk = sin(x * theta[k]);
      v = sk * vec[r + (long long)k * n] + ck * vec[q];
    }
    cp[q] = v;
  }
}

// One Gram-Schmidt of the nb x nb block at u (leading dimension ld):
// columns in order (schmit) or in reverse order (schmib).
int gram_schmidt(int nb, double* u, int ld, int rev, int* flag, int* ii, cudaStream_t s) {
  if (nb <= 0) return MB_OK;
  MB_CUDA(cudaMemsetAsync(ii, 0, sizeof(int), s));
  mgs_prenorm<<<(nb + 7) / 8, 256, 0, s>>>(nb, u, ld, flag);
  MB_LAUNCH_CHECK();
  for (int k = 0; k < nb; ++k) {
    mgs_finish<<<1, kFinThreads, 0, s>>>(k, nb, u, ld, rev, flag, ii);
    MB_LAUNCH_CHECK();
    if (k + 1 < nb) {
      const int later = nb - k - 1;
      mgs_project<<<(later + 7) / 8, 256, 0, s>>>(k, nb, u, ld, rev);
      MB_LAUNCH_CHECK();
    }
  }
  return MB_OK;
}

int gemm(char ta, char tb, int m, int n, int k, const double* a, int lda, const double* b, int ldb, double* c, int ldc,
         cudaStream_t s) {
  if (m <= 0 || n <= 0) return MB_OK;
  if (k <= 0) {
    for (int j = 0; j < n; ++j) MB_CUDA(cudaMemsetAsync(c + (long long)j * ldc, 0, sizeof(double) * m, s));
    return MB_OK;
  }
  return mb_dgemm_ws(ta, tb, m, n, k, 1.0, a, lda, b, ldb, 0.0, c, ldc, nullptr, 0, s);
}

int copy_block(int rows, int cols, const double* src, int lds, double* dst, int ldd, cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return MB_OK;
  MB_CUDA(cudaMemcpy2DAsync(dst, sizeof(double) * ldd, src, sizeof(double) * lds, sizeof(double) * rows, cols,
                            cudaMemcpyDeviceToDevice, s));
  return MB_OK;
}

// spline (interp.F90:349-484) on 1-based arrays x, f, df (index 0 unused);
// returns xmin.
double spline(double* x, double* f, double* df, double xhigh, double xlow, int npnts) {
  const double close = 1.0e-8, big = 500.0, huge = 1.0e10, ustep = 1.0, dstep = 2.0;
  double xmin = x[npnts], fbest = f[npnts], dfbest = df[npnts];
  const int n1 = npnts - 1;
  const int j2 = n1 < 1 ? n1 : 1;
  int k = n1;
  while (k >= j2) {  // the DO loop leaves k = j2 - 1 when it runs out
    if (x[k] < xmin) break;
    x[k + 1] = x[k];
    f[k + 1] = f[k];
    df[k + 1] = df[k];
    --k;
  }
  x[k + 1] = xmin;
  f[k + 1] = fbest;
  df[k + 1] = dfbest;
  double step = df[1] > 0.0 ? dstep : ustep;
  const double xstart = fmax(x[1] - step * (x[2] - x[1]), xlow);
  step = df[npnts] > 0.0 ? ustep : dstep;
  const double xstop = fmin(x[npnts] + step * (x[npnts] - x[n1]), xhigh);
  for (k = 1; k <= n1; ++k) {
    bool skip1 = k != 1, skip2 = k != n1;
    if (f[k] < fbest) {
      xmin = x[k];
      fbest = f[k];
      dfbest = df[k];
    }
    const double dx = x[k + 1] - x[k];
    if (dx <= close) continue;
    const double x1 = k == 1 ? xstart - x[1] : 0.0;
    const double x2 = k == n1 ? xstop - x[n1] : dx;
    const double dum = (f[k + 1] - f[k]) / dx;
    const double a = (df[k] + df[k + 1] - dum - dum) / (dx * dx);
    const double b = (dum + dum + dum - df[k] - df[k] - df[k + 1]) / dx;
    const double c = df[k];
    const double bb = b * b, ac3 = (a + a + a) * c;
    bool have = false;
    double xk = 0.0;
    if (!(bb < ac3)) {
      if (b <= 0.0) {
        if (!(fabs(b) > huge * fabs(a))) {
          xk = (-b + sqrt(bb - ac3)) / (a + a + a);
          have = true;
        }
      } else if (bb > big * fabs(ac3)) {  // label 60
        const double r = ac3 / bb;
        xk = -(((0.039063 * r + 0.0625) * r + 0.125) * r + 0.5) * c / b;
        have = true;
      } else {
        xk = (-b + sqrt(bb - ac3)) / (a + a + a);
        have = true;
      }
      if (have && (xk < x1 || xk > x2)) have = false;
    }
    for (;;) {
      if (have) {  // label 80
        const double fm = ((a * xk + b) * xk + c) * xk + f[k];
        if (fm <= fbest) {
          xmin = xk + x[k];
          fbest = fm;
          dfbest = ((a + a + a) * xk + b + b) * xk + c;
        }
      }
      if (!skip1) {  // label 90
        skip1 = true;
        xk = x1;
        have = true;
        continue;
      }
      if (!skip2) {  // label 100
        skip2 = true;
        xk = x2;
        have = true;
        continue;
      }
      break;
    }
  }
  (void)dfbest;
  return xmin;
}

}  // namespace

// interp's state: the SAVE variables and iter's vec_ai, fock_ai, p_ai,
// theta and eold_alpha, for one SCF.
struct mb_campking {
  int n = 0;
  double *vec = nullptr, *fk = nullptr, *pi = nullptr, *ffull = nullptr, *tmp = nullptr, *hpk = nullptr,
         *vecl = nullptr, *w = nullptr, *theta = nullptr, *red = nullptr;
  int *flag = nullptr, *ii = nullptr;
  double x[13] = {0}, f[13] = {0}, df[13] = {0};
  double xold = 0.0, xnow = 0.0, xlow = 0.0, xhigh = 0.0, emin = 0.0, eold_ref = 0.0;
  int npnts = 0, ipoint = 0;
};

extern "C" void mb_campking_destroy(mb_campking* ck) {
  if (!ck) return;
  void* ptrs[] = {ck->vec, ck->fk, ck->pi, ck->ffull, ck->tmp, ck->hpk, ck->vecl, ck->w, ck->theta, ck->red,
                  ck->flag, ck->ii};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete ck;
}

extern "C" int mb_campking_create(int n, mb_campking** out) {
  if (n <= 0 || !out) return mb_set_error(MB_ERR_ARG, "mb_campking_create: bad args");
  mb_campking* ck = new mb_campking();
  ck->n = n;
  const size_t nn = (size_t)n * n;
  cudaError_t e = cudaSuccess;
#define CK_ALLOC(p, bytes) if (e == cudaSuccess) e = cudaMalloc((void**)&(p), (bytes))
  CK_ALLOC(ck->vec, sizeof(double) * nn);
  CK_ALLOC(ck->fk, sizeof(double) * nn);
  CK_ALLOC(ck->pi, sizeof(double) * nn);
  CK_ALLOC(ck->ffull, sizeof(double) * nn);
  CK_ALLOC(ck->tmp, sizeof(double) * nn);
  CK_ALLOC(ck->hpk, sizeof(double) * (nn / 2 + n + 1));
  CK_ALLOC(ck->vecl, sizeof(double) * nn);
  CK_ALLOC(ck->w, sizeof(double) * n);
  CK_ALLOC(ck->theta, sizeof(double) * n);
  CK_ALLOC(ck->red, sizeof(double) * 8);
  CK_ALLOC(ck->flag, sizeof(int) * n);
  CK_ALLOC(ck->ii, sizeof(int));
#undef CK_ALLOC
  // interp's arrays start at zero (iter.F90:789-793) and so do its saved
  // vectors' unused parts
  if (e == cudaSuccess) e = cudaMemset(ck->vec, 0, sizeof(double) * nn);
  if (e == cudaSuccess) e = cudaMemset(ck->fk, 0, sizeof(double) * nn);
  if (e == cudaSuccess) e = cudaMemset(ck->pi, 0, sizeof(double) * nn);
  if (e == cudaSuccess) e = cudaMemset(ck->theta, 0, sizeof(double) * n);
  if (e != cudaSuccess) {
    const int r = mb_set_cuda_error(e, "mb_campking_create", __FILE__, __LINE__);
    mb_campking_destroy(ck);
    return r;
  }
  *out = ck;
  return MB_OK;
}

// interp.F90:16-346.  np_ filled and nq = n - np_ empty levels; e: the
// energy (escf / fpc_9); fp: the packed Fock matrix (device); cp: the n x n
// vectors (device, column-major), replaced by the interpolated ones when the
// returned mode is 3.  eig_ws: mb_eigh_ws_bytes(n) bytes (idle during the
// call); status: a device int for the eigensolver.
extern "C" int mb_campking_interp(mb_campking* ck, int np_, int mode, double e, const double* fp, double* cp,
                                  void* eig_ws, int* status, cudaStream_t s, int* mode_out, int* rotated) {
  if (!ck || !fp || !cp || !eig_ws || !status || !mode_out || !rotated || np_ < 0 || np_ > ck->n)
    return mb_set_error(MB_ERR_ARG, "mb_campking_interp: bad args");
  const int n = ck->n, nq = n - np_, m = np_ < nq ? np_ : nq;
  *rotated = 0;
  if (np_ == 0 || nq == 0) {  // nothing to rotate
    *mode_out = 2;
    return MB_OK;
  }
  double *VEC = ck->vec, *FK = ck->fk, *PI = ck->pi, *F = ck->ffull, *T = ck->tmp;
  const long long ln = n;
  const int grid = 148 * 4;
  MB_TRY(mb_unpack_dev(n, fp, F, n, 0, nullptr, s));
  if (mode != 2) {
    // :86-109  F C_v, then C_o^T F C_v
    MB_TRY(gemm('N', 'N', n, nq, n, F, n, cp + np_ * ln, n, PI, n, s));
    MB_TRY(gemm('T', 'N', np_, nq, n, cp, n, PI, n, FK, n, s));
    if (mode != 3) {  // :110-118
      MB_CUDA(cudaMemcpyAsync(VEC, cp, sizeof(double) * n * ln, cudaMemcpyDeviceToDevice, s));
      ck->eold_ref = e;
      ck->xold = 1.0;
      *mode_out = 2;
      return MB_OK;
    }
    ck->npnts += 1;  // :125-127
    ck->ipoint = ck->npnts;
  } else {
    // :135-142  S = C^T VEC (rows >= np only against the virtual columns)
    MB_TRY(gemm('T', 'N', np_, n, n, cp, n, VEC, n, PI, n, s));
    MB_TRY(gemm('T', 'N', nq, nq, n, cp + np_ * ln, n, VEC + np_ * ln, n, PI + np_ + np_ * ln, n, s));
    const double* sov = PI + np_ * ln;  // rows < np, columns >= np
    // :147-155  H = S_ov S_ov^T, rsp
    MB_TRY(gemm('N', 'T', np_, np_, nq, sov, n, sov, n, T, np_, s));
    pack_lower_rows<<<grid, 256, 0, s>>>(np_, T, np_, ck->hpk);
    MB_LAUNCH_CHECK();
    if (np_ == 1) {  // rsp.F90:23-27
      MB_CUDA(cudaMemcpyAsync(ck->w, ck->hpk, sizeof(double), cudaMemcpyDeviceToDevice, s));
      const double one = 1.0;
      MB_CUDA(cudaMemcpyAsync(ck->vecl, &one, sizeof(double), cudaMemcpyHostToDevice, s));
      MB_CUDA(cudaStreamSynchronize(s));  // `one` lives on this stack frame
    } else {
      MB_CUDA(cudaMemsetAsync(status, 0, sizeof(int), s));
      MB_TRY(mb_eigh_ws(np_, ck->hpk, 1, ck->vecl, ck->w, eig_ws, status, s));
      int st = 0;
      MB_CUDA(cudaMemcpyAsync(&st, status, sizeof(int), cudaMemcpyDeviceToHost, s));
      MB_CUDA(cudaStreamSynchronize(s));
      if (st != 0) return mb_set_error(MB_ERR_NUMERIC, "Camp-King: eigensolver failed (inverse iteration)");
    }
    // :156-174  descending order, rotation angles
    reverse_eigen<<<grid, 256, 0, s>>>(np_, m, ck->w, ck->vecl, ck->theta, VEC, n);
    MB_LAUNCH_CHECK();
    // :180-186  W = S_ov^T E (first m columns of the virtual block), schmit
    MB_TRY(gemm('T', 'N', nq, m, np_, sov, n, VEC, n, VEC + np_ * ln, n, s));
    MB_TRY(gram_schmidt(nq, VEC + np_ * ln, n, 0, ck->flag, ck->ii, s));
    // :191-208  U_p = S_oo^T E, schmib
    MB_TRY(gemm('T', 'N', np_, np_, np_, PI, n, VEC, n, T, n, s));
    MB_TRY(copy_block(np_, np_, T, n, PI, n, s));
    MB_TRY(gram_schmidt(np_, PI, n, 1, ck->flag, ck->ii, s));
    // :212-219  U_q = S_vv W, schmib
    MB_TRY(gemm('N', 'N', nq, nq, nq, PI + np_ + np_ * ln, n, VEC + np_ * ln, n, T, n, s));
    MB_TRY(copy_block(nq, nq, T, n, PI + np_ * ln, n, s));
    MB_TRY(gram_schmidt(nq, PI + np_ * ln, n, 1, ck->flag, ck->ii, s));
    // :223-237  dE/dx at the old point: sum_k theta_k sum_i U_p(i,k) (FK W)(i,k)
    MB_TRY(gemm('N', 'N', np_, m, nq, FK, n, VEC + np_ * ln, n, T, n, s));
    theta_dot<<<1, 1024, 0, s>>>(np_, m, ck->theta, PI, T, n, ck->red, 0);
    MB_LAUNCH_CHECK();
    // :241-254  the corresponding current orbitals: VEC = [C_o E, C_v U_q]
    MB_TRY(copy_block(np_, np_, VEC, n, PI, n, s));
    MB_TRY(gemm('N', 'N', n, np_, np_, cp, n, PI, n, T, n, s));
    MB_TRY(gemm('N', 'N', n, nq, nq, cp + np_ * ln, n, PI + np_ * ln, n, T + np_ * ln, n, s));
    MB_CUDA(cudaMemcpyAsync(VEC, T, sizeof(double) * n * ln, cudaMemcpyDeviceToDevice, s));
    // :260-283  F in the corresponding representation
    MB_TRY(gemm('N', 'N', n, nq, n, F, n, VEC + np_ * ln, n, PI, n, s));
    MB_TRY(gemm('T', 'N', np_, nq, n, VEC, n, PI, n, FK, n, s));
    double h[2] = {0.0, 0.0};
    MB_CUDA(cudaMemcpyAsync(&h[0], ck->red, sizeof(double), cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaMemcpyAsync(&h[1], ck->theta, sizeof(double), cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    ck->x[2] = ck->xold;  // :234-237
    ck->f[2] = ck->eold_ref;
    ck->df[2] = -4.0 * h[0];
    ck->npnts = 2;  // :287-294
    ck->ipoint = 1;
    ck->xnow = 0.0;
    ck->xhigh = 3.14159265358979323846 / (2.0 * h[1]);
    ck->xlow = -0.5 * ck->xhigh;
  }
  // :301-312  the current point and the spline
  theta_diag<<<1, 1024, 0, s>>>(m, ck->theta, FK, n, ck->red, 1);
  MB_LAUNCH_CHECK();
  double dedx = 0.0;
  MB_CUDA(cudaMemcpyAsync(&dedx, ck->red + 1, sizeof(double), cudaMemcpyDeviceToHost, s));
  MB_CUDA(cudaStreamSynchronize(s));
  const double enow = e;
  const int ip = ck->ipoint;
  if (ip < 1 || ip > 12 || ck->npnts < 2 || ck->npnts > 12)
    return mb_set_error(MB_ERR_NUMERIC, "Camp-King: interpolation point out of range");
  ck->x[ip] = ck->xnow;
  ck->f[ip] = enow;
  ck->df[ip] = -4.0 * dedx;
  const double xmin = spline(ck->x, ck->f, ck->df, ck->xhigh, ck->xlow, ck->npnts);
  if (ck->eold_ref - enow <= 0.9 * (ck->eold_ref - ck->emin) && ip <= 10) {
    // :313-327  the interpolated vectors
    ck->xnow = xmin;
    rotate_pairs<<<grid, 256, 0, s>>>(n, np_, m, xmin, ck->theta, VEC, cp);
    MB_LAUNCH_CHECK();
    *rotated = 1;
    *mode_out = 3;
    return MB_OK;
  }
  if (mode != 2) {  // :333-336
    MB_CUDA(cudaMemcpyAsync(VEC, cp, sizeof(double) * n * ln, cudaMemcpyDeviceToDevice, s));
    mode = 2;
  }
  ck->eold_ref = enow;
  *mode_out = mode;
  return MB_OK;
}
