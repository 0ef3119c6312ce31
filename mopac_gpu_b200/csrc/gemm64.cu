// FP64 GEMM / packed SYRK (column-major, LAPACK argument conventions).
//
// Two tile engines:
//  * DMMA: 128 x 128 per CTA, BK = 16, 8 warps of 64 x 32, each warp issuing
//    mma.sync m8n8k4 f64 on the FP64 tensor path (8 x 4 fragments, 64
//    accumulators per lane).  Used for every product whose output has more
//    than 64 rows and columns.
//  * FFMA: 64 x 64 per CTA, 4 x 4 outputs per thread; its 8 shared loads per
//    16 FMAs bind it at half the FP64 rate, so it only serves skinny outputs.
// Both double-buffer shared memory through register staging.  The
// split-precision tensor-core path lives in gemm_tc.cu.
#include "mb_common.cuh"

namespace {

constexpr int BM = 64, BN = 64, BK = 16, NT = 256;
constexpr int TM = 4, TN = 4;  // per-thread outputs: rows ty + 16*i, cols tx + 16*j

template <bool TA>
__device__ __forceinline__ double load_a(const double* a, int lda, int m, int k, int r, int kk) {
  if (r >= m || kk >= k) return 0.0;
  return TA ? a[(long long)r * lda + kk] : a[(long long)kk * lda + r];
}
template <bool TB>
__device__ __forceinline__ double load_b(const double* b, int ldb, int n, int k, int kk, int c) {
  if (c >= n || kk >= k) return 0.0;
  return TB ? b[(long long)kk * ldb + c] : b[(long long)c * ldb + kk];
}

// C tile (bm, bn) accumulation, shared by dgemm and packed syrk.
template <bool TA, bool TB>
__device__ __forceinline__ void tile_mma(const double* __restrict__ a, int lda, const double* __restrict__ b,
                                         int ldb, int m, int n, int kbeg, int kend, int bm, int bn,
                                         double acc[TM][TN]) {
  const int k = kend;
  __shared__ double As[2][BK][BM + 1];
  __shared__ double Bs[2][BK][BN + 1];
  const int tid = threadIdx.x;
  const int tx = tid % 16, ty = tid / 16;
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = 0.0;
  // staging: A tile 64x16 and B tile 16x64, 4 elements per thread each
  double ra[4], rb[4];
  auto gload = [&](int k0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int e = tid + q * NT;
      int r, kk;
      if (TA) { kk = e % BK; r = e / BK; } else { r = e % BM; kk = e / BM; }
      ra[q] = load_a<TA>(a, lda, m, k, bm + r, k0 + kk);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int e = tid + q * NT;
      int c, kk;
      if (TB) { c = e % BN; kk = e / BN; } else { kk = e % BK; c = e / BK; }
      rb[q] = load_b<TB>(b, ldb, n, k, k0 + kk, bn + c);
    }
  };
  auto sstore = [&](int buf) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int e = tid + q * NT;
      int r, kk;
      if (TA) { kk = e % BK; r = e / BK; } else { r = e % BM; kk = e / BM; }
      As[buf][kk][r] = ra[q];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int e = tid + q * NT;
      int c, kk;
      if (TB) { c = e % BN; kk = e / BN; } else { kk = e % BK; c = e / BK; }
      Bs[buf][kk][c] = rb[q];
    }
  };
  const int nk = (kend - kbeg + BK - 1) / BK;
  gload(kbeg);
  sstore(0);
  __syncthreads();
  for (int t = 0; t < nk; ++t) {
    const int cur = t & 1;
    if (t + 1 < nk) gload(kbeg + (t + 1) * BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      double av[TM], bv[TN];
#pragma unroll
      for (int i = 0; i < TM; ++i) av[i] = As[cur][kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < TN; ++j) bv[j] = Bs[cur][kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
    }
    if (t + 1 < nk) sstore(cur ^ 1);
    __syncthreads();
  }
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(NT) dgemm_kernel(int m, int n, int k, double alpha, const double* __restrict__ a,
                                                   int lda, const double* __restrict__ b, int ldb, double beta,
                                                   double* __restrict__ c, int ldc) {
  // split-K: slice z of gridDim.z covers k in [z*kchunk, min(k, (z+1)*kchunk))
  // and, when gridDim.z > 1, writes its raw partial sum to c + z*m*n (ld = m)
  const int bm = blockIdx.y * BM, bn = blockIdx.x * BN;
  const int kchunk = (k + gridDim.z - 1) / gridDim.z;
  const int kb = blockIdx.z * kchunk, ke = min(k, kb + kchunk);
  double acc[TM][TN];
  tile_mma<TA, TB>(a, lda, b, ldb, m, n, kb, ke, bm, bn, acc);
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const bool partial = gridDim.z > 1;
  double* cz = partial ? c + (long long)blockIdx.z * m * n : c;
  const int ldz = partial ? m : ldc;
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    int r = bm + ty + 16 * i;
    if (r >= m) continue;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      int cc = bn + tx + 16 * j;
      if (cc >= n) continue;
      double* p = cz + (long long)cc * ldz + r;
      if (partial) *p = acc[i][j];
      else *p = (beta == 0.0) ? alpha * acc[i][j] : alpha * acc[i][j] + beta * (*p);
    }
  }
}

// ------------------------------------------------------------------ DMMA
constexpr int DBM = 128, DBN = 128, DBK = 16, DPAD = 4;  // row stride 132 doubles: conflict-free fragments
constexpr int DMMA_SMEM = (int)sizeof(double) * 2 * DBK * (DBM + DPAD + DBN + DPAD);

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// 128 x 128 tile of op(A) op(B) over k in [kbeg, kend).  Warp w covers rows
// (w % 2) * 64 .. +64 and columns (w / 2) * 32 .. +32; fragment (i, j) of a
// lane holds C(row0 + 8 i + lane / 4, col0 + 8 j + 2 (lane % 4) + {0, 1}).
template <bool TA, bool TB>
__device__ __forceinline__ void tile_dmma(const double* __restrict__ a, int lda, const double* __restrict__ b,
                                          int ldb, int m, int n, int kbeg, int kend, int bm, int bn,
                                          double (&acc)[8][4][2]) {
  extern __shared__ double dmma_sh[];  // DMMA_SMEM bytes: As[2][DBK][DBM+DPAD], Bs[2][DBK][DBN+DPAD]
  double(*As)[DBK][DBM + DPAD] = reinterpret_cast<double(*)[DBK][DBM + DPAD]>(dmma_sh);
  double(*Bs)[DBK][DBN + DPAD] = reinterpret_cast<double(*)[DBK][DBN + DPAD]>(dmma_sh + 2 * DBK * (DBM + DPAD));
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp & 1) * 64, wn = (warp >> 1) * 32;
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  double ra[8], rb[8];  // 128 x 16 tiles: 8 elements per thread each
  auto gload = [&](int k0) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = tid + q * NT;
      int r, kk;
      if (TA) { kk = e % DBK; r = e / DBK; } else { r = e % DBM; kk = e / DBM; }
      ra[q] = load_a<TA>(a, lda, m, kend, bm + r, k0 + kk);
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = tid + q * NT;
      int cc, kk;
      if (TB) { cc = e % DBN; kk = e / DBN; } else { kk = e % DBK; cc = e / DBK; }
      rb[q] = load_b<TB>(b, ldb, n, kend, k0 + kk, bn + cc);
    }
  };
  auto sstore = [&](int buf) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = tid + q * NT;
      int r, kk;
      if (TA) { kk = e % DBK; r = e / DBK; } else { r = e % DBM; kk = e / DBM; }
      As[buf][kk][r] = ra[q];
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int e = tid + q * NT;
      int cc, kk;
      if (TB) { cc = e % DBN; kk = e / DBN; } else { kk = e % DBK; cc = e / DBK; }
      Bs[buf][kk][cc] = rb[q];
    }
  };
  const int nk = (kend - kbeg + DBK - 1) / DBK;
  gload(kbeg);
  sstore(0);
  __syncthreads();
  const int fr = lane >> 2, fk = lane & 3;
  for (int t = 0; t < nk; ++t) {
    const int cur = t & 1;
    if (t + 1 < nk) gload(kbeg + (t + 1) * DBK);
#pragma unroll
    for (int kk = 0; kk < DBK; kk += 4) {
      double av[8], bv[4];
#pragma unroll
      for (int i = 0; i < 8; ++i) av[i] = As[cur][kk + fk][wm + 8 * i + fr];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[cur][kk + fk][wn + 8 * j + fr];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j], av[i], bv[j]);
    }
    if (t + 1 < nk) sstore(cur ^ 1);
    __syncthreads();
  }
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(NT) dgemm_dmma_kernel(int m, int n, int k, double alpha,
                                                        const double* __restrict__ a, int lda,
                                                        const double* __restrict__ b, int ldb, double beta,
                                                        double* __restrict__ c, int ldc) {
  const int bm = blockIdx.y * DBM, bn = blockIdx.x * DBN;
  const int kchunk = (k + gridDim.z - 1) / gridDim.z;
  const int kb = blockIdx.z * kchunk, ke = min(k, kb + kchunk);
  double acc[8][4][2];
  tile_dmma<TA, TB>(a, lda, b, ldb, m, n, kb, ke, bm, bn, acc);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r0 = bm + (warp & 1) * 64 + (lane >> 2), c0 = bn + (warp >> 1) * 32 + 2 * (lane & 3);
  const bool partial = gridDim.z > 1;
  double* cz = partial ? c + (long long)blockIdx.z * m * n : c;
  const int ldz = partial ? m : ldc;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = r0 + 8 * i;
    if (r >= m) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int cc = c0 + 8 * j + t;
        if (cc >= n) continue;
        double* p = cz + (long long)cc * ldz + r;
        if (partial) *p = acc[i][j][t];
        else *p = (beta == 0.0) ? alpha * acc[i][j][t] : alpha * acc[i][j][t] + beta * (*p);
      }
  }
}

// Packed lower P = occ * A A^T (+ P when acc) on the DMMA engine (tiles meeting the lower triangle).
__global__ void __launch_bounds__(NT) syrk_packed_dmma_kernel(int n, int k, double occ, const double* __restrict__ a,
                                                              int lda, double* __restrict__ p, int acc_p) {
  const int bm = blockIdx.y * DBM, bn = blockIdx.x * DBN;
  if (bn > bm + DBM - 1) return;
  double acc[8][4][2];
  tile_dmma<false, true>(a, lda, a, lda, n, n, 0, k, bm, bn, acc);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r0 = bm + (warp & 1) * 64 + (lane >> 2), c0 = bn + (warp >> 1) * 32 + 2 * (lane & 3);
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = r0 + 8 * i;
    if (r >= n) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int cc = c0 + 8 * j + t;
        if (cc > r) continue;
        const long long q = mb_tri(r, cc);
        p[q] = acc_p ? occ * acc[i][j][t] + p[q] : occ * acc[i][j][t];
      }
  }
}

// Opt the DMMA kernels into their dynamic shared memory once per process.
int dmma_attrs() {
  static bool done = false;
  if (done) return MB_OK;
  MB_CUDA(cudaFuncSetAttribute(dgemm_dmma_kernel<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, DMMA_SMEM));
  MB_CUDA(cudaFuncSetAttribute(dgemm_dmma_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, DMMA_SMEM));
  MB_CUDA(cudaFuncSetAttribute(dgemm_dmma_kernel<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, DMMA_SMEM));
  MB_CUDA(cudaFuncSetAttribute(dgemm_dmma_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, DMMA_SMEM));
  MB_CUDA(cudaFuncSetAttribute(syrk_packed_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, DMMA_SMEM));
  done = true;
  return MB_OK;
}

// C = alpha * sum_z part[z] + beta * C, slices summed in order (deterministic).
__global__ void splitk_reduce(int m, int n, int nz, double alpha, const double* __restrict__ part, double beta,
                              double* __restrict__ c, int ldc) {
  const long long mn = (long long)m * n;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < mn; q += (long long)gridDim.x * blockDim.x) {
    double s = part[q];
    for (int z = 1; z < nz; ++z) s += part[z * mn + q];
    const int r = (int)(q % m), cc = (int)(q / m);
    double* p = c + (long long)cc * ldc + r;
    *p = (beta == 0.0) ? alpha * s : alpha * s + beta * (*p);
  }
}

// P(packed lower) = occ * A A^T (+ P when acc) with A = c[:, 0:k] (n x k,
// column-major).  Grid over 64x64 tiles intersecting the lower triangle.
__global__ void __launch_bounds__(NT) syrk_packed_kernel(int n, int k, double occ, const double* __restrict__ a,
                                                         int lda, double* __restrict__ p, int ntn, int acc_p) {
  const int bm = blockIdx.y * BM, bn = blockIdx.x * BN;
  if (bn > bm + BM - 1) return;  // tile entirely above the diagonal
  double acc[TM][TN];
  tile_mma<false, true>(a, lda, a, lda, n, n, 0, k, bm, bn, acc);
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    int r = bm + ty + 16 * i;
    if (r >= n) continue;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      int cc = bn + tx + 16 * j;
      if (cc > r) continue;
      const long long q = mb_tri(r, cc);
      p[q] = acc_p ? occ * acc[i][j] + p[q] : occ * acc[i][j];
    }
  }
}

// P_ii = cst + P_ii (the constant of the positron-equivalent density).
__global__ void add_diag_kernel(int n, double cst, double* __restrict__ p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[mb_tri(i, i)] = cst + p[mb_tri(i, i)];
}

}  // namespace

// GEMM with optional split-K: when the output has too few 64x64 tiles to fill
// the GPU and k is long, the k loop is cut into slices whose partial sums go to
// ws (nsplit * m * n doubles) and are reduced in a fixed order.
extern "C" int mb_dgemm_ws(char transa, char transb, int m, int n, int k, double alpha, const double* a, int lda,
                           const double* b, int ldb, double beta, double* c, int ldc, double* ws, size_t ws_elems,
                           cudaStream_t stream) {
  if (m < 0 || n < 0 || k < 0) return mb_set_error(MB_ERR_ARG, "mb_dgemm: negative size");
  if (m == 0 || n == 0) return MB_OK;
  bool ta = (transa == 'T' || transa == 't' || transa == 'C' || transa == 'c');
  bool tb = (transb == 'T' || transb == 't' || transb == 'C' || transb == 'c');
  const bool wide = m > BM && n > BN;  // DMMA engine for all but skinny outputs
  const int tbm = wide ? DBM : BM, tbn = wide ? DBN : BN;
  const int tiles = ((n + tbn - 1) / tbn) * ((m + tbm - 1) / tbm);
  const int target = wide ? 148 : 296;
  int nz = 1;
  if (ws && k >= 512 && tiles < target) {
    nz = (target + tiles - 1) / tiles;
    if (nz > k / 128) nz = k / 128;
    if (nz > 32) nz = 32;
    while (nz > 1 && (size_t)nz * m * n > ws_elems) --nz;
  }
  dim3 grid((n + tbn - 1) / tbn, (m + tbm - 1) / tbm, nz);
  double* out = nz > 1 ? ws : c;
  if (wide) {
    MB_TRY(dmma_attrs());
    if (!ta && !tb) dgemm_dmma_kernel<false, false><<<grid, NT, DMMA_SMEM, stream>>>(m, n, k, alpha, a, lda, b, ldb, beta, out, ldc);
    else if (!ta && tb) dgemm_dmma_kernel<false, true><<<grid, NT, DMMA_SMEM, stream>>>(m, n, k, alpha, a, lda, b, ldb, beta, out, ldc);
    else if (ta && !tb) dgemm_dmma_kernel<true, false><<<grid, NT, DMMA_SMEM, stream>>>(m, n, k, alpha, a, lda, b, ldb, beta, out, ldc);
    else dgemm_dmma_kernel<true, true><<<grid, NT, DMMA_SMEM, stream>>>(m, n, k, alpha, a, lda, b, ldb, beta, out, ldc);
  } else {
    if (!ta && !tb) dgemm_kernel<false, false><<<grid, NT, 0, stream>>>(m, n, k, alpha, a, lda, b, ldb, beta, out, ldc);
    else if (!ta && tb) dgemm_kernel<false, true><<<grid, NT, 0, stream>>>(m, n, k, alpha, a, lda, b, ldb, beta, out, ldc);
    else if (ta && !tb) dgemm_kernel<true, false><<<grid, NT, 0, stream>>>(m, n, k, alpha, a, lda, b, ldb, beta, out, ldc);
    else dgemm_kernel<true, true><<<grid, NT, 0, stream>>>(m, n, k, alpha, a, lda, b, ldb, beta, out, ldc);
  }
  MB_LAUNCH_CHECK();
  if (nz > 1) {
    long long mn = (long long)m * n;
    int blocks = (int)((mn + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    splitk_reduce<<<blocks, 256, 0, stream>>>(m, n, nz, alpha, ws, beta, c, ldc);
    MB_LAUNCH_CHECK();
  }
  return MB_OK;
}

extern "C" int mb_dgemm_dev(char transa, char transb, int m, int n, int k, double alpha, const double* a,
                            int lda, const double* b, int ldb, double beta, double* c, int ldc,
                            cudaStream_t stream) {
  return mb_dgemm_ws(transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, nullptr, 0, stream);
}

namespace {

// P = alpha * C[:, k0:k1] C[:, k0:k1]^T (+ P when acc), packed lower.  An
// empty column range gives alpha * 0 (+ P), as a GEMM with k = 0 does.
int syrk_range(int n, int k0, int k1, double alpha, const double* c, int ldc, double* p, bool acc,
               cudaStream_t stream) {
  const int k = k1 > k0 ? k1 - k0 : 0;
  const double* a = c + (long long)(k > 0 ? k0 : 0) * ldc;
  if (n > BM) {
    dim3 grid((n + DBN - 1) / DBN, (n + DBM - 1) / DBM);
    MB_TRY(dmma_attrs());
    syrk_packed_dmma_kernel<<<grid, NT, DMMA_SMEM, stream>>>(n, k, alpha, a, ldc, p, acc ? 1 : 0);
  } else {
    dim3 grid((n + BN - 1) / BN, (n + BM - 1) / BM);
    syrk_packed_kernel<<<grid, NT, 0, stream>>>(n, k, alpha, a, ldc, p, grid.x, acc ? 1 : 0);
  }
  MB_LAUNCH_CHECK();
  return MB_OK;
}

}  // namespace

extern "C" int mb_density_dev(int n, int nocc, double occ, const double* c, int ldc, double* p,
                              cudaStream_t stream) {
  if (n <= 0 || nocc < 0 || nocc > n) return mb_set_error(MB_ERR_ARG, "mb_density_dev: bad size");
  if (nocc == 0) {
    MB_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * (size_t)n * (n + 1) / 2, stream));
    return MB_OK;
  }
  mb_kstat_mark(MB_KSTAT_DENSITY, stream, true);
  const int rc = syrk_range(n, 0, nocc, occ, c, ldc, p, false, stream);
  mb_kstat_mark(MB_KSTAT_DENSITY, stream, false);
  return rc;
}

// density_for_GPU (matrix/density_for_GPU.F90:16-130) and densit
// (matrix/densit.F90): closed-shell, fractional and UHF occupations.
// iopc 2, 3: the DGEMM form; 4: occ * C_d C_d^T; 5: that below fract 0.01,
// else the explicit sums; 6 (no reference iopc): densit, the explicit sums
// at any fract.
extern "C" int mb_density_occ_dev(int n, int ndubl, int nsingl, double occ, double fract, int mode, int iopc,
                                  const double* c, int ldc, double* p, cudaStream_t stream) {
  if (n <= 0 || ldc < n || ndubl < 0 || ndubl > n || nsingl < 0 || nsingl > n || !c || !p)
    return mb_set_error(MB_ERR_ARG, "mb_density_occ_dev: bad size");
  if (iopc < 2 || iopc > 6) return mb_set_error(MB_ERR_ARG, "mb_density_occ_dev: iopc must be 2..6");
  // iopc 4 (and 5 below fract 0.01): the closed-shell product occ * C_d C_d^T
  if (iopc == 4 || (iopc == 5 && fract < 1.0e-2)) return mb_density_dev(n, ndubl, occ, c, ldc, p, stream);
  // electron or positron equivalent (density_for_GPU.F90:32-54, densit.F90:19-36)
  double sign = 1.0, frac = fract, cst = 0.0;
  int nl2 = 1, nu2 = ndubl, nl1 = ndubl + 1, nu1 = nsingl;
  if (ndubl != 0 && nsingl > n / 2 && mode != 2) {
    sign = -1.0;
    frac = occ - fract;
    cst = occ;
    nl2 = nsingl + 1;
    nu2 = n;
    nl1 = ndubl + 1;
    nu1 = nsingl;
  }
  // iopc 2/3 (the DGEMM form): 2*sign*G2, then + frac*sign*G1; iopc 5/6 (the
  // explicit sums, densit): sign*(occ*G2 + frac*G1).  G = C C^T over the
  // 1-based column ranges [nl, nu]; then P_ii = cst + P_ii.
  const double a2 = (iopc <= 3 ? 2.0 : occ) * sign, a1 = frac * sign;
  mb_kstat_mark(MB_KSTAT_DENSITY, stream, true);
  int rc = syrk_range(n, nl2 - 1, nu2, a2, c, ldc, p, false, stream);
  if (rc == MB_OK) rc = syrk_range(n, nl1 - 1, nu1, a1, c, ldc, p, true, stream);
  mb_kstat_mark(MB_KSTAT_DENSITY, stream, false);
  if (rc != MB_OK) return rc;
  if (cst != 0.0) {
    add_diag_kernel<<<(n + 255) / 256, 256, 0, stream>>>(n, cst, p);
    MB_LAUNCH_CHECK();
  }
  return MB_OK;
}
