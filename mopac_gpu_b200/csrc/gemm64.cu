// FP64 GEMM / packed SYRK on the CUDA cores (column-major, LAPACK argument
// conventions).  B200 has the same FP64 rate on DMMA and FFMA, so a register-
// tiled FFMA kernel is the FP64 baseline; the split-precision tensor-core path
// lives in gemm_split.cu.
//
// Tile: 64 x 64 per CTA, BK = 16, 256 threads, 4 x 4 outputs per thread,
// double-buffered shared memory fed by register staging.
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

// P(packed lower) = occ * A A^T with A = c[:, 0:k] (n x k, column-major).
// Grid over 64x64 tiles intersecting the lower triangle.
__global__ void __launch_bounds__(NT) syrk_packed_kernel(int n, int k, double occ, const double* __restrict__ a,
                                                         int lda, double* __restrict__ p, int ntn) {
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
      p[mb_tri(r, cc)] = occ * acc[i][j];
    }
  }
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
  const int tiles = ((n + BN - 1) / BN) * ((m + BM - 1) / BM);
  int nz = 1;
  if (ws && k >= 512 && tiles < 296) {
    nz = (296 + tiles - 1) / tiles;
    if (nz > k / 128) nz = k / 128;
    if (nz > 32) nz = 32;
    while (nz > 1 && (size_t)nz * m * n > ws_elems) --nz;
  }
  dim3 grid((n + BN - 1) / BN, (m + BM - 1) / BM, nz);
  double* out = nz > 1 ? ws : c;
  if (!ta && !tb) dgemm_kernel<false, false><<<grid, NT, 0, stream>>>(m, n, k, alpha, a, lda, b, ldb, beta, out, ldc);
  else if (!ta && tb) dgemm_kernel<false, true><<<grid, NT, 0, stream>>>(m, n, k, alpha, a, lda, b, ldb, beta, out, ldc);
  else if (ta && !tb) dgemm_kernel<true, false><<<grid, NT, 0, stream>>>(m, n, k, alpha, a, lda, b, ldb, beta, out, ldc);
  else dgemm_kernel<true, true><<<grid, NT, 0, stream>>>(m, n, k, alpha, a, lda, b, ldb, beta, out, ldc);
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

extern "C" int mb_density_dev(int n, int nocc, double occ, const double* c, int ldc, double* p,
                              cudaStream_t stream) {
  if (n <= 0 || nocc < 0 || nocc > n) return mb_set_error(MB_ERR_ARG, "mb_density_dev: bad size");
  if (nocc == 0) {
    MB_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * (size_t)n * (n + 1) / 2, stream));
    return MB_OK;
  }
  dim3 grid((n + BN - 1) / BN, (n + BM - 1) / BM);
  mb_kstat_mark(MB_KSTAT_DENSITY, stream, true);
  syrk_packed_kernel<<<grid, NT, 0, stream>>>(n, nocc, occ, c, ldc, p, grid.x);
  mb_kstat_mark(MB_KSTAT_DENSITY, stream, false);
  MB_LAUNCH_CHECK();
  return MB_OK;
}
