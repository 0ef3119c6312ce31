// Pulay's DIIS converger (SCF/pulay.F90:16-180) on device-resident histories.
//
// One call stores the current packed Fock matrix F in slot lfock of the Fock
// history, forms the commutator [P, F] = P F - F P (sym_commute,
// pulay.F90:219-247) packed by the 'U' convention of pack_matrix
// (pulay.F90:181-191) into slot lfock of the commutator history, extends the
// bordered error matrix B with the dot products of the new commutator with
// every stored one, inverts B on the host with the Gauss-Jordan routine of
// matrix/osinv.F90 and replaces F by the extrapolation sum_j c_j F_j.
//
// History layouts are the reference's, so that iter's aliasing of its cnvg
// arrays onto them (pold = commutator history, pold2 = Fock history,
// iter.F90:826-831) is reproduced exactly:
//   commutators: slot l (0-based) is the planar block fppf[l*linear ...];
//   Fock:        entry i of slot l is fock[l + i*mfock] (interleaved).
//
// Device work per call: two unpacks, one n^3 FP64 GEMM (M = P F), one pass
// that forms M(i,j) - M(j,i) for i <= j through 32x32 shared-memory tile
// pairs, writes it and dots it against the stored commutators, a fixed-order
// reduction of the dot partials, and the extrapolation (one read of the
// interleaved Fock history, one write of F).  Everything but the small B
// matrix stays on the device.
#include <math.h>
#include <string.h>

#include <vector>

#include "mb_common.cuh"

extern "C" int mb_unpack_dev(int n, const double* pk, double* a, int lda, int perturb, double* pk_mut,
                             cudaStream_t stream);
extern "C" int mb_dgemm_ws(char transa, char transb, int m, int n, int k, double alpha, const double* a, int lda,
                           const double* b, int ldb, double beta, double* c, int ldc, double* ws, size_t ws_elems,
                           cudaStream_t stream);

namespace {

constexpr int CT = 32;       // commutator tile edge
constexpr int CROWS = 8;     // thread rows per commutator tile
constexpr int NPMAX = 16;    // largest history this build accepts

struct Coeffs {
  double c[NPMAX];
};

__global__ void store_fock_kernel(long long lin, int mfock, int slot, const double* __restrict__ f,
                                  double* __restrict__ fock) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < lin; i += (long long)gridDim.x * blockDim.x)
    fock[slot + i * mfock] = f[i];
}

// Tile pair (tr >= tc) of the lower triangle of tiles from the linear block id.
__device__ __forceinline__ void tile_of_block(long long b, int& tr, int& tc) {
  long long r = (long long)((sqrt(8.0 * (double)b + 1.0) - 1.0) * 0.5);
  while (r * (r + 1) / 2 > b) --r;
  while ((r + 1) * (r + 2) / 2 <= b) ++r;
  tr = (int)r;
  tc = (int)(b - r * (r + 1) / 2);
}

// Commutator element (row c, column r), c <= r, of M - M^T stored at packed
// index r(r+1)/2 + c of slot `slot`; partial dots with slots 0..nfock-1 go to
// partials[block * NPMAX + s] (fixed order inside the block).
__global__ void __launch_bounds__(CT * CROWS) commutator_dots_kernel(int n, const double* __restrict__ M,
                                                                   double* __restrict__ fppf, long long lin, int slot,
                                                                   int nfock, double* __restrict__ partials) {
  __shared__ double sA[CT][CT + 1];  // sA[cl][rl] = M(c0 + cl, r0 + rl)
  __shared__ double sB[CT][CT + 1];  // sB[rl][cl] = M(r0 + rl, c0 + cl)
  __shared__ double red[CROWS][NPMAX];
  int tr, tc;
  tile_of_block(blockIdx.x, tr, tc);
  const int r0 = tr * CT, c0 = tc * CT;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int rl = ty; rl < CT; rl += CROWS) {
    const int r = r0 + rl, c = c0 + tx;
    sA[tx][rl] = (r < n && c < n) ? M[(long long)r * n + c] : 0.0;
  }
  for (int cl = ty; cl < CT; cl += CROWS) {
    const int r = r0 + tx, c = c0 + cl;
    sB[tx][cl] = (r < n && c < n) ? M[(long long)c * n + r] : 0.0;
  }
  __syncthreads();
  double acc[NPMAX];
#pragma unroll
  for (int s = 0; s < NPMAX; ++s) acc[s] = 0.0;
  double* out = fppf + (long long)slot * lin;
  for (int rl = ty; rl < CT; rl += CROWS) {
    const int r = r0 + rl, c = c0 + tx;
    if (r >= n || c > r) continue;
    const double v = sA[tx][rl] - sB[rl][tx];
    const long long k = (long long)r * (r + 1) / 2 + c;
    out[k] = v;
#pragma unroll
    for (int s = 0; s < NPMAX; ++s) {
      if (s < nfock) {
        const double o = (s == slot) ? v : fppf[(long long)s * lin + k];
        acc[s] = fma(v, o, acc[s]);
      }
    }
  }
#pragma unroll
  for (int s = 0; s < NPMAX; ++s) {
    double x = acc[s];
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    if (tx == 0) red[ty][s] = x;
  }
  __syncthreads();
  if (ty == 0 && tx < NPMAX) {
    double x = 0.0;
    for (int w = 0; w < CROWS; ++w) x += red[w][tx];
    partials[(long long)blockIdx.x * NPMAX + tx] = x;
  }
}

// out[s] = sum over blocks of partials[b*NPMAX + s], one CTA per s, fixed order.
__global__ void __launch_bounds__(256) reduce_partials_kernel(long long nblocks, const double* __restrict__ partials,
                                                             double* __restrict__ out) {
  __shared__ double red[256];
  const int s = blockIdx.x;
  double x = 0.0;
  for (long long b = threadIdx.x; b < nblocks; b += blockDim.x) x += partials[b * NPMAX + s];
  red[threadIdx.x] = x;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[s] = red[0];
}

// f(i) = sum_{j < nfock} coeffs(j) * fock(j + i*mfock), summed from zero in j
// order with one rounding per operation, as the loop at pulay.F90:170-178.
__global__ void extrapolate_kernel(long long lin, int mfock, int nfock, Coeffs cf, const double* __restrict__ fock,
                                   double* __restrict__ f) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < lin; i += (long long)gridDim.x * blockDim.x) {
    const double* row = fock + i * mfock;
    double sum = 0.0;
#pragma unroll
    for (int j = 0; j < NPMAX; ++j)
      if (j < nfock) sum = DADD(sum, DMUL(cf.c[j], row[j]));
    f[i] = sum;
  }
}

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

long long commutator_blocks(int n) {
  long long t = (n + CT - 1) / CT;
  return t * (t + 1) / 2;
}

}  // namespace

// In-place Gauss-Jordan inversion with full pivoting of the column-major
// n x n matrix a (matrix/osinv.F90:1-118): returns the running product of
// pivots clamped at 1e10, or 0 when a pivot falls below 1e-8 (a is then
// partially reduced, as in the reference).
extern "C" double mb_osinv(double* a, int n) {
  const double tol = 1.0e-8;
  double d = 1.0;
  std::vector<int> L(n + 1), M(n + 1);
  auto A = [&](long long i) -> double& { return a[i - 1]; };  // 1-based flat index
  long long nk = -n;
  for (int k = 1; k <= n; ++k) {
    nk += n;
    L[k] = k;
    M[k] = k;
    const long long kk = nk + k;
    double biga = A(kk);
    for (int j = k; j <= n; ++j) {
      const long long iz = (long long)n * (j - 1);
      for (int i = k; i <= n; ++i) {
        const long long ij = iz + i;
        if (fabs(biga) - fabs(A(ij)) >= 0.0) continue;
        biga = A(ij);
        L[k] = i;
        M[k] = j;
      }
    }
    int j = L[k];
    if (j - k > 0) {  // interchange rows
      long long ki = k - n;
      for (int i = 1; i <= n; ++i) {
        ki += n;
        const double holo = -A(ki);
        const long long ji = ki - k + j;
        A(ki) = A(ji);
        A(ji) = holo;
      }
    }
    int i = M[k];
    if (i - k > 0) {  // interchange columns
      const long long jp = (long long)n * (i - 1);
      for (int jj = 1; jj <= n; ++jj) {
        const long long jk = nk + jj, ji = jp + jj;
        const double holo = -A(jk);
        A(jk) = A(ji);
        A(ji) = holo;
      }
    }
    if (fabs(biga) - tol < 0.0) return 0.0;
    for (int ii = 1; ii <= n; ++ii) {  // divide the pivot column by -pivot
      if (ii == k) continue;
      const long long ik = nk + ii;
      A(ik) = A(ik) / (-biga);
    }
    for (int ii = 1; ii <= n; ++ii) {  // reduce
      const long long ik = nk + ii;
      long long ij = ii - n;
      if (ii == k) continue;
      for (int jj = 1; jj <= n; ++jj) {
        ij += n;
        if (jj == k) continue;
        const long long kj = ij - ii + k;
        A(ij) = A(ik) * A(kj) + A(ij);
      }
    }
    long long kj = k - n;
    for (int jj = 1; jj <= n; ++jj) {  // divide the pivot row by the pivot
      kj += n;
      if (jj == k) continue;
      A(kj) = A(kj) / biga;
    }
    d = fmin(d * biga, 1.0e10);
    A(kk) = 1.0 / biga;
  }
  for (int k = n - 1; k > 0; --k) {  // final row and column interchange
    const int i = L[k];
    if (i - k > 0) {
      const long long jq = (long long)n * (k - 1), jr = (long long)n * (i - 1);
      for (int j = 1; j <= n; ++j) {
        const long long jk = jq + j, ji = jr + j;
        const double holo = A(jk);
        A(jk) = -A(ji);
        A(ji) = holo;
      }
    }
    const int j = M[k];
    if (j - k <= 0) continue;
    long long ki = k - n;
    for (int ii = 1; ii <= n; ++ii) {
      ki += n;
      const double holo = A(ki);
      const long long ji = ki + j - k;
      A(ki) = -A(ji);
      A(ji) = holo;
    }
  }
  return d;
}

extern "C" size_t mb_pulay_ws_bytes(int n) {
  const size_t nn = (size_t)n * n;
  return 3 * align256(sizeof(double) * nn) + align256(sizeof(double) * NPMAX * (size_t)commutator_blocks(n)) +
         align256(sizeof(double) * NPMAX) + 256;
}

extern "C" int mb_pulay_ws(int n, double* f, const double* p, double* fppf, double* fock, int mfock, double* emat,
                           int ldemat, int* lfock, int* nfock, int* start, double* pl, void* ws, cudaStream_t stream) {
  if (n <= 0 || !f || !p || !fppf || !fock || !emat || !lfock || !nfock || !start || !pl || !ws)
    return mb_set_error(MB_ERR_ARG, "mb_pulay: bad args");
  if (mfock < 1 || mfock > NPMAX || ldemat < mfock + 1)
    return mb_set_error(MB_ERR_ARG, "mb_pulay: history length must be 1..16 and ldemat >= mfock + 1");
  if (((uintptr_t)ws & 255) != 0) return mb_set_error(MB_ERR_ARG, "mb_pulay: workspace must be 256-byte aligned");
  const long long lin = (long long)n * (n + 1) / 2;
  const size_t nn = (size_t)n * n;
  // ---- history bookkeeping (pulay.F90:55-74)
  if (*start) {
    *nfock = 1;
    *lfock = 1;
    *start = 0;
  } else {
    if (*nfock < mfock) *nfock += 1;
    *lfock = (*lfock != mfock) ? *lfock + 1 : 1;
  }
  const int slot = *lfock - 1, nf = *nfock;
  char* w = (char*)ws;
  double* P = (double*)w; w += align256(sizeof(double) * nn);
  double* F = (double*)w; w += align256(sizeof(double) * nn);
  double* Mx = (double*)w; w += align256(sizeof(double) * nn);
  const long long nblk = commutator_blocks(n);
  double* partials = (double*)w; w += align256(sizeof(double) * NPMAX * (size_t)nblk);
  double* dots = (double*)w;
  const int sblocks = (int)((lin + 255) / 256 > 148 * 8 ? 148 * 8 : (lin + 255) / 256);
  store_fock_kernel<<<sblocks, 256, 0, stream>>>(lin, mfock, slot, f, fock);
  MB_LAUNCH_CHECK();
  // ---- commutator (pulay.F90:76-79) and its dots with the history (:81-86)
  MB_TRY(mb_unpack_dev(n, p, P, n, 0, nullptr, stream));
  MB_TRY(mb_unpack_dev(n, f, F, n, 0, nullptr, stream));
  MB_TRY(mb_dgemm_ws('N', 'N', n, n, n, 1.0, P, n, F, n, 0.0, Mx, n, nullptr, 0, stream));
  commutator_dots_kernel<<<(unsigned)nblk, dim3(CT, CROWS), 0, stream>>>(n, Mx, fppf, lin, slot, nf, partials);
  MB_LAUNCH_CHECK();
  reduce_partials_kernel<<<nf, 256, 0, stream>>>(nblk, partials, dots);
  MB_LAUNCH_CHECK();
  double hd[NPMAX];
  MB_CUDA(cudaMemcpyAsync(hd, dots, sizeof(double) * nf, cudaMemcpyDeviceToHost, stream));
  MB_CUDA(cudaStreamSynchronize(stream));
  // ---- bordered B matrix (emat is column-major ldemat x ldemat, 1-based in the comments)
  auto E = [&](int i, int j) -> double& { return emat[(size_t)(j - 1) * ldemat + (i - 1)]; };
  const int L1 = *lfock, nf1 = nf + 1;
  for (int i = 1; i <= nf; ++i) {
    E(nf1, i) = -1.0;
    E(i, nf1) = -1.0;
    E(L1, i) = hd[i - 1];
    E(i, L1) = E(L1, i);
  }
  *pl = E(L1, L1) / (double)lin;
  E(nf1, nf1) = 0.0;
  if (E(L1, L1) < 1.0e-20) return MB_OK;
  double cst = 1.0 / E(L1, L1);
  for (int j = 1; j <= nf; ++j)
    for (int i = 1; i <= nf; ++i) E(i, j) = E(i, j) * cst;
  double evec[(NPMAX + 1) * (NPMAX + 1)];
  int l = 0;
  for (int i = 1; i <= nf1; ++i) {  // row i of emat becomes column i of evec
    for (int j = 1; j <= nf1; ++j) evec[l + j - 1] = E(i, j);
    l += nf1;
  }
  cst = 1.0 / cst;
  for (int j = 1; j <= nf; ++j)
    for (int i = 1; i <= nf; ++i) E(i, j) = E(i, j) * cst;
  const double d = mb_osinv(evec, nf1);
  if (fabs(d) < 1.0e-6) {
    *start = 1;
    return MB_OK;
  }
  if (nf < 2) return MB_OK;
  Coeffs cf;
  memset(&cf, 0, sizeof(cf));
  const int il = nf * nf1;
  for (int j = 0; j < nf; ++j) cf.c[j] = -evec[il + j];
  extrapolate_kernel<<<sblocks, 256, 0, stream>>>(lin, mfock, nf, cf, fock, f);
  MB_LAUNCH_CHECK();
  return MB_OK;
}
