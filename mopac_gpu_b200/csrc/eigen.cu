// Full symmetric eigensolver in FP64 on the device, replacing the LAPACK /
// cuSOLVER dsyevd call of eigenvectors_LAPACK (matrix/eigenvectors_LAPACK.F90
// :53-121, cuda_wrappers.cu:469-505).
//
//   1. i*1e-10 added to diagonal element i of the packed input (the
//      reference's parity-critical perturbation, eigenvectors_LAPACK.F90:53-55),
//      then unpacked to a full column-major matrix.
//   2. Householder tridiagonalisation, blocked: a cooperative kernel forms each
//      panel of NB reflectors (three grid barriers per column: column update,
//      reflector + symmetric matrix-vector product, correction), and the
//      trailing matrix gets the rank-2*NB update A -= V W^T + W V^T as FP64 GEMM.
//   3. Eigenvalues of the tridiagonal matrix by bisection on Sturm counts, one
//      thread per eigenvalue.
//   4. Eigenvectors of the tridiagonal matrix by inverse iteration with partial
//      pivoting; eigenvalues closer than 1e-8 * ||T|| form clusters whose
//      vectors are re-orthogonalised inside the iteration (one thread per
//      cluster, members in order).
//   5. Back-transformation C = Q Z with the compact WY form of each panel,
//      Z -= V (T (V^T Z)), as FP64 GEMMs.
// Eigenvalues ascend; eigenvectors are the columns of C.
#include <cooperative_groups.h>

#include "mb_common.cuh"

namespace cg = cooperative_groups;

namespace {

constexpr int NB = 32;         // panel width
constexpr int TPB = 256;       // threads per CTA in the panel kernel
constexpr int TCH = 16;        // row chunks per dot product in t1/t2

struct PanelArgs {
  int n, k, ib, lda;
  double* a;
  double* vp;      // n x NB, panel reflectors (v_j[j+1] = 1, zero above)
  double* wp;      // n x NB
  double* vall;    // n x n, all reflectors (column j holds v_j)
  double* d;
  double* e;
  double* tau;
  double* part;    // gridDim partial norms (column j)
  double* partd;   // gridDim partial dots (w.v)
  double* tvec;    // unused
  double* tpart;   // 2*NB*TCH chunk partials of t1 = W^T v, t2 = V^T v
  double* wvec;    // n
};

__device__ double block_sum(double v, double* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r += sh[i];
  }
  __syncthreads();
  return r;  // valid in thread 0
}

// Sum of the gridDim.x per-CTA partials, computed by warp 0 of each CTA and
// broadcast to the whole CTA (one load per lane per 32 partials).
__device__ double grid_partials_sum(const double* part, double* sh_out) {
  if (threadIdx.x < 32) {
    double s = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += 32) s += part[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) *sh_out = s;
  }
  __syncthreads();
  const double r = *sh_out;
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(TPB) tridiag_panel(PanelArgs p) {
  // Two grid barriers per column.  For column j = k + i:
  //   phase A  finish W(:, i-1) for the CTA's rows (w = tau (p - corr) + alpha v,
  //            with w.v = tau (p.v - 2 t1.t2) so no extra reduction is needed),
  //            update column j with the panel's earlier reflectors, partial
  //            norm of A(j+2:n, j).                                   -> barrier
  //   phase D  reflector, v, p = A22 v (one warp per row), partial p.v and the
  //            chunked t1 = W^T v, t2 = V^T v.                        -> barrier
  cg::grid_group grid = cg::this_grid();
  __shared__ double sh[32];
  __shared__ double s_scal[4];
  __shared__ double s_sum;
  __shared__ double s_vj[NB], s_wj[NB], s_t1[NB], s_t2[NB];
  __shared__ double s_pv[TPB / 32];
  const int n = p.n, lda = p.lda;
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long gstride = (long long)gridDim.x * blockDim.x;
  const int gwarp = (int)(gtid >> 5), nwarps = (int)(gstride >> 5), lane = threadIdx.x & 31;
  double* A = p.a;
#define AE(r, c) A[(long long)(c) * lda + (r)]
#define VP(r, c) p.vp[(long long)(c) * n + (r)]
#define WP(r, c) p.wp[(long long)(c) * n + (r)]
  double prev_tau = 0.0;
  for (int i = 0; i <= p.ib; ++i) {
    const int j = p.k + i;
    // ---------------- phase A
    double alpha_prev = 0.0;
    if (i > 0) {
      const int il = i - 1;  // the column whose W is finished here
      if (threadIdx.x < (unsigned)(2 * il)) {
        const int dotq = threadIdx.x, l = dotq >> 1;
        double t = 0.0;
        for (int ch = 0; ch < TCH; ++ch) t += p.tpart[dotq * TCH + ch];
        if ((dotq & 1) == 0) s_t1[l] = t; else s_t2[l] = t;
      }
      const double pv = grid_partials_sum(p.partd, &s_sum);  // also syncs s_t1/s_t2
      double tt = 0.0;
      for (int l = 0; l < il; ++l) tt += s_t1[l] * s_t2[l];
      const double dot = prev_tau * (pv - 2.0 * tt);
      alpha_prev = -0.5 * prev_tau * dot;
      if (i == p.ib) {
        // last column of the panel: finish W(:, il) and leave
        for (long long r = gtid; r < n; r += gstride) {
          if (r < j) continue;
          double corr = 0.0;
          for (int l = 0; l < il; ++l) corr += VP(r, l) * s_t1[l] + WP(r, l) * s_t2[l];
          WP(r, il) = prev_tau * (p.wvec[r] - corr) + alpha_prev * VP(r, il);
        }
        break;
      }
      if (threadIdx.x == 0) {  // row j of W(:, il), needed by every CTA below
        double corr = 0.0;
        for (int l = 0; l < il; ++l) corr += VP(j, l) * s_t1[l] + WP(j, l) * s_t2[l];
        s_wj[il] = prev_tau * (p.wvec[j] - corr) + alpha_prev * VP(j, il);
      }
    }
    if (threadIdx.x < (unsigned)i) {
      const int l = threadIdx.x;
      s_vj[l] = VP(j, l);
      if (l < i - 1) s_wj[l] = WP(j, l);
    }
    __syncthreads();
    // Rows r >= j, eight lanes per row: lane q handles reflectors l = q, q+8, ...
    // (independent loads), partial sums are combined with shuffles.  The group
    // finishes W(r, i-1) and updates A(r, j); lane 0 accumulates the norm.
    double sig = 0.0;
    {
      const int q = lane & 7;
      const long long gstep = gstride >> 3;         // 8-lane groups in the grid
      const long long gw0 = (gtid >> 5) << 2;       // first group of this warp
      const int il = i - 1;
      // the loop is warp-uniform (shuffles need every lane); each group checks
      // its own row
      for (long long base = j + gw0; base < n; base += gstep) {
        const long long r = base + (lane >> 3);
        const bool act = r < n;
        if (i > 0) {
          double corr = 0.0;
          if (act)
            for (int l = q; l < il; l += 8) corr += VP(r, l) * s_t1[l] + WP(r, l) * s_t2[l];
          corr += __shfl_xor_sync(0xffffffffu, corr, 4);
          corr += __shfl_xor_sync(0xffffffffu, corr, 2);
          corr += __shfl_xor_sync(0xffffffffu, corr, 1);
          const double wr_il = act ? prev_tau * (p.wvec[r] - corr) + alpha_prev * VP(r, il) : 0.0;
          double upd = 0.0;
          if (act)
            for (int l = q; l < i; l += 8) {
              const double wrl = (l == il) ? wr_il : WP(r, l);
              upd += VP(r, l) * s_wj[l] + wrl * s_vj[l];
            }
          upd += __shfl_xor_sync(0xffffffffu, upd, 4);
          upd += __shfl_xor_sync(0xffffffffu, upd, 2);
          upd += __shfl_xor_sync(0xffffffffu, upd, 1);
          if (act && q == 0) {
            WP(r, il) = wr_il;
            AE(r, j) = AE(r, j) - upd;
          }
        }
        if (act && q == 0) {
          if (r == j) p.d[j] = AE(j, j);
          if (r >= j + 2) {
            const double x = AE(r, j);
            sig += x * x;
          }
        }
      }
    }
    double bs = block_sum(sig, sh);
    if (threadIdx.x == 0) p.part[blockIdx.x] = bs;
    grid.sync();
    // ---------------- phase D
    const double snorm = grid_partials_sum(p.part, &s_sum);
    if (threadIdx.x == 0) {
      const double alpha = AE(j + 1, j);
      double beta, tau, scal;
      if (snorm == 0.0) {
        beta = alpha; tau = 0.0; scal = 0.0;
      } else {
        beta = -copysign(sqrt(alpha * alpha + snorm), alpha);
        tau = (beta - alpha) / beta;
        scal = 1.0 / (alpha - beta);
      }
      s_scal[0] = tau;
      s_scal[1] = scal;
      s_scal[2] = beta;
    }
    __syncthreads();
    const double tau = s_scal[0], scal = s_scal[1];
    if (gtid == 0) {
      p.e[j] = s_scal[2];
      p.tau[j] = tau;
    }
    for (long long r = gtid; r < n; r += gstride) {
      const double v = (r == j + 1) ? 1.0 : (r > j + 1 ? AE(r, j) * scal : 0.0);
      VP(r, i) = v;
      p.vall[(long long)j * n + r] = v;
    }
    // p(r) = sum_{c > j} A(c, r) v(c), one warp per row r > j, eight loads in
    // flight per lane; the warp also accumulates p(r) v(r) for p.v.
    double pvw = 0.0;
    {
      const double* colj = A + (long long)j * lda;
      for (int r = j + 1 + gwarp; r < n; r += nwarps) {
        const double* colr = A + (long long)r * lda;
        double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;
        int c = j + 1 + lane;
        for (; c + 224 < n; c += 256) {
          double x[8], y[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) x[u] = __ldcs(colr + c + 32 * u);
#pragma unroll
          for (int u = 0; u < 8; ++u) y[u] = colj[c + 32 * u];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const double v = (c + 32 * u == j + 1) ? 1.0 : y[u] * scal;
            if ((u & 3) == 0) acc0 += x[u] * v;
            else if ((u & 3) == 1) acc1 += x[u] * v;
            else if ((u & 3) == 2) acc2 += x[u] * v;
            else acc3 += x[u] * v;
          }
        }
        for (; c < n; c += 32) {
          const double v = (c == j + 1) ? 1.0 : colj[c] * scal;
          acc0 += colr[c] * v;
        }
        double acc = (acc0 + acc1) + (acc2 + acc3);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) {
          p.wvec[r] = acc;
          const double vr = (r == j + 1) ? 1.0 : colj[r] * scal;
          pvw += acc * vr;
        }
      }
      for (int r = gtid; r <= j && r < n; r += (int)gstride) p.wvec[r] = 0.0;
    }
    if (lane == 0) s_pv[threadIdx.x >> 5] = pvw;
    // t1/t2 chunk partials (TCH row chunks per dot product)
    {
      const int rows = n - (j + 1);
      const int chunk = (rows + TCH - 1) / TCH;
      for (int q = nwarps - 1 - gwarp; q < 2 * i * TCH; q += nwarps) {
        const int dotq = q / TCH, ch = q % TCH;
        const int l = dotq >> 1;
        const bool isw = (dotq & 1) == 0;
        const double* col = isw ? p.wp + (long long)l * n : p.vp + (long long)l * n;
        const int rb = j + 1 + ch * chunk, re = min(n, rb + chunk);
        double acc = 0.0;
        for (int r = rb + lane; r < re; r += 32) {
          const double v = (r == j + 1) ? 1.0 : AE(r, j) * scal;
          acc += col[r] * v;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) p.tpart[q] = acc;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_pv[w];
      p.partd[blockIdx.x] = t;
    }
    prev_tau = tau;
    grid.sync();
  }
#undef AE
#undef VP
#undef WP
}

// Second form of the panel kernel, used when every row of the matrix can own
// an 8-lane group of the grid for the whole panel (n <= grid * TPB / 8).
// Row r belongs to group r throughout, so the group keeps its own V(r, l) and
// W(r, l) in registers (lane q holds l = q, q+8, q+16, q+24), prefetches
// A(r, j+1) before the column's last barrier, and updates A(r, j) with no
// global loads but p(r).  After each barrier the loads that remain (the
// per-CTA partials, the broadcast row j, p(r)) are issued by different warps at
// once.  The symmetric matrix-vector product gives each row 1, 2, 4 or 8
// warps of one CTA as the trailing matrix shrinks, so late columns are not
// bound by one warp's chain of loads.  Arithmetic per element follows the
// first form, except that p(r) is summed in wpr column slices for wpr > 1.
__global__ void __launch_bounds__(TPB) tridiag_panel2(PanelArgs p) {
  cg::grid_group grid = cg::this_grid();
  __shared__ double sh[32];
  __shared__ double s_scal[4];
  __shared__ double s_sum, s_alpha, s_wjr;
  __shared__ double s_vj[NB], s_wj[NB], s_t1[NB], s_t2[NB];
  __shared__ double s_pv[TPB / 32];
  __shared__ double s_symv[TPB / 32];
  __shared__ double s_gv[TPB / 8][NB], s_gw[TPB / 8][NB];  // V(r, l), W(r, l) of the CTA's rows
  const int n = p.n, lda = p.lda;
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long gstride = (long long)gridDim.x * blockDim.x;
  const int gwarp = (int)(gtid >> 5), nwarps = (int)(gstride >> 5), lane = threadIdx.x & 31;
  const int wid = threadIdx.x >> 5, q = lane & 7;
  double* A = p.a;
#define AE(r, c) A[(long long)(c) * lda + (r)]
#define VP(r, c) p.vp[(long long)(c) * n + (r)]
#define WP(r, c) p.wp[(long long)(c) * n + (r)]
  const int r = (int)(gtid >> 3);  // the row this group owns
  const bool own = r < n;
  const int g = threadIdx.x >> 3;
  double* gv = s_gv[g];
  double* gw = s_gw[g];
  double a_cur = (own && r >= p.k) ? AE(r, p.k) : 0.0;  // A(r, j) as the panel found it
  double prev_tau = 0.0;
  for (int i = 0; i <= p.ib; ++i) {
    const int j = p.k + i;
    const bool act = own && r >= j;
    double anew = a_cur;
    // ---------------- phase A
    if (i > 0) {
      const int il = i - 1;
      double wv = act ? p.wvec[r] : 0.0;
      if (wid == 0) {
        double sacc = 0.0;
        for (int b = lane; b < (int)gridDim.x; b += 32) sacc += p.partd[b];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sacc += __shfl_down_sync(0xffffffffu, sacc, o);
        if (lane == 0) s_sum = sacc;
      } else if (threadIdx.x >= 32 && threadIdx.x < (unsigned)(32 + 2 * il)) {
        const int dotq = threadIdx.x - 32, l = dotq >> 1;
        double t = 0.0;
        for (int ch = 0; ch < TCH; ++ch) t += p.tpart[dotq * TCH + ch];
        if ((dotq & 1) == 0) s_t1[l] = t; else s_t2[l] = t;
      } else if (wid == TPB / 32 - 1) {
        for (int l = lane; l < i; l += 32) {
          s_vj[l] = VP(j, l);
          if (l < il) s_wj[l] = WP(j, l);
        }
        if (lane == 0) s_wjr = p.wvec[j];
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double tt = 0.0;
        for (int l = 0; l < il; ++l) tt += s_t1[l] * s_t2[l];
        const double dot = prev_tau * (s_sum - 2.0 * tt);
        const double ap = -0.5 * prev_tau * dot;
        double corr = 0.0;
        for (int l = 0; l < il; ++l) corr += s_vj[l] * s_t1[l] + s_wj[l] * s_t2[l];
        s_wj[il] = prev_tau * (s_wjr - corr) + ap * s_vj[il];
        s_scal[3] = ap;
      }
      __syncthreads();
      const double alpha_prev = s_scal[3];
      // W(r, il) from the group's registers
      double corr = 0.0;
      if (act)
        for (int l = q; l < il; l += 8) corr += gv[l] * s_t1[l] + gw[l] * s_t2[l];
      corr += __shfl_xor_sync(0xffffffffu, corr, 4);
      corr += __shfl_xor_sync(0xffffffffu, corr, 2);
      corr += __shfl_xor_sync(0xffffffffu, corr, 1);
      const double wr_il = act ? prev_tau * (wv - corr) + alpha_prev * gv[il] : 0.0;
      if (act && q == 0) WP(r, il) = wr_il;
      if (i == p.ib) break;  // last column of the panel: W(:, il) was all that was left
      double upd = 0.0;
      if (act)
        for (int l = q; l < i; l += 8) {
          const double wrl = (l == il) ? wr_il : gw[l];
          upd += gv[l] * s_wj[l] + wrl * s_vj[l];
        }
      __syncwarp();
      if (q == (il & 7)) gw[il] = wr_il;
      upd += __shfl_xor_sync(0xffffffffu, upd, 4);
      upd += __shfl_xor_sync(0xffffffffu, upd, 2);
      upd += __shfl_xor_sync(0xffffffffu, upd, 1);
      anew = a_cur - upd;
      if (act && q == 0) AE(r, j) = anew;
    }
    double sig = 0.0;
    if (act && q == 0) {
      if (r == j) p.d[j] = anew;
      if (r >= j + 2) sig = anew * anew;
    }
    const double bs = block_sum(sig, sh);
    if (threadIdx.x == 0) p.part[blockIdx.x] = bs;
    grid.sync();
    // ---------------- phase D
    if (wid == 0) {
      double sacc = 0.0;
      for (int b = lane; b < (int)gridDim.x; b += 32) sacc += p.part[b];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sacc += __shfl_down_sync(0xffffffffu, sacc, o);
      if (lane == 0) s_sum = sacc;
    } else if (wid == 1 && lane == 0) {
      s_alpha = AE(j + 1, j);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const double snorm = s_sum, alpha = s_alpha;
      double beta, tau, scal;
      if (snorm == 0.0) {
        beta = alpha; tau = 0.0; scal = 0.0;
      } else {
        beta = -copysign(sqrt(alpha * alpha + snorm), alpha);
        tau = (beta - alpha) / beta;
        scal = 1.0 / (alpha - beta);
      }
      s_scal[0] = tau;
      s_scal[1] = scal;
      s_scal[2] = beta;
    }
    __syncthreads();
    const double tau = s_scal[0], scal = s_scal[1];
    if (gtid == 0) {
      p.e[j] = s_scal[2];
      p.tau[j] = tau;
    }
    {
      const double v = !own ? 0.0 : (r == j + 1 ? 1.0 : (r > j + 1 ? anew * scal : 0.0));
      if (q == 0) {
        gv[i] = v;
        if (own) {
          VP(r, i) = v;
          p.vall[(long long)j * n + r] = v;
        }
      }
    }
    const double* colj = A + (long long)j * lda;
    // p(r) = sum_{c > j} A(c, r) v(c) with wpr warps of one CTA per row
    double pvw = 0.0;
    {
      const int R = n - j - 1;
      int wpr = 1;
      while (wpr < 8 && (long long)gridDim.x * (TPB / 32 / (wpr * 2)) >= R) wpr *= 2;
      const int rpc = (TPB / 32) / wpr;
      const int sub = wid % wpr;
      const int rounds = (R + (int)gridDim.x * rpc - 1) / ((int)gridDim.x * rpc);
      for (int t = 0; t < rounds; ++t) {
        const int rho = (t * (int)gridDim.x + (int)blockIdx.x) * rpc + wid / wpr;
        const int rr = j + 1 + rho;
        double acc = 0.0;
        if (rho < R) {
          const double* colr = A + (long long)rr * lda;
          double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;
          const int step = 32 * wpr;
          int c = j + 1 + lane + 32 * sub;
          for (; c + 7 * step < n; c += 8 * step) {
            double x[8], y[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) x[u] = __ldcs(colr + c + step * u);
#pragma unroll
            for (int u = 0; u < 8; ++u) y[u] = colj[c + step * u];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
              const double v = (c + step * u == j + 1) ? 1.0 : y[u] * scal;
              if ((u & 3) == 0) acc0 += x[u] * v;
              else if ((u & 3) == 1) acc1 += x[u] * v;
              else if ((u & 3) == 2) acc2 += x[u] * v;
              else acc3 += x[u] * v;
            }
          }
          for (; c < n; c += step) {
            const double v = (c == j + 1) ? 1.0 : colj[c] * scal;
            acc0 += colr[c] * v;
          }
          acc = (acc0 + acc1) + (acc2 + acc3);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (wpr > 1) {
          if (lane == 0) s_symv[wid] = acc;
          __syncthreads();
          if (sub == 0 && lane == 0 && rho < R) {
            double tot = 0.0;
            for (int u = 0; u < wpr; ++u) tot += s_symv[wid + u];
            acc = tot;
          }
          __syncthreads();
        }
        if (sub == 0 && lane == 0 && rho < R) {
          p.wvec[rr] = acc;
          const double vr = (rr == j + 1) ? 1.0 : colj[rr] * scal;
          pvw += acc * vr;
        }
      }
      for (int rz = (int)gtid; rz <= j && rz < n; rz += (int)gstride) p.wvec[rz] = 0.0;
    }
    if (lane == 0) s_pv[wid] = pvw;
    // t1/t2 chunk partials (TCH row chunks per dot product)
    {
      const int rows = n - (j + 1);
      const int chunk = (rows + TCH - 1) / TCH;
      for (int qq = nwarps - 1 - gwarp; qq < 2 * i * TCH; qq += nwarps) {
        const int dotq = qq / TCH, ch = qq % TCH;
        const int l = dotq >> 1;
        const bool isw = (dotq & 1) == 0;
        const double* col = isw ? p.wp + (long long)l * n : p.vp + (long long)l * n;
        const int rb = j + 1 + ch * chunk, re = min(n, rb + chunk);
        double acc = 0.0;
        for (int rw = rb + lane; rw < re; rw += 32) {
          const double v = (rw == j + 1) ? 1.0 : AE(rw, j) * scal;
          acc += col[rw] * v;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) p.tpart[qq] = acc;
      }
    }
    // the next column of A for this row, in flight across the barrier
    a_cur = (own && r >= j + 1 && i < p.ib) ? AE(r, j + 1) : 0.0;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_pv[w];
      p.partd[blockIdx.x] = t;
    }
    prev_tau = tau;
    grid.sync();
  }
#undef AE
#undef VP
#undef WP
}

__global__ void copy_last_diag(int n, const double* a, int lda, double* d) {
  if (threadIdx.x == 0 && blockIdx.x == 0) d[n - 1] = a[(long long)(n - 1) * lda + (n - 1)];
}

// ---------------------------------------------------------------- bisection
// 1/q from the hardware's approximate reciprocal refined by two Newton steps,
// r <- r + r (1 - q r): about 1e-16 relative, cheaper than the IEEE division.
// |q| >= pivmin (a normal number) here, so flushing subnormals loses nothing.
// A Sturm count is exact for a matrix within a few ulps of T, so the
// eigenvalue bounds keep the bisection's accuracy.
__device__ __forceinline__ double recip_nr2(double q) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(q));
  double e = fma(-q, r, 1.0);
  r = fma(r, e, r);
  e = fma(-q, r, 1.0);
  return fma(r, e, r);
}

__device__ __forceinline__ int sturm_count(int n, const double* __restrict__ d, const double* __restrict__ e2,
                                           double x, double pivmin) {
  int cnt = 0;
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  cnt += q < 0.0;
  // operands of eight rows are fetched ahead of the dependent recurrence
  for (int i0 = 1; i0 < n; i0 += 8) {
    double db[8], eb[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int i = i0 + u;
      db[u] = i < n ? d[i] : 0.0;
      eb[u] = i < n ? e2[i - 1] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      if (i0 + u >= n) break;
      q = db[u] - x - eb[u] * recip_nr2(q);
      if (fabs(q) < pivmin) q = -pivmin;
      cnt += q < 0.0;
    }
  }
  return cnt;
}

__global__ void tri_bounds(int n, const double* d, const double* e, double* e2, double* bnd) {
  __shared__ double slo[1024], shi[1024], se[1024];
  double lo = 1e300, hi = -1e300, em = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < n - 1 ? fabs(e[i]) : 0.0);
    lo = fmin(lo, d[i] - r);
    hi = fmax(hi, d[i] + r);
    if (i < n - 1) {
      e2[i] = e[i] * e[i];
      em = fmax(em, e2[i]);
    }
  }
  slo[threadIdx.x] = lo; shi[threadIdx.x] = hi; se[threadIdx.x] = em;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      slo[threadIdx.x] = fmin(slo[threadIdx.x], slo[threadIdx.x + s]);
      shi[threadIdx.x] = fmax(shi[threadIdx.x], shi[threadIdx.x + s]);
      se[threadIdx.x] = fmax(se[threadIdx.x], se[threadIdx.x + s]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double tnorm = fmax(fabs(slo[0]), fabs(shi[0]));
    double pad = 2.0 * 2.220446049250313e-16 * tnorm * n + 1e-300;
    bnd[0] = slo[0] - pad;
    bnd[1] = shi[0] + pad;
    bnd[2] = fmax(1e-290, 2.2250738585072014e-308 * fmax(1.0, se[0]));  // pivmin
    bnd[3] = tnorm;
  }
}

// One warp per eigenvalue: each pass the 32 lanes evaluate Sturm counts at 32
// interior points of the bracket, shrinking it 33-fold (about a dozen passes
// instead of ~60 bisection steps, with 32x the parallelism).
__global__ void bisect_kernel(int n, const double* __restrict__ d, const double* __restrict__ e2,
                              const double* __restrict__ bnd, double* __restrict__ w) {
  const int m = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (m >= n) return;
  double lo = bnd[0], hi = bnd[1];
  const double pivmin = bnd[2];
  const double eps = 2.220446049250313e-16;
  for (int it = 0; it < 64; ++it) {
    if (hi - lo <= 2.0 * eps * fmax(fabs(lo), fabs(hi)) + pivmin) break;
    const double x = lo + (hi - lo) * ((double)(lane + 1) / 33.0);
    const int cnt = sturm_count(n, d, e2, x, pivmin);
    const unsigned above = __ballot_sync(0xffffffffu, cnt > m);  // lanes whose point lies above eigenvalue m
    double nlo = lo, nhi = hi;
    if (above == 0u) {
      nlo = __shfl_sync(0xffffffffu, x, 31);
    } else {
      const int first = __ffs(above) - 1;
      nhi = __shfl_sync(0xffffffffu, x, first);
      if (first > 0) nlo = __shfl_sync(0xffffffffu, x, first - 1);
    }
    if (!(nlo > lo) && !(nhi < hi)) break;  // no representable progress
    lo = nlo;
    hi = nhi;
  }
  if (lane == 0) w[m] = 0.5 * (lo + hi);
}

// --------------------------------------------------------- inverse iteration
// LU with partial pivoting of T - lam I and solve, in place on x (stride ld).
// u0/u1/u2 (stride ld) receive the U factor; pivots are re-derived per solve.
// Both sweeps fetch eight rows of operands ahead of the dependent chain, so
// the chain waits on arithmetic, not on one L2 round trip per row.
__device__ void tri_solve(int n, const double* __restrict__ d, const double* __restrict__ e, double lam,
                          double tiny, double* u0, double* u1, double* u2, double* x, long long ld) {
  constexpr int B = 8;
  // factorisation and forward substitution in one pass
  double dd = d[0] - lam;          // current pivot row diagonal
  double du = n > 1 ? e[0] : 0.0;  // current pivot row super-diagonal
  double du2 = 0.0;
  double xr = x[0];
  for (int i0 = 0; i0 < n - 1; i0 += B) {
    double sb[B], dnb[B], enb[B], xnb[B];
#pragma unroll
    for (int u = 0; u < B; ++u) {
      const int i = i0 + u;
      if (i < n - 1) {
        sb[u] = e[i];
        dnb[u] = d[i + 1];
        enb[u] = (i + 1 < n - 1) ? e[i + 1] : 0.0;
        xnb[u] = x[(long long)(i + 1) * ld];
      }
    }
#pragma unroll
    for (int u = 0; u < B; ++u) {
      const int i = i0 + u;
      if (i >= n - 1) break;
      const double sub = sb[u];          // T(i+1, i)
      const double dn = dnb[u] - lam;    // T(i+1, i+1)
      const double en = enb[u];
      const double xn = xnb[u];
      if (fabs(dd) >= fabs(sub)) {
        // no interchange
        double piv_ = dd;
        if (fabs(piv_) < tiny) piv_ = copysign(tiny, piv_ == 0.0 ? 1.0 : piv_);
        const double l = sub / piv_;
        u0[(long long)i * ld] = piv_;
        u1[(long long)i * ld] = du;
        u2[(long long)i * ld] = du2;
        x[(long long)i * ld] = xr;
        dd = dn - l * du;
        du = en;
        du2 = 0.0;
        xr = xn - l * xr;
      } else {
        // interchange rows i and i+1
        const double l = dd / sub;
        u0[(long long)i * ld] = sub;
        u1[(long long)i * ld] = dn;
        u2[(long long)i * ld] = en;
        x[(long long)i * ld] = xn;
        const double ndd = du - l * dn;
        const double ndu = -l * en;
        dd = ndd;
        du = ndu;
        du2 = 0.0;
        xr = xr - l * xn;
      }
    }
  }
  double last = dd;
  if (fabs(last) < tiny) last = copysign(tiny, last == 0.0 ? 1.0 : last);
  u0[(long long)(n - 1) * ld] = last;
  // back substitution
  double x1 = xr / last;  // x[n-1]
  x[(long long)(n - 1) * ld] = x1;
  double x2 = 0.0;        // x[i+2]
  for (int i0 = n - 2; i0 >= 0; i0 -= B) {
    double xb[B], a0[B], a1[B], a2[B];
#pragma unroll
    for (int u = 0; u < B; ++u) {
      const int i = i0 - u;
      if (i >= 0) {
        xb[u] = x[(long long)i * ld];
        a0[u] = u0[(long long)i * ld];
        a1[u] = u1[(long long)i * ld];
        a2[u] = u2[(long long)i * ld];
      }
    }
#pragma unroll
    for (int u = 0; u < B; ++u) {
      const int i = i0 - u;
      if (i < 0) break;
      const double v = (xb[u] - a1[u] * x1 - a2[u] * x2) / a0[u];
      x[(long long)i * ld] = v;
      x2 = x1;
      x1 = v;
    }
  }
}

// x (stride ld) normalised to unit 2-norm; returns the norm before scaling.
// Eight independent loads per step keep the three sweeps bandwidth-bound.
__device__ double normalise(int n, double* x, long long ld) {
  constexpr int B = 8;
  double mx = 0.0;
  for (int i0 = 0; i0 < n; i0 += B) {
    double t[B];
#pragma unroll
    for (int u = 0; u < B; ++u) t[u] = (i0 + u < n) ? x[(long long)(i0 + u) * ld] : 0.0;
#pragma unroll
    for (int u = 0; u < B; ++u) mx = fmax(mx, fabs(t[u]));
  }
  if (mx == 0.0) return 0.0;
  const double inv = 1.0 / mx;
  double s = 0.0;
  for (int i0 = 0; i0 < n; i0 += B) {
    double t[B];
#pragma unroll
    for (int u = 0; u < B; ++u) t[u] = (i0 + u < n) ? x[(long long)(i0 + u) * ld] : 0.0;
#pragma unroll
    for (int u = 0; u < B; ++u) {
      const double v = t[u] * inv;
      s += v * v;
    }
  }
  const double sc = inv / sqrt(s);
  for (int i0 = 0; i0 < n; i0 += B) {
    double t[B];
#pragma unroll
    for (int u = 0; u < B; ++u) t[u] = (i0 + u < n) ? x[(long long)(i0 + u) * ld] : 0.0;
#pragma unroll
    for (int u = 0; u < B; ++u)
      if (i0 + u < n) x[(long long)(i0 + u) * ld] = t[u] * sc;
  }
  return mx * sqrt(s);
}

// One thread per cluster start; X is n x n with X[i*n + m] = component i of
// vector m (so consecutive threads touch consecutive addresses).
__global__ void inverse_iteration(int n, const double* __restrict__ d, const double* __restrict__ e,
                                  const double* __restrict__ w, const double* __restrict__ bnd,
                                  double* __restrict__ X, double* __restrict__ U0, double* __restrict__ U1,
                                  double* __restrict__ U2, int* status) {
  const int m0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (m0 >= n) return;
  const double tnorm = bnd[3];
  const double ortol = 1.0e-8 * tnorm;
  if (m0 > 0 && !(w[m0] - w[m0 - 1] > ortol)) return;  // not a cluster start
  int m1 = m0 + 1;
  while (m1 < n && !(w[m1] - w[m1 - 1] > ortol)) ++m1;
  const double eps = 2.220446049250313e-16;
  const double tiny = eps * fmax(tnorm, 1e-300);
  const long long ld = n;
  double* u0 = U0 + m0;
  double* u1 = U1 + m0;
  double* u2 = U2 + m0;
  double lam_prev = 0.0;
  for (int m = m0; m < m1; ++m) {
    double lam = w[m];
    if (m > m0) {  // separate exactly coincident shifts (dstein's perturbation)
      const double pertol = 10.0 * fabs(eps * lam) + tiny;
      if (lam - lam_prev < pertol) lam = lam_prev + pertol;
    }
    lam_prev = lam;
    double* x = X + m;
    // deterministic start vector
    unsigned long long s = 0x9E3779B97F4A7C15ull ^ (unsigned long long)(m + 1) * 0xBF58476D1CE4E5B9ull;
    for (int i = 0; i < n; ++i) {
      s ^= s >> 31; s *= 0x94D049BB133111EBull; s ^= s >> 29;
      x[(long long)i * ld] = ((double)(s >> 11) * (1.0 / 9007199254740992.0)) - 0.5;
    }
    normalise(n, x, ld);
    const int nits = (m1 - m0 > 1) ? 4 : 2;
    for (int it = 0; it < nits; ++it) {
      tri_solve(n, d, e, lam, tiny, u0, u1, u2, x, ld);
      // re-orthogonalise against earlier members of the cluster (MGS)
      for (int q = m0; q < m; ++q) {
        const double* y = X + q;
        double dt = 0.0;
        for (int i = 0; i < n; ++i) dt += y[(long long)i * ld] * x[(long long)i * ld];
        for (int i = 0; i < n; ++i) x[(long long)i * ld] -= dt * y[(long long)i * ld];
      }
      double nr = normalise(n, x, ld);
      if (!(nr > 0.0) || !isfinite(nr)) { atomicExch(status, MB_ERR_NUMERIC); return; }
    }
  }
}

// Z (column-major n x n) = X^T in the X[i*n + m] layout, i.e. plain copy with
// swapped meaning: Z(i, m) = X[i*n + m].
__global__ void transpose_kernel(int n, const double* __restrict__ X, double* __restrict__ Z) {
  __shared__ double t[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  // X viewed as row-major [i][m]: tile rows i = by.., cols m = bx..
  for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
    int i = by + yy, m = bx + threadIdx.x;
    if (i < n && m < n) t[yy][threadIdx.x] = X[(long long)i * n + m];
  }
  __syncthreads();
  // Z column-major: Z(i, m) at m*n + i; write with i fastest
  for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
    int m = bx + yy, i = by + threadIdx.x;
    if (i < n && m < n) Z[(long long)m * n + i] = t[threadIdx.x][yy];
  }
}

// T factor of a block of reflectors (dlarft, forward columnwise):
// T(i,i) = tau_i, T(0:i, i) = -tau_i T(0:i, 0:i) S(0:i, i) with S = V^T V.
// S and T both live in (dynamic) shared memory.
constexpr int BT = 64;  // reflectors per back-transformation block
constexpr size_t LARFT_SMEM = sizeof(double) * 2 * BT * (BT + 1);

// One CTA per block of reflectors: block b holds reflectors k = b*BT ..
// k+ib-1 of nref, S and T at b*BT*BT.
__global__ void larft_kernel(int nref, const double* __restrict__ Sall, const double* __restrict__ tau_all,
                             double* __restrict__ Tall) {
  extern __shared__ double larft_sh[];
  const int k = blockIdx.x * BT;
  const int ib = (BT < nref - k) ? BT : nref - k;
  if (ib <= 0) return;
  const double* S = Sall + (size_t)blockIdx.x * BT * BT;
  const double* tau = tau_all + k;
  double* T = Tall + (size_t)blockIdx.x * BT * BT;
  double(*st)[BT + 1] = reinterpret_cast<double(*)[BT + 1]>(larft_sh);
  double(*ss)[BT + 1] = reinterpret_cast<double(*)[BT + 1]>(larft_sh + BT * (BT + 1));
  for (int q = threadIdx.x; q < ib * ib; q += blockDim.x) {
    const int r = q % ib, c = q / ib;
    ss[r][c] = S[(long long)c * ib + r];
    st[r][c] = 0.0;
  }
  __syncthreads();
  for (int i = 0; i < ib; ++i) {
    if (threadIdx.x < (unsigned)i) {
      const int r = threadIdx.x;
      double acc = 0.0;
      for (int c = r; c < i; ++c) acc += st[r][c] * ss[c][i];
      st[r][i] = -tau[i] * acc;
    }
    if (threadIdx.x == 0) st[i][i] = tau[i];
    __syncthreads();
  }
  for (int q = threadIdx.x; q < ib * ib; q += blockDim.x) {
    const int r = q % ib, c = q / ib;
    T[(long long)c * ib + r] = st[r][c];
  }
}

}  // namespace

extern "C" int mb_unpack_dev(int n, const double* pk, double* a, int lda, int perturb, double* pk_mut,
                             cudaStream_t stream);
extern "C" int mb_dgemm_ws(char transa, char transb, int m, int n, int k, double alpha, const double* a, int lda,
                           const double* b, int ldb, double beta, double* c, int ldc, double* ws, size_t ws_elems,
                           cudaStream_t stream);

// Workspace: A n*n | V n*n | Z n*n | X n*n | U0,U1,U2 3*n*n | vp,wp 2*n*NB |
// d,e,e2,tau,wvec 5n | small scratch
extern "C" size_t mb_eigh_ws_bytes(int n) {
  size_t nn = (size_t)n * n;
  return sizeof(double) * (7 * nn + 3 * (size_t)n * NB + 5 * (size_t)n + 2 * NB + 2 * NB * TCH + 4096 +
                           (size_t)BT * BT * 2 * (size_t)((n + BT - 1) / BT) +
                           (size_t)BT * n) + 256;
}

extern "C" int mb_eigh_ws(int n, double* fpacked, int perturb, double* c, double* eigs, void* ws, int* status_dev,
                          cudaStream_t stream) {
  const size_t nn = (size_t)n * n;
  double* b = (double*)ws;
  double* A = b; b += nn;
  double* V = b; b += nn;
  double* Z = b; b += nn;
  double* X = b; b += nn;
  double* U0 = b; b += nn;
  double* U1 = b; b += nn;
  double* U2 = b; b += nn;
  double* vwv = b; b += (size_t)n * 3 * NB;  // [V | W | V] panel columns
  double* vp = vwv;
  double* wp = vwv + (size_t)n * NB;
  double* d = b; b += n;
  double* e = b; b += n;
  double* e2 = b; b += n;
  double* tau = b; b += n;
  double* wvec = b; b += n;
  double* tvec = b; b += 2 * NB;
  double* tpart = b; b += 2 * NB * TCH;
  double* part = b; b += 4096;
  const int nblk_bt = (n + BT - 1) / BT;
  double* S = b; b += (size_t)BT * BT * nblk_bt;   // S_b = V_b^T V_b of every back-transformation block
  double* Tm = b; b += (size_t)BT * BT * nblk_bt;  // their T factors
  double* Y = b; b += (size_t)BT * n;
  double* bnd = part + 2048;

  MB_CUDA(cudaMemsetAsync(status_dev, 0, sizeof(int), stream));
  if (n == 1) {
    MB_TRY(mb_unpack_dev(1, fpacked, A, 1, perturb, fpacked, stream));
    MB_CUDA(cudaMemcpyAsync(eigs, A, sizeof(double), cudaMemcpyDeviceToDevice, stream));
    const double one = 1.0;
    MB_CUDA(cudaMemcpyAsync(c, &one, sizeof(double), cudaMemcpyHostToDevice, stream));
    return MB_OK;
  }
  MB_TRY(mb_unpack_dev(n, fpacked, A, n, perturb, fpacked, stream));
  MB_CUDA(cudaMemsetAsync(V, 0, sizeof(double) * nn, stream));
  MB_CUDA(cudaMemsetAsync(e, 0, sizeof(double) * n, stream));

  // cooperative grid size: co-resident CTAs of the panel form in use
  static int sms = 0, per1 = 0;
  if (sms == 0) {
    int dev = 0;
    MB_CUDA(cudaGetDevice(&dev));
    MB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per1, tridiag_panel, TPB, 0));
    if (per1 > 4) per1 = 4;
    if (per1 < 1) return mb_set_error(MB_ERR_CUDA, "tridiag_panel: cannot be co-resident");
  }
  const size_t smem2 = 0;
  bool v2 = true;
  int per = per1;
  if (v2) {
    int per2 = 0;
    MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per2, tridiag_panel2, TPB, smem2));
    if (per2 > 3) per2 = 3;  // wider grids cost more per barrier than they add in bandwidth
    // every row needs its own 8-lane group
    if (per2 >= 1 && (long long)sms * per2 * TPB / 8 >= n) per = per2;
    else v2 = false;
  }
  int grid = sms * per;
  if (grid > 1024) grid = 1024;
  for (int k = 0; k < n - 1; k += NB) {
    const int ib = (NB < n - 1 - k) ? NB : n - 1 - k;
    MB_CUDA(cudaMemsetAsync(vwv, 0, sizeof(double) * (size_t)n * 2 * NB, stream));
    PanelArgs pa;
    pa.n = n; pa.k = k; pa.ib = ib; pa.lda = n;
    pa.a = A; pa.vp = vp; pa.wp = wp; pa.vall = V; pa.d = d; pa.e = e; pa.tau = tau;
    pa.part = part; pa.partd = part + 1024; pa.tvec = tvec; pa.tpart = tpart; pa.wvec = wvec;
    void* args[] = {&pa};
    mb_kstat_mark(MB_KSTAT_TRIDIAG, stream, true);
    // rows own 8-lane groups when the grid has enough of them
    void* kfn = v2 ? (void*)tridiag_panel2 : (void*)tridiag_panel;
    MB_CUDA(cudaLaunchCooperativeKernel(kfn, grid, TPB, args, 0, stream));
    mb_kstat_mark(MB_KSTAT_TRIDIAG, stream, false);
    mb_count_launch();
    const int t = k + ib;
    if (t < n) {
      const int m = n - t;
      double* At = A + (size_t)t * n + t;
      if (ib == NB) {
        // A -= [V W] [W V]^T as one GEMM with k = 2*NB
        MB_CUDA(cudaMemcpyAsync(vwv + (size_t)n * 2 * NB, vp, sizeof(double) * (size_t)n * NB,
                                cudaMemcpyDeviceToDevice, stream));
        MB_TRY(mb_dgemm_dev('N', 'T', m, m, 2 * NB, -1.0, vwv + t, n, wp + t, n, 1.0, At, n, stream));
      } else {
        MB_TRY(mb_dgemm_dev('N', 'T', m, m, ib, -1.0, vp + t, n, wp + t, n, 1.0, At, n, stream));
        MB_TRY(mb_dgemm_dev('N', 'T', m, m, ib, -1.0, wp + t, n, vp + t, n, 1.0, At, n, stream));
      }
    }
  }
  copy_last_diag<<<1, 32, 0, stream>>>(n, A, n, d);
  MB_LAUNCH_CHECK();
  // eigenvalues
  tri_bounds<<<1, 1024, 0, stream>>>(n, d, e, e2, bnd);
  MB_LAUNCH_CHECK();
  bisect_kernel<<<(n * 32 + 255) / 256, 256, 0, stream>>>(n, d, e2, bnd, eigs);
  MB_LAUNCH_CHECK();
  // eigenvectors of T
  MB_CUDA(cudaMemsetAsync(status_dev, 0, sizeof(int), stream));
  inverse_iteration<<<(n + 127) / 128, 128, 0, stream>>>(n, d, e, eigs, bnd, X, U0, U1, U2, status_dev);
  MB_LAUNCH_CHECK();
  {
    dim3 g((n + 31) / 32, (n + 31) / 32), blk(32, 8);
    transpose_kernel<<<g, blk, 0, stream>>>(n, X, Z);
    MB_LAUNCH_CHECK();
  }
  // back-transformation, blocks of BT reflectors in reverse order:
  // Z <- (I - V T V^T) Z
  {
    static bool larft_attr = false;
    if (!larft_attr) {
      MB_CUDA(cudaFuncSetAttribute(larft_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LARFT_SMEM));
      larft_attr = true;
    }
    const int nref = n - 1;  // reflectors 0 .. n-2
    const int last_k = ((nref - 1) / BT) * BT;
    const int nblk = last_k / BT + 1;
    // every block's T factor first (they depend on V only), in one launch
    for (int k = 0; k <= last_k; k += BT) {
      const int ib = (BT < nref - k) ? BT : nref - k;
      const int r0 = k + 1;
      const double* Vk = V + (size_t)k * n + r0;
      MB_TRY(mb_dgemm_ws('T', 'N', ib, ib, n - r0, 1.0, Vk, n, Vk, n, 0.0, S + (size_t)(k / BT) * BT * BT, ib, U0,
                         3 * nn, stream));
    }
    larft_kernel<<<nblk, BT, LARFT_SMEM, stream>>>(nref, S, tau, Tm);
    MB_LAUNCH_CHECK();
    for (int k = last_k; k >= 0; k -= BT) {
      const int ib = (BT < nref - k) ? BT : nref - k;
      if (ib <= 0) continue;
      const int r0 = k + 1;  // first nonzero row of the block's reflectors
      const int m = n - r0;
      const double* Vk = V + (size_t)k * n + r0;
      const double* Tk = Tm + (size_t)(k / BT) * BT * BT;
      MB_TRY(mb_dgemm_ws('T', 'N', ib, n, m, 1.0, Vk, n, Z + r0, n, 0.0, Y, ib, U0, 3 * nn, stream));
      MB_TRY(mb_dgemm_dev('N', 'N', ib, n, ib, 1.0, Tk, ib, Y, ib, 0.0, X, ib, stream));
      MB_TRY(mb_dgemm_dev('N', 'N', m, n, ib, -1.0, Vk, n, X, ib, 1.0, Z + r0, n, stream));
    }
  }
  MB_CUDA(cudaMemcpyAsync(c, Z, sizeof(double) * nn, cudaMemcpyDeviceToDevice, stream));
  return MB_OK;
}

extern "C" int mb_eigh_packed_dev(int n, double* fpacked, double* c, double* eigs, cudaStream_t stream) {
  if (n <= 0) return mb_set_error(MB_ERR_ARG, "mb_eigh_packed_dev: n <= 0");
  void* ws = nullptr;
  int* st = nullptr;
  MB_CUDA(cudaMalloc(&ws, mb_eigh_ws_bytes(n)));
  cudaError_t ce = cudaMalloc((void**)&st, sizeof(int));
  if (ce != cudaSuccess) { cudaFree(ws); return mb_set_cuda_error(ce, "cudaMalloc", __FILE__, __LINE__); }
  int rc = mb_eigh_ws(n, fpacked, 1, c, eigs, ws, st, stream);
  int hst = 0;
  if (rc == MB_OK) {
    ce = cudaMemcpyAsync(&hst, st, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(stream);
    if (ce != cudaSuccess) rc = mb_set_cuda_error(ce, "eigh status", __FILE__, __LINE__);
    else if (hst != 0) rc = mb_set_error(MB_ERR_NUMERIC, "eigensolver: inverse iteration failed");
  }
  cudaFree(ws);
  cudaFree(st);
  return rc;
}
