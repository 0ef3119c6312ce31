// SCF step kernels other than the Fock build and the eigensolver:
//   helect   integrals/helect.F90          electronic energy
//   cnvg     SCF/cnvg.F90                  density extrapolation / damping
//   unpack   dtpttr('u') as used by eigenvectors_LAPACK.F90:56 and
//            diag_for_GPU.F90:101-114
//   pseudo-diagonalisation, diag_for_GPU.F90:116-206: Fmo = C_v^T F C_o by
//            FP64 GEMM, tiny = 0.05 max|Fmo|, rotation coefficients and the
//            ordered 2x2 rotation sweep over the columns of C.
#include <cooperative_groups.h>

#include "mb_common.cuh"

namespace cg = cooperative_groups;

namespace {

// ------------------------------------------------------------------ helect
// Row sums of P(H+F) below the diagonal and the diagonal terms; one warp/row.
__global__ void helect_rows(int n, const double* __restrict__ p, const double* __restrict__ h,
                            const double* __restrict__ f, double* __restrict__ rows,
                            double* __restrict__ diag) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const long long base = (long long)warp * (warp + 1) / 2;
  double s = 0.0;
  for (int c = lane; c < warp; c += 32) s += p[base + c] * (h[base + c] + f[base + c]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) {
    rows[warp] = s;
    diag[warp] = p[base + warp] * (h[base + warp] + f[base + warp]);
  }
}

// ee = sum(rows) + 0.5 * sum(diag), fixed-order block reduction.
__global__ void helect_final(int n, const double* __restrict__ rows, const double* __restrict__ diag,
                             double* __restrict__ out) {
  __shared__ double sr[1024], sd[1024];
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) { a += rows[i]; b += diag[i]; }
  sr[threadIdx.x] = a;
  sd[threadIdx.x] = b;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) { sr[threadIdx.x] += sr[threadIdx.x + s]; sd[threadIdx.x] += sd[threadIdx.x + s]; }
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sr[0] + 0.5 * sd[0];
}

// -------------------------------------------------------------------- cnvg
// Scalars shared between the three cnvg phases (device scratch).
struct CnvgState {
  double fac;
  double pl;
};

// Phase 1 (one CTA): diagonal statistics in reference order (thread 0), the
// history update p1 <- p_ii and p_ii <- pnew_ii, and the extrapolation factor.
__global__ void cnvg_diag1(int norbs, const double* __restrict__ pnew, double* __restrict__ p,
                           double* __restrict__ p1, int niter, CnvgState* st, double* sum1_out) {
  extern __shared__ double sh[];
  double* sa_new = sh;           // pnew_ii
  double* sa_old = sh + norbs;   // p_ii
  for (int i = threadIdx.x; i < norbs; i += blockDim.x) {
    long long k = mb_tri(i, i);
    sa_new[i] = pnew[k];
    sa_old[i] = p[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const bool extrap = (niter % 3) != 0;
    double pl = 0.0, faca = 0.0, facb = 0.0, sum1 = 0.0;
    for (int i = 0; i < norbs; ++i) {
      double a = sa_new[i];
      sum1 = DADD(sum1, a);
      double sa = fabs(DSUB(a, sa_old[i]));
      if (sa > pl) pl = sa;
      if (!extrap) {
        faca = DADD(faca, DMUL(sa, sa));
        double t = DADD(DSUB(a, DMUL(2.0, sa_old[i])), p1[i]);
        facb = DADD(facb, DMUL(t, t));
      }
    }
    double fac = 0.0;
    if (facb > 1.0e-10 && faca < DMUL(100.0, facb)) fac = sqrt(faca / facb);
    st->fac = fac;
    st->pl = pl;
    *sum1_out = sum1;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < norbs; i += blockDim.x) {
    long long k = mb_tri(i, i);
    p1[i] = sa_old[i];
    p[k] = sa_new[i];
  }
}

// Phase 2 (one CTA per row): off-diagonal extrapolation p = a + fac (a - p).
__global__ void cnvg_offdiag(int norbs, double* __restrict__ pnew, double* __restrict__ p,
                             const CnvgState* __restrict__ st) {
  const double fac = st->fac;
  for (int r = blockIdx.x; r < norbs; r += gridDim.x) {
    const long long base = (long long)r * (r + 1) / 2;
    for (int c = threadIdx.x; c < r; c += blockDim.x) {
      const long long idx = base + c;
      double a = pnew[idx];
      double v = DADD(a, DMUL(fac, DSUB(a, p[idx])));
      p[idx] = v;
      pnew[idx] = v;
    }
  }
}

// Phase 3 (one CTA, thread 0 sequential): diagonal damping, clamp to [0, 2],
// trace renormalisation loop; exactly the reference's order.
__global__ void cnvg_diag2(int norbs, double* __restrict__ pnew, double* __restrict__ p,
                           const double* __restrict__ p1, int niter, const CnvgState* st,
                           const double* sum1_in, double* pl_out) {
  extern __shared__ double sh[];
  double* pd = sh;
  double* p1s = sh + norbs;
  for (int i = threadIdx.x; i < norbs; i += blockDim.x) {
    pd[i] = p[mb_tri(i, i)];
    p1s[i] = p1[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double rhfuhf = 2.0;
    const double damp = (niter > 3) ? 0.05 : 1.0e10;
    const double fac = st->fac;
    double sum2 = 0.0;
    for (int i = 0; i < norbs; ++i) {
      double v = pd[i];
      double dlt = DSUB(v, p1s[i]);
      if (fabs(dlt) > damp) v = DADD(p1s[i], copysign(damp, dlt));
      else v = DADD(v, DMUL(fac, dlt));
      double t = v > 0.0 ? v : 0.0;
      v = t < rhfuhf ? t : rhfuhf;
      sum2 = DADD(sum2, v);
      pd[i] = v;
    }
    double sum0 = *sum1_in, sum1 = sum0;
    for (int guard = 0; guard < 1000; ++guard) {
      double sum = sum2 > 1.0e-3 ? sum1 / sum2 : 0.0;
      sum1 = sum0;
      if (sum2 < 1.0e-3 || fabs(DSUB(sum, 1.0)) < 1.0e-5) break;
      sum2 = 0.0;
      for (int i = 0; i < norbs; ++i) {
        double v = DADD(DMUL(pd[i], sum), 1.0e-20);
        v = v > 0.0 ? v : 0.0;
        if (v > rhfuhf) {
          v = rhfuhf;
          sum1 = DSUB(sum1, rhfuhf);
        } else {
          sum2 = DADD(sum2, v);
        }
        pd[i] = v;
      }
    }
    *pl_out = st->pl;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < norbs; i += blockDim.x) {
    long long k = mb_tri(i, i);
    p[k] = pd[i];
    pnew[k] = pd[i];
  }
}

// ------------------------------------------------------------------ unpack
// Full symmetric column-major matrix from packed lower storage.
__global__ void unpack_sym(int n, const double* __restrict__ pk, double* __restrict__ a, int lda) {
  const int col = blockIdx.y;
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < n; row += gridDim.x * blockDim.x) {
    long long idx = row >= col ? mb_tri(row, col) : mb_tri(col, row);
    a[(long long)col * lda + row] = pk[idx];
  }
}

__global__ void perturb_diag(int n, double* __restrict__ pk) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    long long k = mb_tri(i, i);
    pk[k] = DADD(pk[k], DMUL((double)(i + 1), 1.0e-10));
  }
}

// -------------------------------------------------------- pseudo-diag sweep
constexpr int RT = 16;          // rotation tile: 16 occupied x 16 virtual columns

__global__ void absmax_kernel(long long len, const double* __restrict__ x, unsigned long long* out) {
  double m = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < len; i += (long long)gridDim.x * blockDim.x)
    m = fmax(m, fabs(x[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __double_as_longlong(m));  // m >= 0: bit order == value order
}

// Rotation coefficients for every (occupied i, virtual a) pair in the
// reference's arithmetic (diag_for_GPU.F90:176-206).  act = 0 means skipped.
// Layout is tile-major: the 16 x 16 tile (I, J) of pairs (occupied block I,
// virtual block J) occupies the 256 entries from (I * ntile_v + J) * 256,
// element (u, v) at u * 16 + v; positions past nocc or nvirt hold an inactive
// identity rotation.
__global__ void rot_coeff_kernel(int nocc, int nvirt, const double* __restrict__ fmo,
                                 const double* __restrict__ eig, const unsigned long long* tinybits,
                                 double tiny_direct, double bigeps, double* __restrict__ alpha, double* __restrict__ beta,
                                 unsigned char* __restrict__ act, unsigned int* __restrict__ tile_cnt,
                                 unsigned long long* __restrict__ nrot, int ntile_o, int ntile_v) {
  // tiny = 0.05 * max|Fmo| (diag_for_GPU.F90:151-152) unless given directly
  const double tiny = tiny_direct >= 0.0 ? tiny_direct : __longlong_as_double(*tinybits) * 0.05;
  const long long total = (long long)ntile_o * ntile_v * (RT * RT);
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < total; p += (long long)gridDim.x * blockDim.x) {
    const long long tile = p / (RT * RT);
    const int e = (int)(p % (RT * RT));
    const int I = (int)(tile / ntile_v), J = (int)(tile % ntile_v);
    const int i = I * RT + e / RT, av = J * RT + e % RT;
    unsigned char on = 0;
    double al = 1.0, be = 0.0;
    if (i < nocc && av < nvirt) {
      const double x = fmo[av + (long long)nvirt * i];
      if (!(fabs(x) < tiny)) {
        const double d = DSUB(eig[i], eig[nocc + av]);
        if (!(fabs(x / d) < bigeps)) {
          const double ee = copysign(sqrt(DADD(DMUL(DMUL(4.0, x), x), DMUL(d, d))), d);
          al = sqrt(DMUL(0.5, DADD(1.0, d / ee)));
          be = -copysign(sqrt(DSUB(1.0, DMUL(al, al))), x);
          on = 1;
        }
      }
    }
    alpha[p] = al;
    beta[p] = be;
    act[p] = on;
    if (on) {
      atomicAdd(&tile_cnt[tile], 1u);
      atomicAdd(nrot, 1ull);
    }
  }
}

// Apply all active rotations to C in the reference order.  Tiles are 16 x 16
// pairs (occupied block I, virtual block J); tile (I, J) touches columns I
// (occupied) and J (virtual) only and must follow (I, J-1), which last
// touched columns I, and (I-1, J), which last touched columns J.  Tiles on one
// anti-diagonal I + J = t touch disjoint columns, so they run in parallel,
// and every column still sees its rotations in the sequential sweep's order
// (occupied i outer, virtual j inner) -- rotations on disjoint column pairs
// commute exactly, so C is bit-identical to the sequential sweep.
//
// One cooperative launch per sweep, scheduled as a dataflow graph: rows are
// independent (a rotation mixes two columns of each row separately), so the
// work item is (tile (I, J), block rb of CROWS rows), and item (I, J, rb)
// depends on (I - 1, J, rb) and (I, J - 1, rb) only.  CTAs take items from a
// queue ordered by anti-diagonal I + J, wait for the item's two predecessors'
// done flags, rotate, and set the item's own flag -- no grid barrier, so
// blocks of rows run ahead on later anti-diagonals while others finish the
// current one.  Every predecessor of an item sits earlier in the queue and
// was taken by a resident CTA (a CTA takes its next item only while working
// on the current one), so the smallest unfinished item always has its inputs
// and the sweep cannot stall; each wait is still bounded (2 s of
// %globaltimer), after which the kernel raises an abort flag that ends every
// CTA's loop and sets bit 4 of *err.  A CTA stages the tile's 256
// coefficients in shared memory (every thread reads them by broadcast) and
// each thread rotates one row of the tile's 32 columns in registers; the
// arithmetic of every element is that of the sequential sweep, so C is
// bit-identical to it.
constexpr int CROWS = 128;
constexpr unsigned long long kFlowWaitNs = 2000000000ull;

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// sync[0]: queue head; sync[1]: abort; sync[2 + (I * ntile_v + J) * nrb + rb]:
// done flag of item (I, J, rb).  All zero at launch.
__global__ void __launch_bounds__(CROWS, 3) rot_sweep_kernel(int n, int nocc, int nvirt, double* __restrict__ c,
                                                            const double* __restrict__ alpha,
                                                            const double* __restrict__ beta,
                                                            const unsigned int* __restrict__ tile_cnt, int ntile_o,
                                                            int ntile_v, int* __restrict__ sync,
                                                            int* __restrict__ err) {
  __shared__ double2 s_ab[2][RT * RT];
  __shared__ double s_xi[RT][CROWS];   // the occupied values of each thread's row
  __shared__ int s_next[4];            // the next item: I, J, rb, valid
  __shared__ int s_go;                 // 0 once the sweep is aborted
  const int nrb = (n + CROWS - 1) / CROWS;
  const int ndiag = ntile_o + ntile_v - 1;
  int* const head = sync;
  int* const abort_flag = sync + 1;
  int* const done = sync + 2;
  constexpr int PER = RT * RT / CROWS;  // coefficients each thread stages
  // thread 0's cursor over the queue: items of anti-diagonal t are
  // [t_start, t_start + width(t) * nrb), taken in increasing order
  int t_cur = 0;
  long long t_start = 0;
  auto width = [&](int t) {
    const int jlo = t - (ntile_o - 1) > 0 ? t - (ntile_o - 1) : 0;
    const int jhi = t < ntile_v - 1 ? t : ntile_v - 1;
    return jhi - jlo + 1;
  };
  auto take = [&]() {  // thread 0: the next item into s_next
    const long long q = atomicAdd(head, 1);
    while (t_cur < ndiag && q >= t_start + (long long)width(t_cur) * nrb) {
      t_start += (long long)width(t_cur) * nrb;
      ++t_cur;
    }
    if (t_cur >= ndiag) {
      s_next[3] = 0;
      return;
    }
    const long long loc = q - t_start;
    const int jlo = t_cur - (ntile_o - 1) > 0 ? t_cur - (ntile_o - 1) : 0;
    const int J = jlo + (int)(loc / nrb);
    s_next[0] = t_cur - J;
    s_next[1] = J;
    s_next[2] = (int)(loc % nrb);
    s_next[3] = 1;
  };
  auto stage = [&](int I, int J, double2* pre) {
    const long long tb = ((long long)I * ntile_v + J) * (RT * RT);
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int e = threadIdx.x + q * CROWS;
      pre[q] = make_double2(alpha[tb + e], beta[tb + e]);
    }
  };
  if (threadIdx.x == 0) {
    take();
    s_go = 1;
  }
  __syncthreads();
  int I = s_next[0], J = s_next[1], rb = s_next[2], valid = s_next[3];
  int buf = 0;
  if (valid) {
    double2 pre[PER];
    stage(I, J, pre);
#pragma unroll
    for (int q = 0; q < PER; ++q) s_ab[0][threadIdx.x + q * CROWS] = pre[q];
  }
  __syncthreads();
  while (valid) {
    // the next item, and its coefficients in flight while this one runs
    if (threadIdx.x == 0) take();
    __syncthreads();
    const int nI = s_next[0], nJ = s_next[1], nrb_ = s_next[2], nvalid = s_next[3];
    double2 pre[PER];
    if (nvalid) stage(nI, nJ, pre);
    // wait for the item's predecessors
    if (threadIdx.x == 0) {
      bool ok = true;
      const int* deps[2] = {I > 0 ? done + ((long long)(I - 1) * ntile_v + J) * nrb + rb : nullptr,
                            J > 0 ? done + ((long long)I * ntile_v + (J - 1)) * nrb + rb : nullptr};
      for (int d = 0; d < 2 && ok; ++d) {
        if (!deps[d]) continue;
        const unsigned long long t0 = global_ns();
        while (ld_acquire_gpu(deps[d]) == 0) {
          if (ld_acquire_gpu(abort_flag) != 0 || global_ns() - t0 > kFlowWaitNs) {
            ok = false;
            break;
          }
          __nanosleep(32);
        }
      }
      if (!ok) {
        atomicExch(abort_flag, 1);
        if (err) atomicOr(err, 4);
        s_go = 0;
      }
    }
    __syncthreads();
    if (!s_go) break;
    const int r = rb * CROWS + threadIdx.x;
    if (tile_cnt[I * ntile_v + J] != 0 && r < n) {
      const int i0 = I * RT, j0 = J * RT;
      const double2* ab = s_ab[buf];
      // All 32 values of the thread's row are loaded at once (one memory
      // latency per item; past L1, which may hold lines another SM has
      // since rewritten): the 16 virtual ones stay in registers for the
      // tile, the 16 occupied ones wait in shared memory, since occupied
      // column u is touched by row u of the tile only.  A skipped pair
      // carries the identity (alpha 1, beta 0): applying it leaves both
      // values equal (1*a + 0*b == a), so the rotations run without a
      // branch, each row's coefficients read from shared memory ahead of
      // its dependent chain.
      double xj[RT];
#pragma unroll
      for (int u = 0; u < RT; ++u)
        s_xi[u][threadIdx.x] = (i0 + u < nocc) ? __ldcg(c + (long long)(i0 + u) * n + r) : 0.0;
#pragma unroll
      for (int v = 0; v < RT; ++v) xj[v] = (j0 + v < nvirt) ? __ldcg(c + (long long)(nocc + j0 + v) * n + r) : 0.0;
#pragma unroll 1
      for (int u = 0; u < RT; ++u) {
        double x = s_xi[u][threadIdx.x];
        double2 w[RT];
#pragma unroll
        for (int v = 0; v < RT; ++v) w[v] = ab[u * RT + v];
#pragma unroll
        for (int v = 0; v < RT; ++v) {
          const double b = xj[v];
          const double na = DADD(DMUL(w[v].x, x), DMUL(w[v].y, b));
          xj[v] = DSUB(DMUL(w[v].x, b), DMUL(w[v].y, x));
          x = na;
        }
        s_xi[u][threadIdx.x] = x;
      }
#pragma unroll
      for (int u = 0; u < RT; ++u)
        if (i0 + u < nocc) c[(long long)(i0 + u) * n + r] = s_xi[u][threadIdx.x];
#pragma unroll
      for (int v = 0; v < RT; ++v)
        if (j0 + v < nvirt) c[(long long)(nocc + j0 + v) * n + r] = xj[v];
    }
    if (nvalid) {
#pragma unroll
      for (int q = 0; q < PER; ++q) s_ab[buf ^ 1][threadIdx.x + q * CROWS] = pre[q];
    }
    __syncthreads();  // the item's rows are written; the next buffer is filled
    if (threadIdx.x == 0) {
      __threadfence();
      st_release_gpu(done + ((long long)I * ntile_v + J) * nrb + rb, 1);
    }
    buf ^= 1;
    I = nI;
    J = nJ;
    rb = nrb_;
    valid = nvalid;
  }
}

// sync ints a sweep needs: the queue head, the abort flag and a done flag per
// (tile, row block) item.
size_t flow_sync_ints(int n, int nocc) {
  const size_t to = (size_t)(nocc + RT - 1) / RT, tv = (size_t)(n - nocc + RT - 1) / RT;
  return 2 + to * tv * (size_t)((n + CROWS - 1) / CROWS);
}

int launch_wavefronts(int n, int nocc, int nvirt, double* c, const double* al, const double* be,
                      const unsigned char* act, const unsigned int* tcnt, int to, int tv, int* sync, int* err,
                      cudaStream_t stream) {
  static int grid = 0;
  if (grid == 0) {
    int dev = 0, sms = 0, per = 0;
    MB_CUDA(cudaGetDevice(&dev));
    MB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, rot_sweep_kernel, CROWS, 0));
    if (per < 1) return mb_set_error(MB_ERR_CUDA, "rot_sweep_kernel: no CTA fits on an SM");
    grid = sms * per;
  }
  (void)act;  // skipped pairs carry the identity rotation in al / be
  MB_CUDA(cudaMemsetAsync(sync, 0, sizeof(int) * flow_sync_ints(n, nocc), stream));
  void* args[] = {&n, &nocc, &nvirt, &c, &al, &be, &tcnt, &to, &tv, &sync, &err};
  // cooperative: every CTA resident, which the dataflow queue relies on
  MB_CUDA(cudaLaunchCooperativeKernel((void*)rot_sweep_kernel, grid, CROWS, args, 0, stream));
  mb_count_launch();
  return MB_OK;
}

}  // namespace

// ------------------------------------------------------------------- C ABI
extern "C" int mb_helect_dev(int n, const double* p, const double* h, const double* f, double* out,
                             cudaStream_t stream) {
  if (n <= 0) return mb_set_error(MB_ERR_ARG, "mb_helect_dev: n <= 0");
  double* tmp = nullptr;
  MB_CUDA(mb_malloc_async(&tmp, sizeof(double) * 2 * (size_t)n, stream));
  const int threads = 256;
  const int blocks = (int)(((long long)n * 32 + threads - 1) / threads);
  helect_rows<<<blocks, threads, 0, stream>>>(n, p, h, f, tmp, tmp + n);
  MB_LAUNCH_CHECK();
  helect_final<<<1, 1024, 0, stream>>>(n, tmp, tmp + n, out);
  MB_LAUNCH_CHECK();
  MB_CUDA(cudaFreeAsync(tmp, stream));
  return MB_OK;
}

// Workspace-taking variants used by the SCF driver (no allocation per call).
extern "C" int mb_helect_ws(int n, const double* p, const double* h, const double* f, double* out,
                            double* ws /* 2n */, cudaStream_t stream) {
  const int threads = 256;
  const int blocks = (int)(((long long)n * 32 + threads - 1) / threads);
  helect_rows<<<blocks, threads, 0, stream>>>(n, p, h, f, ws, ws + n);
  MB_LAUNCH_CHECK();
  helect_final<<<1, 1024, 0, stream>>>(n, ws, ws + n, out);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

extern "C" int mb_cnvg_ws(int norbs, double* pnew, double* p, double* p1, int niter, double* pl_out,
                          double* ws /* 4 doubles */, cudaStream_t stream) {
  CnvgState* st = reinterpret_cast<CnvgState*>(ws);
  double* sum1 = ws + 2;
  size_t sh = sizeof(double) * 2 * (size_t)norbs;
  if (sh > 200 * 1024) return mb_set_error(MB_ERR_ARG, "mb_cnvg: norbs too large for one CTA");
  if (sh > 48 * 1024) {
    MB_CUDA(cudaFuncSetAttribute(cnvg_diag1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
    MB_CUDA(cudaFuncSetAttribute(cnvg_diag2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
  }
  cnvg_diag1<<<1, 1024, sh, stream>>>(norbs, pnew, p, p1, niter, st, sum1);
  MB_LAUNCH_CHECK();
  cnvg_offdiag<<<norbs, 256, 0, stream>>>(norbs, pnew, p, st);
  MB_LAUNCH_CHECK();
  cnvg_diag2<<<1, 1024, sh, stream>>>(norbs, pnew, p, p1, niter, st, sum1, pl_out);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

extern "C" int mb_cnvg_dev(int norbs, double* pnew, double* p, double* p1, int niter, double* pl_out,
                           cudaStream_t stream) {
  if (norbs <= 0) return mb_set_error(MB_ERR_ARG, "mb_cnvg_dev: norbs <= 0");
  double* ws = nullptr;
  MB_CUDA(mb_malloc_async(&ws, sizeof(double) * 4, stream));
  int rc = mb_cnvg_ws(norbs, pnew, p, p1, niter, pl_out, ws, stream);
  cudaFreeAsync(ws, stream);
  return rc;
}

extern "C" int mb_unpack_dev(int n, const double* pk, double* a, int lda, int perturb, double* pk_mut,
                             cudaStream_t stream) {
  if (perturb) {
    perturb_diag<<<(n + 255) / 256, 256, 0, stream>>>(n, pk_mut);
    MB_LAUNCH_CHECK();
  }
  dim3 grid((n + 255) / 256, n);
  unpack_sym<<<grid, 256, 0, stream>>>(n, pk, a, lda);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

// Every workspace region starts on a 256-byte boundary.
static inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Workspace layout for the pseudo-diagonalisation (bytes):
//   F full n*n | fck n*max(k,v) | fmo v*k | alpha, beta, act over the
//   ceil(k/16) x ceil(v/16) tiles of 256 pairs (tile-major) | tile counts |
//   tiny bits | nrot
extern "C" size_t mb_pseudo_ws_bytes(int n, int nocc) {
  size_t v = (size_t)(n - nocc), k = (size_t)nocc;
  size_t kv = k * v;
  size_t to = (k + RT - 1) / RT, tv = (v + RT - 1) / RT;
  size_t b = 0;
  b += align256(sizeof(double) * (size_t)n * n);
  b += align256(sizeof(double) * (size_t)n * (k > v ? k : v));
  const size_t kt = to * tv * (size_t)(RT * RT);  // tile-major coefficient entries
  b += align256(sizeof(double) * kv);
  b += 2 * align256(sizeof(double) * kt);
  b += align256(kt);
  b += align256(sizeof(unsigned int) * (to * tv + 64));
  b += 256;
  b += align256(sizeof(int) * flow_sync_ints(n, nocc));  // the sweep's queue and done flags
  return b;
}

extern "C" int mb_gemm_split_ws(char transa, char transb, int m, int n, int k, double alpha, const double* a, int lda,
                                const double* b, int ldb, double beta, double* c, int ldc, void* ws, size_t ws_bytes,
                                int* err_dev, cudaStream_t stream);

// The Fmo GEMMs run in FP64, or -- when split_ws is given -- with the
// three-product BF16 split on the tensor cores (mb_gemm_split_ws).  bigeps is
// the reference's relative rotation threshold (1.5e-7, diag_for_GPU.F90:33)
// and tiny_direct < 0 selects its absolute one, 0.05 max|Fmo|
// (diag_for_GPU.F90:151-152); the SCF's FP64 finish passes 0 for both, so
// that every occupied-virtual pair is rotated.
extern "C" int mb_pseudo_diag_ex(int n, int nocc, const double* fpacked, double* c, const double* eigs,
                                 unsigned long long* nrot_dev, void* ws, void* split_ws, size_t split_ws_bytes,
                                 int* split_err, double bigeps, double tiny_direct, cudaStream_t stream) {
  const int nvirt = n - nocc;
  if (nocc <= 0 || nvirt <= 0) return MB_OK;
  if (((uintptr_t)ws & 255) != 0) return mb_set_error(MB_ERR_ARG, "pseudo-diag workspace must be 256-byte aligned");
  const size_t kv = (size_t)nocc * nvirt;
  char* b = (char*)ws;
  double* ff = (double*)b; b += align256(sizeof(double) * (size_t)n * n);
  double* fck = (double*)b; b += align256(sizeof(double) * (size_t)n * (nocc > nvirt ? nocc : nvirt));
  const int to = (nocc + RT - 1) / RT, tv = (nvirt + RT - 1) / RT;
  const size_t kt = (size_t)to * tv * (RT * RT);
  double* fmo = (double*)b; b += align256(sizeof(double) * kv);
  double* al = (double*)b; b += align256(sizeof(double) * kt);
  double* be = (double*)b; b += align256(sizeof(double) * kt);
  unsigned char* act = (unsigned char*)b; b += align256(kt);
  unsigned int* tcnt = (unsigned int*)b; b += align256(sizeof(unsigned int) * ((size_t)to * tv + 64));
  unsigned long long* tiny = (unsigned long long*)b;
  int* sync = (int*)(b + 256);
  MB_TRY(mb_unpack_dev(n, fpacked, ff, n, 0, nullptr, stream));
  // diag_for_GPU.F90:116-150
  auto gemm = [&](char ta, char tb, int m, int nn, int k, const double* a, int lda, const double* bb, int ldb,
                  double* cc, int ldc) -> int {
    if (split_ws)
      return mb_gemm_split_ws(ta, tb, m, nn, k, 1.0, a, lda, bb, ldb, 0.0, cc, ldc, split_ws, split_ws_bytes, split_err,
                              stream);
    return mb_dgemm_dev(ta, tb, m, nn, k, 1.0, a, lda, bb, ldb, 0.0, cc, ldc, stream);
  };
  if (nocc < nvirt) {
    MB_TRY(gemm('N', 'N', n, nocc, n, ff, n, c, n, fck, n));
    MB_TRY(gemm('T', 'N', nvirt, nocc, n, c + (size_t)nocc * n, n, fck, n, fmo, nvirt));
  } else {
    MB_TRY(gemm('N', 'N', n, nvirt, n, ff, n, c + (size_t)nocc * n, n, fck, n));
    MB_TRY(gemm('T', 'N', nvirt, nocc, n, fck, n, c, n, fmo, nvirt));
  }
  MB_CUDA(cudaMemsetAsync(tiny, 0, sizeof(unsigned long long), stream));
  MB_CUDA(cudaMemsetAsync(tcnt, 0, sizeof(unsigned int) * (size_t)to * tv, stream));
  MB_CUDA(cudaMemsetAsync(nrot_dev, 0, sizeof(unsigned long long), stream));
  int blocks = (int)((kv + 255) / 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  absmax_kernel<<<blocks, 256, 0, stream>>>((long long)kv, fmo, tiny);
  MB_LAUNCH_CHECK();
  int cblocks = (int)((kt + 255) / 256);
  if (cblocks > 148 * 8) cblocks = 148 * 8;
  rot_coeff_kernel<<<cblocks, 256, 0, stream>>>(nocc, nvirt, fmo, eigs, tiny, tiny_direct, bigeps, al, be, act, tcnt,
                                                 nrot_dev, to, tv);
  MB_LAUNCH_CHECK();
  return launch_wavefronts(n, nocc, nvirt, c, al, be, act, tcnt, to, tv, sync, split_err, stream);
}

namespace {
// e[j] = sum_r c[r, j] * g[r, j] for column-major c, g (one CTA per column).
__global__ void coldot_kernel(int n, const double* __restrict__ c, const double* __restrict__ g,
                              double* __restrict__ e) {
  __shared__ double red[256];
  const long long col = (long long)blockIdx.x * n;
  double s = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) s += c[col + r] * g[col + r];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) e[blockIdx.x] = red[0];
}
}  // namespace

// Orbital energies of the current vectors, e_j = c_j^T F c_j (the diagonal of
// C^T F C), for the SCF's FP64 finish: the pseudo-diagonalisation takes its
// rotation angles from the energies of the last full diagonalisation, which
// carry the level shift of that iteration; the finish refreshes them once.
// ws: 2 n^2 doubles.
extern "C" int mb_orbital_energies_ws(int n, const double* fpacked, const double* c, double* eigs, void* ws,
                                      cudaStream_t stream) {
  double* ff = (double*)ws;
  double* g = ff + (size_t)n * n;
  MB_TRY(mb_unpack_dev(n, fpacked, ff, n, 0, nullptr, stream));
  MB_TRY(mb_dgemm_dev('N', 'N', n, n, n, 1.0, ff, n, c, n, 0.0, g, n, stream));
  coldot_kernel<<<n, 256, 0, stream>>>(n, c, g, eigs);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

extern "C" int mb_pseudo_diag_ws(int n, int nocc, const double* fpacked, double* c, const double* eigs,
                                 unsigned long long* nrot_dev, void* ws, cudaStream_t stream) {
  return mb_pseudo_diag_ex(n, nocc, fpacked, c, eigs, nrot_dev, ws, nullptr, 0, nullptr, 1.5e-7, -1.0, stream);
}

// Rotation sweep alone with caller-given Fmo, tiny and bigeps (the arguments
// of the reference's call_rot_cuda_gpu).  ws as for mb_pseudo_diag_ws.
extern "C" int mb_rot_sweep_ws(int n, int nocc, const double* fmo, const double* eigs, double* c, double bigeps,
                               double tiny, unsigned long long* nrot_dev, void* ws, cudaStream_t stream) {
  const int nvirt = n - nocc;
  if (nocc <= 0 || nvirt <= 0) return MB_OK;
  if (((uintptr_t)ws & 255) != 0) return mb_set_error(MB_ERR_ARG, "rotation workspace must be 256-byte aligned");
  const size_t kvs = (size_t)nocc * nvirt;
  const int to = (nocc + RT - 1) / RT, tv = (nvirt + RT - 1) / RT;
  const size_t kt = (size_t)to * tv * (RT * RT);
  char* b = (char*)ws;
  b += align256(sizeof(double) * (size_t)n * n);
  b += align256(sizeof(double) * (size_t)n * (nocc > nvirt ? nocc : nvirt));
  b += align256(sizeof(double) * kvs);
  double* al = (double*)b; b += align256(sizeof(double) * kt);
  double* be = (double*)b; b += align256(sizeof(double) * kt);
  unsigned char* act = (unsigned char*)b; b += align256(kt);
  unsigned int* tcnt = (unsigned int*)b;
  b += align256(sizeof(unsigned int) * ((size_t)to * tv + 64));
  int* sync = (int*)(b + 256);
  MB_CUDA(cudaMemsetAsync(tcnt, 0, sizeof(unsigned int) * (size_t)to * tv, stream));
  MB_CUDA(cudaMemsetAsync(nrot_dev, 0, sizeof(unsigned long long), stream));
  const long long kv = (long long)nocc * nvirt;
  int cblocks = (int)((kt + 255) / 256);
  if (cblocks > 148 * 8) cblocks = 148 * 8;
  rot_coeff_kernel<<<cblocks, 256, 0, stream>>>(nocc, nvirt, fmo, eigs, nullptr, tiny, bigeps, al, be, act, tcnt,
                                                 nrot_dev, to, tv);
  MB_LAUNCH_CHECK();
  return launch_wavefronts(n, nocc, nvirt, c, al, be, act, tcnt, to, tv, sync, nullptr, stream);
}

extern "C" int mb_pseudo_diag_dev(int n, int nocc, const double* fpacked, double* c, const double* eigs,
                                  long long* nrot_out, cudaStream_t stream) {
  if (n <= 0 || nocc < 0 || nocc > n) return mb_set_error(MB_ERR_ARG, "mb_pseudo_diag_dev: bad size");
  void* ws = nullptr;
  unsigned long long* nrot = nullptr;
  MB_CUDA(mb_malloc_async(&ws, mb_pseudo_ws_bytes(n, nocc), stream));
  MB_CUDA(mb_malloc_async((void**)&nrot, sizeof(unsigned long long), stream));
  MB_CUDA(cudaMemsetAsync(nrot, 0, sizeof(unsigned long long), stream));
  int rc = mb_pseudo_diag_ws(n, nocc, fpacked, c, eigs, nrot, ws, stream);
  unsigned long long h = 0;
  if (rc == MB_OK) {
    cudaError_t e = cudaMemcpyAsync(&h, nrot, sizeof(h), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) rc = mb_set_cuda_error(e, "pseudo_diag nrot", __FILE__, __LINE__);
  }
  cudaFreeAsync(ws, stream);
  cudaFreeAsync(nrot, stream);
  if (nrot_out) *nrot_out = (long long)h;
  return rc;
}
