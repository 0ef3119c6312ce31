// Split-precision GEMMs on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// An FP64 operand x is split into two BF16 planes, x = hi + mid + O(2^-16 x)
// (hi = bf16(x), mid = bf16(x - hi), the residual taken in FP64, so exact),
// and a product is formed from three BF16 products accumulated in FP32:
//     a b ~ a_hi b_hi + a_hi b_mid + a_mid b_hi        (relative error ~2^-16)
// All three go through ONE tensor-core K loop: the K axis runs over three
// segments, and the tile loader picks the plane of each operand per segment
// (A: hi, hi, mid; B: hi, mid, hi).  This is the arithmetic the SCF uses for
// its density and pseudo-diagonalisation GEMMs while max|dP| is above the
// precision switch; FP64 takes over after it.
//
// Operands live in plane buffers: row r of an operand holds [hi(r, 0..Kp) |
// mid(r, 0..Kp)] in BF16, K contiguous, rows padded to 128 and K to 64 with
// zeros, so every TMA box is in bounds and 16-byte aligned.
//
// GEMM kernel: one CTA per 128x128 output tile, 4 warps.  Warp 0 lane 0
// streams 128x64 BF16 tiles of A and B into a 4-stage shared-memory ring with
// TMA (cp.async.bulk.tensor, 128-byte swizzle, no multicast); warp 1 lane 0
// issues tcgen05.mma (M=128, N=128, K=16, kind::f16, BF16 in, FP32 out) into a
// 128-column TMEM accumulator and releases each stage with tcgen05.commit;
// then all 4 warps read the accumulator with tcgen05.ld (each warp its own 32
// TMEM lanes) and write FP64 results.  Every mbarrier wait is bounded (2 s of
// %globaltimer); on expiry the CTA records an error in *err, drains what it
// issued, frees its TMEM and returns without writing.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "mb_common.cuh"

namespace {

constexpr int TM = 128;                  // tile rows of A (TMEM lanes)
constexpr int TN = 128;                  // tile rows of B (accumulator columns)
constexpr int TK = 64;                   // K per stage: 64 BF16 = one 128-byte swizzle row
constexpr int STAGES = 4;
constexpr int TILE_BYTES = TM * TK * 2;  // 16 KiB (TN == TM)
constexpr int STAGE_BYTES = 2 * TILE_BYTES;
constexpr int GEMM_SMEM = STAGES * STAGE_BYTES + 1024;
constexpr int GEMM_THREADS = 128;
constexpr unsigned long long WAIT_NS = 2000000000ull;

// kind::f16 instruction descriptor: FP32 accumulator (bits 4-5 = 1), A and B
// BF16 (bits 7-9 = 1, 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
                           ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for the phase of `bar` with the given parity; false (and *flag set) on
// expiry (limit_ns of %globaltimer) or when another role has already flagged
// an error.
__device__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* flag,
                          unsigned long long limit_ns = WAIT_NS) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = gtimer();
  for (uint32_t it = 1; it != 0; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*flag) return false;
    if ((it & 255u) == 0 && gtimer() - t0 > limit_ns) break;
  }
  *flag = 1;
  return false;
}

// Self-test of the bounded wait: one thread waits on an mbarrier that nothing
// arrives at.  out[0] = 1 when the wait gave up, out[1] = nanoseconds waited.
__global__ void bounded_wait_selftest(unsigned long long limit_ns, long long* out) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int flag;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  flag = 0;
  const unsigned long long t0 = gtimer();
  const bool ok = mbar_wait(&bar, 0, &flag, limit_ns);
  out[0] = ok ? 0 : 1;
  out[1] = (long long)(gtimer() - t0);
}

// Same, but does not give up because of another role's error (used to drain).
__device__ void mbar_drain(uint64_t* bar, uint32_t parity) {
  const unsigned long long t0 = gtimer();
  for (uint32_t it = 0; it < (1u << 30); ++it) {
    if (mbar_try_wait(bar, parity)) return;
    if ((it & 255u) == 0 && gtimer() - t0 > WAIT_NS) return;
  }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* tm, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          dst),
      "l"((unsigned long long)tm), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory matrix descriptor for a K-major tile of 128-byte rows with
// the 128-byte swizzle: start address >> 4, leading offset 1 (unused for
// swizzled K-major), stride offset 1024 B between 8-row groups, descriptor
// version 1 (bit 46), layout SWIZZLE_128B (2 at bit 61).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) | ((uint64_t)1 << 46) |
         ((uint64_t)2 << 61);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive FP32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Plane of each operand in K segment s: A uses hi, hi, mid; B uses hi, mid, hi.
__device__ __forceinline__ int plane_a(int seg) { return seg == 2 ? 1 : 0; }
__device__ __forceinline__ int plane_b(int seg) { return seg == 1 ? 1 : 0; }

enum OutMode { OUT_GENERAL = 0, OUT_PACKED_LOWER = 1 };

// MODE OUT_GENERAL: C(m, n) = alpha * sum + beta * C(m, n), column-major, for
//   the tile (blockIdx.y, blockIdx.x) = (A rows, B rows).
// MODE OUT_PACKED_LOWER: symmetric product of one operand with itself; the
//   block is a tile pair (bm >= bn) of the lower triangle; A rows = the bn
//   block (TMEM lane = column index n of the packed row), B rows = the bm
//   block (accumulator column = row index m); writes P[m(m+1)/2 + n] =
//   alpha * sum for n <= m < M.
template <int MODE>
__global__ void __launch_bounds__(GEMM_THREADS, 1)
    gemm_bf16x3_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int M, int N,
                       int kpb, double alpha, double beta, double* __restrict__ C, int ldc, int* __restrict__ err) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[STAGES];
  __shared__ __align__(8) uint64_t empty_bar[STAGES];
  __shared__ __align__(8) uint64_t done_bar;
  __shared__ uint32_t tmem_slot;
  __shared__ int s_err;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int rowA0, rowB0;
  if (MODE == OUT_GENERAL) {
    rowA0 = blockIdx.y * TM;
    rowB0 = blockIdx.x * TN;
  } else {
    const long long b = blockIdx.x;
    long long r = (long long)((sqrt(8.0 * (double)b + 1.0) - 1.0) * 0.5);
    while (r * (r + 1) / 2 > b) --r;
    while ((r + 1) * (r + 2) / 2 <= b) ++r;
    const int bm = (int)r, bn = (int)(b - r * (r + 1) / 2);
    rowA0 = bn * TM;
    rowB0 = bm * TN;
  }
  const uint32_t base = (smem_u32(smem_raw) + 1023u) & ~1023u;  // 1024-aligned ring for the swizzle
  if (threadIdx.x == 0) {
    s_err = 0;
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&done_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(TN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const int nk = 3 * kpb;
  volatile int* flag = &s_err;

  if (warp == 0 && lane == 0) {
    // ---- TMA producer
    int issued = 0;
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      if (kb >= STAGES && !mbar_wait(&empty_bar[s], ((kb / STAGES) - 1) & 1, flag)) break;
      if (*flag) break;
      const int seg = kb / kpb, kin = kb - seg * kpb;
      const uint32_t sa = base + s * STAGE_BYTES, sb = sa + TILE_BYTES;
      mbar_expect_tx(&full_bar[s], STAGE_BYTES);
      tma_load_2d(sa, &tmA, &full_bar[s], plane_a(seg) * kpb * TK + kin * TK, rowA0);
      tma_load_2d(sb, &tmB, &full_bar[s], plane_b(seg) * kpb * TK + kin * TK, rowB0);
      ++issued;
    }
    if (*flag) {  // let the loads already issued land before the CTA exits
      const int first = issued > STAGES ? issued - STAGES : 0;
      for (int kb = first; kb < issued; ++kb) mbar_drain(&full_bar[kb % STAGES], (kb / STAGES) & 1);
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      if (!mbar_wait(&full_bar[s], (kb / STAGES) & 1, flag)) break;
      tc_fence_after();
      const uint32_t sa = base + s * STAGE_BYTES, sb = sa + TILE_BYTES;
      const uint64_t da = sw128_desc(sa), db = sw128_desc(sb);
#pragma unroll
      for (int kk = 0; kk < TK / 16; ++kk)  // K = 16 per instruction: 32 bytes = 2 descriptor units
        umma_bf16(tmem, da + 2 * kk, db + 2 * kk, (kb > 0 || kk > 0) ? 1u : 0u);
      umma_commit(&empty_bar[s]);
    }
    umma_commit(&done_bar);  // fires when every MMA issued above has completed
  }
  __syncwarp();

  // ---- epilogue: every warp reads its 32 TMEM lanes
  if (!mbar_wait(&done_bar, 0, flag)) mbar_drain(&done_bar, 0);
  __syncthreads();  // every role has finished: s_err is final and CTA-uniform
  const bool ok = (s_err == 0);
  tc_fence_after();
  if (ok) {
    const int arow = rowA0 + warp * 32 + lane;
    for (int c = 0; c < TN; c += 32) {
      uint32_t v[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
      if (MODE == OUT_GENERAL) {
        if (arow < M) {
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int n = rowB0 + c + j;
            if (n < N) {
              double x = alpha * (double)__uint_as_float(v[j]);
              double* dst = C + (long long)n * ldc + arow;
              if (beta != 0.0) x += beta * *dst;
              *dst = x;
            }
          }
        }
      } else {
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int m = rowB0 + c + j;
          if (m < M && arow <= m) C[(long long)m * (m + 1) / 2 + arow] = alpha * (double)__uint_as_float(v[j]);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0 && s_err) atomicExch(err, 1);
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TN) : "memory");
  }
}

// Split an FP64 operand into its BF16 planes.  Element (r, k) of the operand is
// X[k + r*ld] when KCONTIG (K runs down a column of X) and X[r + k*ld]
// otherwise; the output row r is [hi(r, 0..Kp) | mid(r, 0..Kp)], zero outside
// R x K.  32x32 tiles through shared memory keep both sides coalesced.
template <bool KCONTIG>
__global__ void __launch_bounds__(256) split_planes_kernel(int R, int K, const double* __restrict__ X, long long ld,
                                                          __nv_bfloat16* __restrict__ Y, int Kp) {
  __shared__ double t[32][33];  // t[r_local][k_local]
  const int r0 = blockIdx.y * 32, k0 = blockIdx.x * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int i = ty; i < 32; i += 8) {
    if (KCONTIG) {
      const int r = r0 + i, k = k0 + tx;
      t[i][tx] = (r < R && k < K) ? X[(long long)r * ld + k] : 0.0;
    } else {
      const int k = k0 + i, r = r0 + tx;
      t[tx][i] = (r < R && k < K) ? X[(long long)k * ld + r] : 0.0;
    }
  }
  __syncthreads();
  for (int i = ty; i < 32; i += 8) {
    const int r = r0 + i, k = k0 + tx;
    const double v = t[i][tx];
    const __nv_bfloat16 hi = __double2bfloat16(v);
    const __nv_bfloat16 mid = __double2bfloat16(v - (double)__bfloat162float(hi));
    __nv_bfloat16* row = Y + (long long)r * (2 * (long long)Kp);
    row[k] = hi;
    row[Kp + k] = mid;
  }
}

inline int pad_to(int x, int m) { return (x + m - 1) / m * m; }
inline size_t align1k(size_t b) { return (b + 1023) & ~(size_t)1023; }
inline size_t plane_bytes(int rows, int k) { return align1k((size_t)pad_to(rows, TM) * 2 * pad_to(k, TK) * 2); }

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_once;
int g_encode_rc = MB_OK;

int get_encoder() {
  std::call_once(g_once, [] {
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) {
      g_encode_rc = mb_set_error(MB_ERR_CUDA, "cuTensorMapEncodeTiled not available from the driver");
      return;
    }
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    if (cudaFuncSetAttribute(gemm_bf16x3_kernel<OUT_GENERAL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             GEMM_SMEM) != cudaSuccess ||
        cudaFuncSetAttribute(gemm_bf16x3_kernel<OUT_PACKED_LOWER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             GEMM_SMEM) != cudaSuccess)
      g_encode_rc = mb_set_error(MB_ERR_CUDA, "cudaFuncSetAttribute (tcgen05 GEMM shared memory)");
  });
  return g_encode_rc;
}

// Tensor map over a plane buffer of rows_pad x (2 Kp) BF16, box 64 x 128.
int make_map(CUtensorMap* map, const __nv_bfloat16* planes, int rows_pad, int kp) {
  cuuint64_t dims[2] = {(cuuint64_t)2 * kp, (cuuint64_t)rows_pad};
  cuuint64_t strides[1] = {(cuuint64_t)2 * kp * sizeof(__nv_bfloat16)};
  cuuint32_t box[2] = {TK, TM};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)planes, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return mb_set_error(MB_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  return MB_OK;
}

int split(int rows, int k, const double* x, long long ld, bool kcontig, __nv_bfloat16* y, cudaStream_t s) {
  const int rp = pad_to(rows, TM), kp = pad_to(k, TK);
  dim3 grid(kp / 32, rp / 32), block(32, 8);
  if (kcontig) split_planes_kernel<true><<<grid, block, 0, s>>>(rows, k, x, ld, y, kp);
  else split_planes_kernel<false><<<grid, block, 0, s>>>(rows, k, x, ld, y, kp);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

}  // namespace

extern "C" size_t mb_gemm_split_ws_bytes(int m, int n, int k) {
  if (m <= 0 || n <= 0 || k <= 0) return 0;
  return plane_bytes(m, k) + plane_bytes(n, k) + 1024;
}

// C = alpha * op(A) op(B) + beta * C (column-major, BLAS conventions) with the
// three-product BF16 split on the tensor cores.  ws: mb_gemm_split_ws_bytes.
extern "C" int mb_gemm_split_ws(char transa, char transb, int m, int n, int k, double alpha, const double* a, int lda,
                                const double* b, int ldb, double beta, double* c, int ldc, void* ws, size_t ws_bytes,
                                int* err_dev, cudaStream_t stream) {
  if (m < 0 || n < 0 || k < 0 || !err_dev) return mb_set_error(MB_ERR_ARG, "mb_gemm_split: bad args");
  if (m == 0 || n == 0) return MB_OK;
  if (k == 0) return mb_set_error(MB_ERR_ARG, "mb_gemm_split: k = 0 is not supported");
  if (!ws || ws_bytes < mb_gemm_split_ws_bytes(m, n, k) || ((uintptr_t)ws & 1023))
    return mb_set_error(MB_ERR_ARG, "mb_gemm_split: workspace too small or not 1024-byte aligned");
  MB_TRY(get_encoder());
  const bool ta = (transa == 'T' || transa == 't' || transa == 'C' || transa == 'c');
  const bool tb = (transb == 'T' || transb == 't' || transb == 'C' || transb == 'c');
  __nv_bfloat16* pa = (__nv_bfloat16*)ws;
  __nv_bfloat16* pb = (__nv_bfloat16*)((char*)ws + plane_bytes(m, k));
  // row r of op(A) is K-contiguous when A is transposed; row r of op(B)^T when B is not
  MB_TRY(split(m, k, a, lda, ta, pa, stream));
  MB_TRY(split(n, k, b, ldb, !tb, pb, stream));
  CUtensorMap ma, mb;
  MB_TRY(make_map(&ma, pa, pad_to(m, TM), pad_to(k, TK)));
  MB_TRY(make_map(&mb, pb, pad_to(n, TN), pad_to(k, TK)));
  dim3 grid(pad_to(n, TN) / TN, pad_to(m, TM) / TM);
  gemm_bf16x3_kernel<OUT_GENERAL><<<grid, GEMM_THREADS, GEMM_SMEM, stream>>>(ma, mb, m, n, pad_to(k, TK) / TK, alpha,
                                                                            beta, c, ldc, err_dev);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

extern "C" size_t mb_density_split_ws_bytes(int n, int nocc) {
  if (n <= 0 || nocc <= 0) return 0;
  return plane_bytes(n, nocc) + 1024;
}

// Packed P (lower triangle by rows) = occ * C[:, 0:nocc] C[:, 0:nocc]^T with
// the three-product BF16 split; C column-major with leading dimension ldc.
extern "C" int mb_density_split_ws(int n, int nocc, double occ, const double* c, int ldc, double* p, void* ws,
                                   size_t ws_bytes, int* err_dev, cudaStream_t stream) {
  if (n <= 0 || nocc < 0 || nocc > n || !err_dev) return mb_set_error(MB_ERR_ARG, "mb_density_split: bad args");
  if (nocc == 0) {
    MB_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * (size_t)n * (n + 1) / 2, stream));
    return MB_OK;
  }
  if (!ws || ws_bytes < mb_density_split_ws_bytes(n, nocc) || ((uintptr_t)ws & 1023))
    return mb_set_error(MB_ERR_ARG, "mb_density_split: workspace too small or not 1024-byte aligned");
  MB_TRY(get_encoder());
  __nv_bfloat16* pc = (__nv_bfloat16*)ws;
  MB_TRY(split(n, nocc, c, ldc, false, pc, stream));  // row r = C(r, 0..nocc), strided in C
  CUtensorMap mc;
  MB_TRY(make_map(&mc, pc, pad_to(n, TM), pad_to(nocc, TK)));
  const long long t = pad_to(n, TM) / TM;
  mb_kstat_mark(MB_KSTAT_DENSITY, stream, true);
  gemm_bf16x3_kernel<OUT_PACKED_LOWER><<<(unsigned)(t * (t + 1) / 2), GEMM_THREADS, GEMM_SMEM, stream>>>(
      mc, mc, n, n, pad_to(nocc, TK) / TK, occ, 0.0, p, 0, err_dev);
  MB_LAUNCH_CHECK();
  mb_kstat_mark(MB_KSTAT_DENSITY, stream, false);
  return MB_OK;
}

// The GEMM's bounded mbarrier wait, made to run out: limit_ns (at most 0.1 s)
// on a barrier that never completes.  out_dev: two long longs (gave up,
// nanoseconds waited).  No reference counterpart: a check of this library's
// failure path that faults nothing.
extern "C" int mb_selftest_bounded_wait(unsigned long long limit_ns, long long* out_dev, cudaStream_t stream) {
  if (!out_dev || limit_ns == 0 || limit_ns > 100000000ull)
    return mb_set_error(MB_ERR_ARG, "mb_selftest_bounded_wait: limit must be 1 ns .. 0.1 s");
  bounded_wait_selftest<<<1, 32, 0, stream>>>(limit_ns, out_dev);
  MB_LAUNCH_CHECK();
  return MB_OK;
}
