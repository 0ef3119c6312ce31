// Two- and one-centre Fock build for the dense NDDO SCF (sp basis).
//
// Replaces fock2 (SCF/fock2.F90:16-374, sp branches :149-298), jab
// (integrals/jab.F90), kab (integrals/kab.F90) and fock1 (SCF/fock1.F90) as
// called from iter (SCF/iter.F90:553), including iter's level-shifted start
// value F = H + shift*PA + 1e-16*i, F_ii -= shift (SCF/iter.F90:317-324).
//
// Result is bit-identical to the reference loop order: every element of F
// receives its contributions in the same sequence (partner atoms in ascending
// order with the one-centre term at the atom's own position), each
// contribution is formed with the same term order, and no FMA is used.
//
// Design: two passes over a staging array.
//
// Pass 1 (fock2_pairs) evaluates every ordered atom pair (A, B), B != A, one
// pair per lane: B's Coulomb contribution to A's diagonal block goes to the
// staging array, and for B < A the exchange block F(A, B) goes straight to F.
// Work is a queue of warp items, taken with an atomic counter:
//   HH  heavy A, 32 heavy partners: the 10 x 10 W blocks stream through the
//       warp as 16 row tiles, in the order of jab's density gather (row
//       pair(x, y) at step 4x + y).  That order is also kab's (mu, lam)
//       order, so the exchange sums and both Coulomb sums keep the
//       reference's term sequence with one W row live per lane.
//   X   every pair with a light atom: 128 partners, four tiles of one block
//       (at most ten doubles) per lane.
// A tile (32 lanes x up to 10 doubles) is copied with cp.async by the whole
// warp over the concatenated blocks -- consecutive lanes copy consecutive
// addresses -- into per-lane slots of 11 doubles (odd, so the lanes' reads
// hit distinct banks); each warp keeps four tiles in flight.
//
// Pass 2 (fock2_fold) runs one CTA per atom: it streams the atom's staged
// contributions through shared memory in partner order, and up to ten owner
// threads fold them into iter's start value, adding fock1's one-centre term
// at the atom's own position.  A light atom's two staged values per partner
// are fock2's one or two additions; an absent second addition is staged as
// -0.0, which leaves every sum unchanged bit for bit.
//
// Traffic: W once per ordered pair (the second read of a block mostly from
// L2), the staged contributions written and read once, one pass over P, PA,
// H and F.
#include <cstdint>
#include <mutex>

#include "mb_common.cuh"

namespace {

constexpr int kWarps = 4;          // warps per CTA of the pair pass
constexpr int kDepth = 4;          // tiles in flight per warp
static_assert(kDepth >= 4 && kDepth <= 4, "an HX item stages its four tiles at once, and cp_async_wait takes n <= 3");
constexpr int kSlot = 11;          // doubles per lane slot in a tile
constexpr int kTile = 32 * kSlot;  // doubles per tile
constexpr int kStageW = 10;        // staged doubles per (A, B) record of a heavy A (a light A uses 2)
constexpr int kFoldThreads = 128;  // pass 2: threads per CTA and partners per chunk
constexpr int kFoldDepth = 3;      // pass 2: chunks in flight

__host__ __device__ constexpr int pair1(int a, int b) {  // 1-based pair index of orbitals a, b (1..4)
  return a > b ? a * (a - 1) / 2 + b : b * (b - 1) / 2 + a;
}

// jab's density gather: term m uses pair index pair1(m / 4 + 1, m % 4 + 1).
__host__ __device__ constexpr int pidx(int m) { return pair1(m / 4 + 1, m % 4 + 1); }

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

// Wait until at most n of this thread's committed groups are pending (n <= 3).
__device__ __forceinline__ void cp_async_wait(int n) {
  switch (n) {
    case 0: asm volatile("cp.async.wait_group 0;\n" ::: "memory"); break;
    case 1: asm volatile("cp.async.wait_group 1;\n" ::: "memory"); break;
    case 2: asm volatile("cp.async.wait_group 2;\n" ::: "memory"); break;
    default: asm volatile("cp.async.wait_group 3;\n" ::: "memory"); break;
  }
}

struct FockArgs {
  MbAtoms at;
  double* f;
  const double* h;
  const double* ptot;
  const double* pa;
  const double* w;
  double shift;
  int use_shift;
};

// Workspace: counts (heavy atoms, light atoms, item counter), the heavy and
// light atom lists (ascending), and the staging array.
struct FockWs {
  int* counts;
  int* hlist;
  int* llist;
  double* stage;
};

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

FockWs carve(void* ws, int numat) {
  char* p = (char*)ws;
  FockWs r;
  r.counts = (int*)p;
  p += 256;
  r.hlist = (int*)p;
  p += align256(sizeof(int) * (size_t)numat);
  r.llist = (int*)p;
  p += align256(sizeof(int) * (size_t)numat);
  r.stage = (double*)p;
  return r;
}

// Staged record of partner B for atom A: a heavy A's ten values at
// (A*numat + B)*10, a light A's two at A*numat*10 + 2B.
__device__ __forceinline__ long long rec_off(int A, int numat, int B, bool heavy) {
  return (long long)A * numat * kStageW + (long long)B * (heavy ? kStageW : 2);
}

__device__ __forceinline__ double f_start(const FockArgs& a, long long idx, bool diag) {
  if (!a.use_shift) return __ldg(a.h + idx);
  double v = DADD(DADD(__ldg(a.h + idx), DMUL(a.shift, __ldg(a.pa + idx))), DMUL((double)(idx + 1), 1.0e-16));
  if (diag) v = DSUB(v, a.shift);
  return v;
}

// f_start with PA(idx) already in a register.
__device__ __forceinline__ double f_start_pa(const FockArgs& a, long long idx, double pa_idx) {
  if (!a.use_shift) return __ldg(a.h + idx);
  return DADD(DADD(__ldg(a.h + idx), DMUL(a.shift, pa_idx)), DMUL((double)(idx + 1), 1.0e-16));
}

// Heavy atom B's diagonal density block in jab's 4 x 4 gather order,
// pjb[x*4 + y] = P(max, min).
__device__ __forceinline__ void diag_block(const FockArgs& a, int fB, double* pjb) {
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) {
      const int r = fB + (x > y ? x : y), cc = fB + (x < y ? x : y);
      pjb[x * 4 + y] = __ldg(a.ptot + mb_tri(r, cc));
    }
}

// A light atom's two additions from heavy B's diagonal block (fock2's
// "ib - ia >= 3" / "jb - ja >= 3" branches with one s orbital on the light
// atom): c[0] = 2 * off-diagonal sum, c[1] = diagonal sum.
__device__ __forceinline__ void light_from_heavy(const FockArgs& a, int fB, const double* wk, double* c) {
  double sumoff = 0.0, sumdia = 0.0;
  int k = 0;
#pragma unroll
  for (int i = 0; i <= 3; ++i) {
#pragma unroll
    for (int j = 1; j <= i; ++j) sumoff = DADD(sumoff, DMUL(__ldg(a.ptot + mb_tri(fB + i, fB + j - 1)), __ldg(wk + j + k - 1)));
    k += i + 1;
    sumdia = DADD(sumdia, DMUL(__ldg(a.ptot + mb_tri(fB + i, fB + i)), __ldg(wk + k - 1)));
  }
  c[0] = DMUL(sumoff, 2.0);
  c[1] = sumdia;
}

// Warp-cooperative tile copy: 32 windows of ten doubles, window i at
// src[i] + add, land in slots 0..31.  Flat element q = 32r + lane of round r
// is element q % 10 of window q / 10, so consecutive lanes copy consecutive
// addresses of one window or the next.  Called by all 32 lanes.
__device__ __forceinline__ void issue_win10(double* tile, const unsigned long long* src, long long add, int lane) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const int q = 32 * r + lane;
    const int i = q / 10, e = q - 10 * i;
    cp_async8(tile + i * kSlot + e, (const double*)src[i] + add + e);
  }
}

// W block of the ordered pair (A, B): for B < A the lA x lB block of row A
// (B's pair index fastest), else the lB x lA block of row B.
__device__ __forceinline__ const double* w_block(const FockArgs& a, int A, int lA, long long wrowA, int B,
                                                 int lB) {
  return B < A ? a.w + wrowA + (long long)lA * __ldg(a.at.cum + B)
               : a.w + __ldg(a.at.wrow + B) + (long long)lB * __ldg(a.at.cum + A);
}

// One pair with at least one light atom, W block read from global memory.
__device__ __forceinline__ void pair_x(const FockArgs& a, int A, int fA, int nA, int B, const double* wk,
                                       double* out) {
  const int fB = __ldg(a.at.first + B), nB = __ldg(a.at.nor + B);
  if (nA == 4) {  // heavy A, light B: ten Coulomb terms
    const double pb = __ldg(a.ptot + (mb_tri(fB, fB)));
#pragma unroll
    for (int q = 0; q < 10; ++q) out[q] = DMUL(pb, __ldg(wk + q));
    if (B < A) {  // kab on the 4 x 1 block
      double pj[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) pj[j] = __ldg(a.pa + (mb_tri(fA + j, fB)));
#pragma unroll
      for (int i = 1; i <= 4; ++i) {
        double sum = 0.0;
#pragma unroll
        for (int j = 1; j <= 4; ++j) sum = DADD(sum, DMUL(pj[j - 1], __ldg(wk + pair1(i, j) - 1)));
        const long long idx = mb_tri(fA + i - 1, fB);
        a.f[idx] = DSUB(f_start(a, idx, false), sum);
      }
    }
  } else if (nB == 4) {  // light A, heavy B: two additions
    light_from_heavy(a, fB, wk, out);
    if (B < A) {  // kab on the 1 x 4 block
      double pl[4];
#pragma unroll
      for (int l = 0; l < 4; ++l) pl[l] = __ldg(a.pa + (mb_tri(fA, fB + l)));
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        double sum = 0.0;
#pragma unroll
        for (int l = 1; l <= 4; ++l) sum = DADD(sum, DMUL(pl[l - 1], __ldg(wk + pair1(i + 1, l) - 1)));
        const long long idx = mb_tri(fA, fB + i);
        a.f[idx] = DSUB(f_start(a, idx, false), sum);
      }
    }
  } else {  // two light atoms: one addition
    out[0] = DMUL(__ldg(a.ptot + (mb_tri(fB, fB))), __ldg(wk));
    out[1] = -0.0;
    if (B < A) {
      const long long idx = mb_tri(fA, fB);
      a.f[idx] = DSUB(f_start(a, idx, false), DMUL(__ldg(a.pa + idx), __ldg(wk)));
    }
  }
}

// Heavy and light atom lists (ascending), their lengths, and a zero item
// counter for the pair pass.  One CTA.
__global__ void fock2_lists(MbAtoms at, FockWs ws) {
  __shared__ int s_warp[32], s_base[2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  if (tid == 0) { s_base[0] = 0; s_base[1] = 0; }
  __syncthreads();
  for (int b0 = 0; b0 < at.numat; b0 += blockDim.x) {
    const int A = b0 + tid;
    const bool valid = A < at.numat;
    const bool heavy = valid && at.nor[A] == 4;
    const unsigned hb = __ballot_sync(0xffffffffu, heavy), vb = __ballot_sync(0xffffffffu, valid);
    const unsigned below = (1u << lane) - 1u;
    const int hpre = __popc(hb & below), vpre = __popc(vb & below);
    if (lane == 0) s_warp[warp] = (__popc(hb) << 16) | __popc(vb);
    __syncthreads();
    int hoff = 0, voff = 0;
    for (int w = 0; w < warp; ++w) { hoff += s_warp[w] >> 16; voff += s_warp[w] & 0xffff; }
    if (heavy) ws.hlist[s_base[0] + hoff + hpre] = A;
    else if (valid) ws.llist[s_base[1] + (voff + vpre) - (hoff + hpre)] = A;
    __syncthreads();
    if (tid == 0) {
      int ht = 0, vt = 0;
      for (int w = 0; w < nw; ++w) { ht += s_warp[w] >> 16; vt += s_warp[w] & 0xffff; }
      s_base[0] += ht;
      s_base[1] += vt - ht;
    }
    __syncthreads();
  }
  if (tid == 0) {
    ws.counts[0] = s_base[0];
    ws.counts[1] = s_base[1];
    ws.counts[2] = 0;
  }
}

__global__ void __launch_bounds__(32 * kWarps, 3) fock2_pairs(FockArgs a, FockWs ws) {
  extern __shared__ double s_tiles[];  // kWarps x kDepth tiles
  __shared__ unsigned long long s_src[kWarps][4][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double* tiles = s_tiles + (size_t)warp * kDepth * kTile;
  const int numat = a.at.numat;
  const int nh = ws.counts[0], nl = ws.counts[1];
  const int th = (nh + 31) / 32, tl = (nl + 127) / 128, ta = (numat + 127) / 128;
  const long long r1 = (long long)nh * th, r2 = r1 + (long long)nh * tl, total = r2 + (long long)nl * ta;

  for (;;) {
    long long item = 0;
    if (lane == 0) item = atomicAdd(&ws.counts[2], 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= total) break;

    if (item < r1) {
      // HH: heavy A, heavy partners hlist[32 t + lane]; W rows through the tile ring
      const int A = __ldg(ws.hlist + (item / th));
      const int hi = 32 * (int)(item % th) + lane;
      const int B = hi < nh ? __ldg(ws.hlist + hi) : A;
      const bool act = B != A, lower = B < A;
      const int fA = __ldg(a.at.first + A), fB = __ldg(a.at.first + B);
      s_src[warp][0][lane] = (unsigned long long)(act ? w_block(a, A, 10, __ldg(a.at.wrow + A), B, 10) : a.w);
      __syncwarp();
#pragma unroll
      for (int m = 0; m < kDepth; ++m) {
        issue_win10(tiles + m * kTile, s_src[warp][0], (pidx(m) - 1) * 10, lane);
        cp_async_commit();
      }
      double* rec = ws.stage + rec_off(A, numat, B, true);
      double pj[16], pk[16], hm[4], sa[10];  // sa[0..3]: a lower lane's exchange sums of the current mu
      if (act) {
        diag_block(a, fB, pj);
        if (lower) {
#pragma unroll
          for (int x = 0; x < 4; ++x)
#pragma unroll
            for (int y = 0; y < 4; ++y) pk[x * 4 + y] = __ldg(a.pa + (mb_tri(fA + x, fB + y)));
        }
      }
#pragma unroll
      for (int m = 0; m < 16; ++m) {
        const int x = m / 4, y = m % 4;
        if (act && lower && y == 0) {
#pragma unroll
          for (int nu = 0; nu < 4; ++nu) hm[nu] = __ldg(a.h + (mb_tri(fA + x, fB + nu)));
        }
        cp_async_wait(m + kDepth <= 16 ? kDepth - 1 : 15 - m);
        __syncwarp();
        const double* row = tiles + (m % kDepth) * kTile + lane * kSlot;  // row pidx(m) of the block
        if (act) {
          if (lower) {
            if (x <= y) {  // first visit of row pidx(m): A's Coulomb term for that pair index
              double sb = DMUL(pj[0], row[pidx(0) - 1]);
#pragma unroll
              for (int mm = 1; mm < 16; ++mm) sb = DADD(sb, DMUL(pj[mm], row[pidx(mm) - 1]));
              rec[pidx(m) - 1] = sb;
            }
            // kab: this row is pair(mu, lam) with mu = x + 1, lam = y + 1
#pragma unroll
            for (int nu = 1; nu <= 4; ++nu)
#pragma unroll
              for (int sig = 1; sig <= 4; ++sig) {
                const double tt = DMUL(pk[y * 4 + sig - 1], row[pair1(nu, sig) - 1]);
                sa[nu - 1] = (y == 0 && sig == 1) ? tt : DADD(sa[nu - 1], tt);
              }
            if (y == 3) {
#pragma unroll
              for (int nu = 0; nu < 4; ++nu) {
                const long long idx = mb_tri(fA + x, fB + nu);
                const double st = a.use_shift
                                      ? DADD(DADD(hm[nu], DMUL(a.shift, pk[x * 4 + nu])), DMUL((double)(idx + 1), 1.0e-16))
                                      : hm[nu];
                a.f[idx] = DSUB(st, sa[nu]);
              }
            }
          } else {
            // block (B, A): term m of each of A's ten elements
#pragma unroll
            for (int q = 0; q < 10; ++q) {
              const double tt = DMUL(pj[m], row[q]);
              sa[q] = m == 0 ? tt : DADD(sa[q], tt);
            }
            if (m == 15) {
#pragma unroll
              for (int q = 0; q < 10; ++q) rec[q] = sa[q];
            }
          }
        }
        __syncwarp();
        if (m + kDepth < 16) {
          issue_win10(tiles + (m % kDepth) * kTile, s_src[warp][0], (pidx(m + kDepth) - 1) * 10, lane);
          cp_async_commit();
        }
      }
    } else if (item < r2) {
      // HX: heavy A, light partners llist[128 t + 32 g + lane]; one ten-double block each
      const long long j = item - r1;
      const int A = __ldg(ws.hlist + (j / tl));
      const int base = (int)(j % tl) * 128;
      const int fA = __ldg(a.at.first + A);
      const long long wrowA = __ldg(a.at.wrow + A);
      int Bs[4];
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        const int idx = base + 32 * g + lane;
        const int B = idx < nl ? __ldg(ws.llist + idx) : -1;
        Bs[g] = B;
        s_src[warp][g][lane] = (unsigned long long)(B >= 0 ? w_block(a, A, 10, wrowA, B, 1) : a.w);
      }
      __syncwarp();
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        issue_win10(tiles + g * kTile, s_src[warp][g], 0, lane);
        cp_async_commit();
      }
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        const int B = Bs[g];
        double pb = 0.0, pj[4];
        int fB = 0;
        if (B >= 0) {
          fB = __ldg(a.at.first + B);
          pb = __ldg(a.ptot + (mb_tri(fB, fB)));
          if (B < A) {
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) pj[jj] = __ldg(a.pa + (mb_tri(fA + jj, fB)));
          }
        }
        cp_async_wait(3 - g);
        __syncwarp();
        if (B >= 0) {
          const double* wk = tiles + g * kTile + lane * kSlot;
          double* rec = ws.stage + rec_off(A, numat, B, true);
#pragma unroll
          for (int q = 0; q < 10; ++q) rec[q] = DMUL(pb, wk[q]);
          if (B < A) {  // kab on the 4 x 1 block
#pragma unroll
            for (int i = 1; i <= 4; ++i) {
              double sum = 0.0;
#pragma unroll
              for (int jj = 1; jj <= 4; ++jj) sum = DADD(sum, DMUL(pj[jj - 1], wk[pair1(i, jj) - 1]));
              const long long idx = mb_tri(fA + i - 1, fB);
              a.f[idx] = DSUB(f_start_pa(a, idx, pj[i - 1]), sum);
            }
          }
        }
      }
      __syncwarp();
    } else {
      // LX: light A, partners 128 t + 32 g + lane; blocks of at most ten
      // doubles read straight from W (row A's are contiguous over B < A)
      const long long j = item - r2;
      const int A = __ldg(ws.llist + (j / ta));
      const int base = (int)(j % ta) * 128;
      const int fA = __ldg(a.at.first + A);
      const long long wrowA = __ldg(a.at.wrow + A);
#pragma unroll 1
      for (int g = 0; g < 4; ++g) {
        const int B = base + 32 * g + lane;
        if (B < numat && B != A) {
          const double* wk = w_block(a, A, 1, wrowA, B, __ldg(a.at.lim + B));
          double out[10];
          pair_x(a, A, fA, 1, B, wk, out);
          double* rec = ws.stage + rec_off(A, numat, B, false);
          rec[0] = out[0];
          rec[1] = out[1];
        }
      }
    }
  }
}

// Pass 2: one CTA per atom; owners e < lim[A] fold in partner order.
__global__ void __launch_bounds__(kFoldThreads) fock2_fold(FockArgs a, FockWs ws) {
  extern __shared__ double s_buf[];  // kFoldDepth chunks of kFoldThreads records
  const int A = blockIdx.x, tid = threadIdx.x;
  const int numat = a.at.numat;
  const int fA = __ldg(a.at.first + A), nA = __ldg(a.at.nor + A), lA = __ldg(a.at.lim + A);
  const bool heavy = nA == 4;
  const int wv = heavy ? kStageW : 2;
  const long long wrowA = __ldg(a.at.wrow + A);
  const double* src = ws.stage + rec_off(A, numat, 0, heavy);

  double run = 0.0, f1 = 0.0;
  long long own_idx = 0;
  if (tid < lA) {
    int iw = 1, jw = 1;  // local (row, col), 1-based, from packed element tid
    {
      int e = tid, r = 1;
      while (e >= r) { e -= r; ++r; }
      iw = r; jw = e + 1;
    }
    own_idx = mb_tri(fA + iw - 1, fA + jw - 1);
    run = f_start(a, own_idx, iw == jw);
    // fock1 (SCF/fock1.F90): one-centre Coulomb and exchange for element (iw, jw)
    const double* w1 = a.w + wrowA + (long long)lA * __ldg(a.at.cum + A);
    const int ilim = lA;
    const int ijw = iw * (iw - 1) / 2 + jw;
    double sum = 0.0;
    for (int kw = 1; kw <= nA; ++kw)
      for (int lw = 1; lw <= nA; ++lw) {
        int ip = kw > lw ? kw : lw, jp = kw < lw ? kw : lw;
        long long ijp = mb_tri(fA + ip - 1, fA + jp - 1);
        int klw = ip * (ip - 1) / 2 + jp;
        int im = kw > jw ? kw : jw, jm = kw < jw ? kw : jw;
        int ikw = im * (im - 1) / 2 + jm;
        im = lw > iw ? lw : iw; jm = lw < iw ? lw : iw;
        int jlw = im * (im - 1) / 2 + jm;
        sum = DSUB(DADD(sum, DMUL(__ldg(a.ptot + ijp), w1[(ijw - 1) + ilim * (klw - 1)])),
                   DMUL(__ldg(a.pa + ijp), w1[(ikw - 1) + ilim * (jlw - 1)]));
      }
    f1 = sum;
  }

  const int nchunk = (numat + kFoldThreads - 1) / kFoldThreads;
  for (int k = 0; k < kFoldDepth + nchunk; ++k) {
    if (k >= kFoldDepth) {
      // fold chunk c = k - kFoldDepth
      const int c = k - kFoldDepth;
      cp_async_wait(kFoldDepth - 1);
      __syncthreads();
      if (tid < lA) {
        const double* buf = s_buf + (c % kFoldDepth) * kFoldThreads * kStageW;
        const int b0 = c * kFoldThreads;
        const int nb = min(kFoldThreads, numat - b0);
        const int tA = (A >= b0 && A < b0 + nb) ? A - b0 : nb;
        if (heavy) {
#pragma unroll 8
          for (int t = 0; t < tA; ++t) run = DADD(run, buf[t * kStageW + tid]);
          if (tA < nb) {
            run = DADD(run, f1);
#pragma unroll 8
            for (int t = tA + 1; t < nb; ++t) run = DADD(run, buf[t * kStageW + tid]);
          }
        } else {
#pragma unroll 8
          for (int t = 0; t < tA; ++t) run = DADD(DADD(run, buf[2 * t]), buf[2 * t + 1]);
          if (tA < nb) {
            run = DADD(run, f1);
#pragma unroll 8
            for (int t = tA + 1; t < nb; ++t) run = DADD(DADD(run, buf[2 * t]), buf[2 * t + 1]);
          }
        }
      }
      __syncthreads();
    }
    // prefetch chunk k into slot k % kFoldDepth (the slot chunk k - kFoldDepth just left)
    if (k < nchunk) {
      const int b0 = k * kFoldThreads;
      const int n = min(kFoldThreads, numat - b0) * wv;
      double* dst = s_buf + (k % kFoldDepth) * kFoldThreads * kStageW;
      for (int q = tid; q < n; q += kFoldThreads) cp_async8(dst + q, src + (long long)b0 * wv + q);
    }
    cp_async_commit();
  }
  cp_async_wait(0);
  if (tid < lA) a.f[own_idx] = run;
}

int fock_attrs() {
  static std::mutex mu;
  static bool done[64] = {};
  int dev = 0;
  MB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return mb_set_error(MB_ERR_UNSUPPORTED, "Fock build: device index out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (!done[dev]) {
    MB_CUDA(cudaFuncSetAttribute(fock2_pairs, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(double) * kWarps * kDepth * kTile)));
    MB_CUDA(cudaFuncSetAttribute(fock2_pairs, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    MB_CUDA(cudaFuncSetAttribute(fock2_fold, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(double) * kFoldDepth * kFoldThreads * kStageW)));
    done[dev] = true;
  }
  return MB_OK;
}

}  // namespace

extern "C" size_t mb_fock2_ws_bytes(int numat) {
  if (numat <= 0) return 0;
  return 256 + 2 * align256(sizeof(int) * (size_t)numat) + sizeof(double) * kStageW * (size_t)numat * numat;
}

extern "C" int mb_fock2_ws(const MbAtomsDev* atoms, double* f, const double* h, const double* ptot,
                           const double* pa, const double* w, double shift, int use_shift, void* ws,
                           size_t ws_bytes, cudaStream_t stream) {
  if (!atoms || atoms->numat <= 0) return mb_set_error(MB_ERR_ARG, "mb_fock2_ws: no atoms");
  if (!ws || ws_bytes < mb_fock2_ws_bytes(atoms->numat))
    return mb_set_error(MB_ERR_ARG, "mb_fock2_ws: workspace smaller than mb_fock2_ws_bytes(numat)");
  if (((uintptr_t)ws & 255) != 0) return mb_set_error(MB_ERR_ARG, "mb_fock2_ws: workspace not 256-byte aligned");
  MB_TRY(fock_attrs());
  FockArgs a;
  a.at.numat = atoms->numat;
  a.at.first = atoms->first;
  a.at.nor = atoms->nor;
  a.at.lim = atoms->lim;
  a.at.wrow = atoms->wrow;
  a.at.cum = atoms->cum;
  a.f = f;
  a.h = h;
  a.ptot = ptot;
  a.pa = pa;
  a.w = w;
  a.shift = shift;
  a.use_shift = use_shift;
  const FockWs fw = carve(ws, atoms->numat);
  int dev = 0, sms = 0;
  MB_CUDA(cudaGetDevice(&dev));
  MB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  mb_kstat_mark(MB_KSTAT_FOCK, stream, true);
  fock2_lists<<<1, 1024, 0, stream>>>(a.at, fw);
  MB_LAUNCH_CHECK();
  fock2_pairs<<<sms * 3, 32 * kWarps, sizeof(double) * kWarps * kDepth * kTile, stream>>>(a, fw);
  MB_LAUNCH_CHECK();
  fock2_fold<<<atoms->numat, kFoldThreads, sizeof(double) * kFoldDepth * kFoldThreads * kStageW, stream>>>(a,
                                                                                                             fw);
  MB_LAUNCH_CHECK();
  mb_kstat_mark(MB_KSTAT_FOCK, stream, false);
  return MB_OK;
}

extern "C" int mb_fock2_dev(const MbAtomsDev* atoms, double* f, const double* h, const double* ptot,
                            const double* pa, const double* w, double shift, int use_shift,
                            cudaStream_t stream) {
  if (!atoms || atoms->numat <= 0) return mb_set_error(MB_ERR_ARG, "mb_fock2_dev: no atoms");
  const size_t bytes = mb_fock2_ws_bytes(atoms->numat);
  void* ws = nullptr;
  MB_CUDA(mb_malloc_async(&ws, bytes, stream));
  const int rc = mb_fock2_ws(atoms, f, h, ptot, pa, w, shift, use_shift, ws, bytes, stream);
  const cudaError_t fe = cudaFreeAsync(ws, stream);
  if (rc != MB_OK) return rc;
  if (fe != cudaSuccess) return mb_set_cuda_error(fe, "cudaFreeAsync", __FILE__, __LINE__);
  return MB_OK;
}
