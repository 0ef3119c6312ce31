// Learned initial guess: an atom-pair MLP that predicts the blocks of the
// starting density matrix from the local geometry.
//
// The reference has no counterpart: MOPAC starts iter from the diagonal guess
// (moldat.F90:731-760) or from a density read with OLDENS
// (SCF/iter.F90:151-158).  A predicted density enters the SCF the way an
// OLDENS density does, so the converged result is the SCF's, not the
// network's; a bad prediction can only cost iterations.
//
// Pipeline (all on the device):
//   1. pairs: every atom's own block and every atom pair closer than rpair,
//      written into one segment per pair type (count pass + emit pass);
//   2. frames and descriptors: a warp per pair.  The frame's z axis runs along
//      the pair (own blocks: towards the nearest neighbour), x towards the
//      nearest neighbour with a clear perpendicular component (distance ranks
//      round(r^2 * 1e5), ties by atom index, so rigid fragments with equal
//      bond lengths pick a frame deterministically).  Descriptors: for each
//      centre, Gaussian radial shells (8, cut off smoothly at 6 A) times ten
//      angular monomials of the neighbour direction in the frame, per element
//      class (H, heavy), plus 16 radial functions of the pair distance, plus
//      each centre's long-range electrostatic environment (potential, field
//      and field gradient of fixed reference charges on all other atoms, in
//      the frame; no cutoff);
//   3. normalisation to BF16 with per-type statistics;
//   4. the MLP (DIN -> 128 -> 128 -> 128 -> 16, SiLU) as BF16 tensor-core
//      GEMMs with FP32 accumulation (mma.sync m16n8k16), one weight set per
//      pair type;
//   5. assembly: each local block is de-normalised, rotated back and written
//      into the packed lower triangle (each packed element has one owner).
// Training uses the same GEMM kernel for the backward pass (dW = dZ^T A and
// dA = dZ W with the SiLU derivative fused) and an Adam kernel that also
// refreshes the BF16 weight copies.
#include <math.h>
#include <string.h>

#include <vector>

#include "mb_common.cuh"

namespace {

constexpr int DIN = MB_GUESS_DIN;
constexpr int HID = MB_GUESS_HID;
constexpr int DOUT = MB_GUESS_DOUT;
constexpr int NT = MB_GUESS_NTYPES;
constexpr int PER_CENTER = 160;
constexpr int NRAD = 8;
constexpr int NANG = 10;
constexpr int NPAIR_RBF = 16;
constexpr int NLR = 10;
constexpr int LR0 = 2 * PER_CENTER + NPAIR_RBF;
// reference charges of the long-range descriptor: PM7 Mulliken charges of an
// isolated water molecule
constexpr double QREF_H = 0.32226;
constexpr double QREF_HEAVY = -0.64452;
constexpr double RC = 6.0;
constexpr double RAD_SIG = 0.65;
constexpr double PAIR_SIG = 0.35;
constexpr double PERP_MIN2 = 0.01;
constexpr double QSCALE = 1.0e5;

// Blob layout per type (floats): in_mean, in_std, W1, b1, W2, b2, W3, b3, W4,
// b4, out_mean, out_std.
constexpr long long OFF_IN_MEAN = 0;
constexpr long long OFF_IN_STD = OFF_IN_MEAN + DIN;
constexpr long long OFF_W1 = OFF_IN_STD + DIN;
constexpr long long OFF_B1 = OFF_W1 + (long long)HID * DIN;
constexpr long long OFF_W2 = OFF_B1 + HID;
constexpr long long OFF_B2 = OFF_W2 + (long long)HID * HID;
constexpr long long OFF_W3 = OFF_B2 + HID;
constexpr long long OFF_B3 = OFF_W3 + (long long)HID * HID;
constexpr long long OFF_W4 = OFF_B3 + HID;
constexpr long long OFF_B4 = OFF_W4 + (long long)DOUT * HID;
constexpr long long OFF_OUT_MEAN = OFF_B4 + DOUT;
constexpr long long OFF_OUT_STD = OFF_OUT_MEAN + DOUT;
constexpr long long PER_TYPE = OFF_OUT_STD + DOUT;
constexpr long long TRAIN_BEGIN = OFF_W1;
constexpr long long TRAIN_END = OFF_OUT_MEAN;
static_assert(PER_TYPE == MB_GUESS_PER_TYPE, "blob layout");

__host__ __device__ inline int nout_of(int t) {
  return t == 0 ? 10 : t == 2 ? 16 : t == 3 ? 4 : 1;
}

__device__ __forceinline__ uint16_t f2bf(float x) {
  uint32_t u = __float_as_uint(x);
  u += 0x7FFFu + ((u >> 16) & 1u);  // round to nearest even (inputs are finite)
  return (uint16_t)(u >> 16);
}
__device__ __forceinline__ float bf2f(uint16_t h) { return __uint_as_float(((uint32_t)h) << 16); }

__device__ __forceinline__ float silu_f(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float dsilu_f(float z) {
  float s = 1.0f / (1.0f + expf(-z));
  return s * (1.0f + z * (1.0f - s));
}

__device__ __forceinline__ int pair_type(int za, int zb, bool same) {
  bool ha = za != 1, hb = zb != 1;
  if (same) return ha ? 0 : 1;
  if (ha && hb) return 2;
  if (ha || hb) return 3;
  return 4;
}

__device__ __forceinline__ double r2_of(const double* c, int a, int b) {
  double dx = DSUB(c[3 * a], c[3 * b]), dy = DSUB(c[3 * a + 1], c[3 * b + 1]), dz = DSUB(c[3 * a + 2], c[3 * b + 2]);
  return DADD(DADD(DMUL(dx, dx), DMUL(dy, dy)), DMUL(dz, dz));
}

// ------------------------------------------------------------------ pairs
__global__ void pairs_count_kernel(int numat, const int* __restrict__ nat, const double* __restrict__ xyz,
                                   double rpair2, int* __restrict__ counts) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= numat) return;
  int local[NT] = {0, 0, 0, 0, 0};
  local[pair_type(nat[a], nat[a], true)]++;
  for (int b = 0; b < a; ++b)
    if (r2_of(xyz, a, b) < rpair2) local[pair_type(nat[a], nat[b], false)]++;
  for (int t = 0; t < NT; ++t)
    if (local[t]) atomicAdd(&counts[t], local[t]);
}

__global__ void pairs_emit_kernel(int numat, const int* __restrict__ nat, const double* __restrict__ xyz, double rpair2,
                                  const int* __restrict__ seg, int* __restrict__ cursor, int* __restrict__ pf,
                                  int* __restrict__ ps, int* __restrict__ pt) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= numat) return;
  {
    int t = pair_type(nat[a], nat[a], true);
    int q = seg[t] + atomicAdd(&cursor[t], 1);
    pf[q] = a; ps[q] = a; pt[q] = t;
  }
  for (int b = 0; b < a; ++b) {
    if (!(r2_of(xyz, a, b) < rpair2)) continue;
    int t = pair_type(nat[a], nat[b], false);
    int f = a, s = b;
    if (t == 3 && nat[a] == 1) { f = b; s = a; }
    int q = seg[t] + atomicAdd(&cursor[t], 1);
    pf[q] = f; ps[q] = s; pt[q] = t;
  }
}

// ---------------------------------------------------------- neighbour lists
// Atoms within RC of each atom, ascending index (the order the descriptor
// sums run in).  nbr_count[a] > NBR_MAX marks an overflow (the host refuses).
constexpr int NBR_MAX = 512;

__global__ void neighbours_kernel(int numat, const double* __restrict__ xyz, int* __restrict__ nbr_count,
                                  int* __restrict__ nbr) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= numat) return;
  int c = 0;
  for (int k = 0; k < numat; ++k) {
    if (k == a || !(r2_of(xyz, k, a) < RC * RC)) continue;
    if (c < NBR_MAX) nbr[(long long)a * NBR_MAX + c] = k;
    ++c;
  }
  nbr_count[a] = c;
}

// --------------------------------------------------- frames + descriptors
__device__ __forceinline__ unsigned long long rank_key(double r2, int k) {
  double q = floor(DADD(DMUL(r2, QSCALE), 0.5));
  if (q > 4.0e12) q = 4.0e12;  // far beyond any cutoff; keeps the key in 64 bits
  return ((unsigned long long)q << 21) | (unsigned long long)k;
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w < v ? w : v;
  }
  return v;
}

// Smallest rank key over the atoms k != f that key_of accepts (key_of returns
// ~0 for the others), over the whole molecule.  The search runs over f's
// neighbour list first: every atom off that list has r2 >= RC^2 by the same
// arithmetic (r2_of), so its key's distance part is at least that of RC^2,
// and a list minimum strictly below it is the global minimum.  Otherwise (no
// candidate on the list, a tie at the boundary, an overflowing list) the
// whole molecule is scanned.
template <class KeyOf>
__device__ __forceinline__ unsigned long long nearest_key(int lane, int numat, int f, const int* __restrict__ nbr_count,
                                                          const int* __restrict__ nbr, KeyOf key_of) {
  const unsigned long long NONE = ~0ull;
  const int nn = nbr_count[f];
  if (nn <= NBR_MAX) {
    unsigned long long best = NONE;
    const int* nl = nbr + (long long)f * NBR_MAX;
    for (int j = lane; j < nn; j += 32) {
      const unsigned long long key = key_of(nl[j]);
      best = key < best ? key : best;
    }
    best = warp_min_u64(best);
    const unsigned long long q_rc = (unsigned long long)floor(DADD(DMUL(RC * RC, QSCALE), 0.5));
    if (best != NONE && (best >> 21) < q_rc) return best;
  }
  unsigned long long best = NONE;
  for (int k = lane; k < numat; k += 32) {
    if (k == f) continue;
    const unsigned long long key = key_of(k);
    best = key < best ? key : best;
  }
  return warp_min_u64(best);
}

// Long-range moments of the reference charges seen from atom c (all k != c,
// g = x_k - x_c, r = |g|): m[0] = sum q/r, m[1..3] = sum q g/r^3, m[4] = sum
// q/r^3, m[5..10] = sum q g g^T/r^5 (xx, yy, zz, xy, xz, yz).  The frame-local
// multipoles of a pair follow from these by one rotation (features_kernel).
constexpr int NMOM = 11;
__device__ __forceinline__ void lr_contrib(const double* __restrict__ xyz, int k, int c, double q, double* m) {
  const double gx = DSUB(xyz[3 * k], xyz[3 * c]), gy = DSUB(xyz[3 * k + 1], xyz[3 * c + 1]),
               gz = DSUB(xyz[3 * k + 2], xyz[3 * c + 2]);
  const double r2 = DADD(DADD(DMUL(gx, gx), DMUL(gy, gy)), DMUL(gz, gz));
  const double r = sqrt(r2), ir = 1.0 / r, ir3 = ir / r2, ir5 = ir3 / r2;
  m[0] = q * ir;
  m[1] = q * gx * ir3; m[2] = q * gy * ir3; m[3] = q * gz * ir3;
  m[4] = q * ir3;
  m[5] = q * gx * gx * ir5; m[6] = q * gy * gy * ir5; m[7] = q * gz * gz * ir5;
  m[8] = q * gx * gy * ir5; m[9] = q * gx * gz * ir5; m[10] = q * gy * gz * ir5;
}

// One warp per atom.
__global__ void __launch_bounds__(128) lr_moments_kernel(int numat, const int* __restrict__ nat,
                                                         const double* __restrict__ xyz, double* __restrict__ mom) {
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (c >= numat) return;
  double acc[NMOM];
#pragma unroll
  for (int j = 0; j < NMOM; ++j) acc[j] = 0.0;
  for (int k = lane; k < numat; k += 32) {
    if (k == c) continue;
    double m[NMOM];
    lr_contrib(xyz, k, c, nat[k] == 1 ? QREF_H : QREF_HEAVY, m);
#pragma unroll
    for (int j = 0; j < NMOM; ++j) acc[j] += m[j];
  }
#pragma unroll
  for (int j = 0; j < NMOM; ++j)
    for (int o = 16; o > 0; o >>= 1) acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], o);
  double mine = 0.0;  // acc[lane] without a dynamically indexed (local-memory) array
#pragma unroll
  for (int j = 0; j < NMOM; ++j) mine = lane == j ? acc[j] : mine;
  if (lane < NMOM) mom[(long long)c * NMOM + lane] = mine;
}

// One warp per pair.  Writes the frame (columns x, y, z: frames[9q + 3c + r]
// = component r of axis c) and the raw descriptors feat[q * DIN + j].
__global__ void __launch_bounds__(128) features_kernel(int numat, const int* __restrict__ nat,
                                                       const double* __restrict__ xyz, int npairs,
                                                       const int* __restrict__ pf, const int* __restrict__ ps,
                                                       const int* __restrict__ nbr_count, const int* __restrict__ nbr,
                                                       const double* __restrict__ mom, float* __restrict__ feat,
                                                       double* __restrict__ frames) {
  const int lane = threadIdx.x & 31;
  const int q = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (q >= npairs) return;
  const int f = pf[q], s = ps[q];
  const double ox = xyz[3 * f], oy = xyz[3 * f + 1], oz = xyz[3 * f + 2];
  const unsigned long long NONE = ~0ull;
  int ex2 = s;
  double zx, zy, zz;
  bool have_z = true;
  if (f != s) {
    zx = DSUB(xyz[3 * s], ox); zy = DSUB(xyz[3 * s + 1], oy); zz = DSUB(xyz[3 * s + 2], oz);
  } else {
    const unsigned long long best =
        nearest_key(lane, numat, f, nbr_count, nbr, [&](int k) { return rank_key(r2_of(xyz, k, f), k); });
    if (best == NONE) {
      have_z = false;
      zx = 0.0; zy = 0.0; zz = 1.0;
      ex2 = f;
    } else {
      int k1 = (int)(best & ((1ull << 21) - 1));
      ex2 = k1;
      zx = DSUB(xyz[3 * k1], ox); zy = DSUB(xyz[3 * k1 + 1], oy); zz = DSUB(xyz[3 * k1 + 2], oz);
    }
  }
  double R[9];  // R[3c + r]
  if (!have_z) {
    R[0] = 1; R[1] = 0; R[2] = 0; R[3] = 0; R[4] = 1; R[5] = 0; R[6] = 0; R[7] = 0; R[8] = 1;
  } else {
    double zn = sqrt(DADD(DADD(DMUL(zx, zx), DMUL(zy, zy)), DMUL(zz, zz)));
    zx = zx / zn; zy = zy / zn; zz = zz / zn;
    const unsigned long long best = nearest_key(lane, numat, f, nbr_count, nbr, [&](int k) {
      if (k == ex2) return NONE;
      double dx = DSUB(xyz[3 * k], ox), dy = DSUB(xyz[3 * k + 1], oy), dz = DSUB(xyz[3 * k + 2], oz);
      double r2 = DADD(DADD(DMUL(dx, dx), DMUL(dy, dy)), DMUL(dz, dz));
      double dd = DADD(DADD(DMUL(dx, zx), DMUL(dy, zy)), DMUL(dz, zz));
      double p2 = DSUB(r2, DMUL(dd, dd));
      if (!(p2 > DMUL(PERP_MIN2, r2))) return NONE;
      return rank_key(r2, k);
    });
    double px, py, pz;
    if (best == NONE) {
      double ax = fabs(zx), ay = fabs(zy), az = fabs(zz);
      double ex = 0, ey = 0, ez = 0;
      if (ax <= ay && ax <= az) ex = 1; else if (ay <= az) ey = 1; else ez = 1;
      double dd = DADD(DADD(DMUL(ex, zx), DMUL(ey, zy)), DMUL(ez, zz));
      px = DSUB(ex, DMUL(dd, zx)); py = DSUB(ey, DMUL(dd, zy)); pz = DSUB(ez, DMUL(dd, zz));
    } else {
      int k = (int)(best & ((1ull << 21) - 1));
      double dx = DSUB(xyz[3 * k], ox), dy = DSUB(xyz[3 * k + 1], oy), dz = DSUB(xyz[3 * k + 2], oz);
      double dd = DADD(DADD(DMUL(dx, zx), DMUL(dy, zy)), DMUL(dz, zz));
      px = DSUB(dx, DMUL(dd, zx)); py = DSUB(dy, DMUL(dd, zy)); pz = DSUB(dz, DMUL(dd, zz));
    }
    double pn = sqrt(DADD(DADD(DMUL(px, px), DMUL(py, py)), DMUL(pz, pz)));
    double xx = px / pn, xy = py / pn, xz = pz / pn;
    R[0] = xx; R[1] = xy; R[2] = xz;
    R[3] = DSUB(DMUL(zy, xz), DMUL(zz, xy));
    R[4] = DSUB(DMUL(zz, xx), DMUL(zx, xz));
    R[5] = DSUB(DMUL(zx, xy), DMUL(zy, xx));
    R[6] = zx; R[7] = zy; R[8] = zz;
  }
  if (lane < 9) frames[9ll * q + lane] = R[lane];

  // descriptors: lane -> (element class e, shell m, angular half)
  const int e = (lane & 15) >> 3, m = lane & 7, half = lane >> 4;
  const double mu = 0.8 + (RC - 0.8) * m / (NRAD - 1);
  float* out = feat + (long long)q * DIN;
  const int ncent = f == s ? 1 : 2;
  for (int ci = 0; ci < ncent; ++ci) {
    const int c = ci == 0 ? f : s;
    const double cx = xyz[3 * c], cy = xyz[3 * c + 1], cz = xyz[3 * c + 2];
    double acc[5] = {0, 0, 0, 0, 0};
    const int nn = min(nbr_count[c], NBR_MAX);  // an overflow is reported by the host after the launch
    const int* nl = nbr + (long long)c * NBR_MAX;
    for (int j = 0; j < nn; ++j) {
      const int k = nl[j];
      if (k == f || k == s) continue;
      if ((nat[k] != 1) != (e == 1)) continue;
      double dx = DSUB(xyz[3 * k], cx), dy = DSUB(xyz[3 * k + 1], cy), dz = DSUB(xyz[3 * k + 2], cz);
      double r2 = DADD(DADD(DMUL(dx, dx), DMUL(dy, dy)), DMUL(dz, dz));
      if (!(r2 < RC * RC)) continue;
      double r = sqrt(r2);
      double lx = DADD(DADD(DMUL(dx, R[0]), DMUL(dy, R[1])), DMUL(dz, R[2])) / r;
      double ly = DADD(DADD(DMUL(dx, R[3]), DMUL(dy, R[4])), DMUL(dz, R[5])) / r;
      double lz = DADD(DADD(DMUL(dx, R[6]), DMUL(dy, R[7])), DMUL(dz, R[8])) / r;
      double fc = 0.5 * (cos(M_PI * r / RC) + 1.0);
      double t = r - mu;
      double g = exp(-(t * t) / (2.0 * RAD_SIG * RAD_SIG)) * fc;
      if (half == 0) {
        acc[0] += g; acc[1] += g * lx; acc[2] += g * ly; acc[3] += g * lz; acc[4] += g * (lx * lx);
      } else {
        acc[0] += g * (ly * ly); acc[1] += g * (lz * lz); acc[2] += g * (lx * ly); acc[3] += g * (lx * lz);
        acc[4] += g * (ly * lz);
      }
    }
    float* o = out + ci * PER_CENTER + e * (NRAD * NANG) + m * NANG + half * 5;
    for (int j = 0; j < 5; ++j) o[j] = (float)acc[j];
  }
  if (ncent == 1)
    for (int j = lane; j < PER_CENTER; j += 32) out[PER_CENTER + j] = 0.f;
  // long-range electrostatic environment of each centre: the centre's
  // moments over all other atoms less the pair partner's share, rotated into
  // the pair frame (x = a_x . g, so sum q x/r^3 = a_x . m[1..3] and sum q (3 x
  // x' - r^2 d)/r^5 = 3 a^T M a' - d m[4])
  for (int ci = 0; ci < 2; ++ci) {
    if (ci == 1 && ncent == 1) {
      if (lane < NLR) out[LR0 + NLR + lane] = 0.f;
      continue;
    }
    const int c = ci == 0 ? f : s, o = ci == 0 ? s : f;
    double m[NMOM];
    for (int j = 0; j < NMOM; ++j) m[j] = mom[(long long)c * NMOM + j];
    if (ncent == 2) {
      double mo[NMOM];
      lr_contrib(xyz, o, c, nat[o] == 1 ? QREF_H : QREF_HEAVY, mo);
      for (int j = 0; j < NMOM; ++j) m[j] -= mo[j];
    }
    // M a for the three axes a = R[0..2], R[3..5], R[6..8]
    double Ma[9];
    for (int a = 0; a < 3; ++a) {
      const double ax = R[3 * a], ay = R[3 * a + 1], az = R[3 * a + 2];
      Ma[3 * a] = m[5] * ax + m[8] * ay + m[9] * az;
      Ma[3 * a + 1] = m[8] * ax + m[6] * ay + m[10] * az;
      Ma[3 * a + 2] = m[9] * ax + m[10] * ay + m[7] * az;
    }
    auto aMb = [&](int a, int b) { return R[3 * a] * Ma[3 * b] + R[3 * a + 1] * Ma[3 * b + 1] + R[3 * a + 2] * Ma[3 * b + 2]; };
    if (lane == 0) {
      float* lr = out + LR0 + ci * NLR;
      lr[0] = (float)m[0];
      for (int a = 0; a < 3; ++a) lr[1 + a] = (float)(R[3 * a] * m[1] + R[3 * a + 1] * m[2] + R[3 * a + 2] * m[3]);
      for (int a = 0; a < 3; ++a) lr[4 + a] = (float)(3.0 * aMb(a, a) - m[4]);
      lr[7] = (float)(3.0 * aMb(0, 1));
      lr[8] = (float)(3.0 * aMb(0, 2));
      lr[9] = (float)(3.0 * aMb(1, 2));
    }
  }
  if (lane < NPAIR_RBF) {
    float v = 0.f;
    if (f != s) {
      double r = sqrt(r2_of(xyz, f, s));
      double mu2 = 0.8 + (6.0 - 0.8) * lane / (NPAIR_RBF - 1);
      double t = r - mu2;
      v = (float)exp(-(t * t) / (2.0 * PAIR_SIG * PAIR_SIG));
    }
    out[2 * PER_CENTER + lane] = v;
  }
}

__global__ void normalize_kernel(int n, const float* __restrict__ raw, const float* __restrict__ mean,
                                 const float* __restrict__ stdv, uint16_t* __restrict__ x) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)n * DIN) return;
  int j = (int)(i % DIN);
  x[i] = f2bf((raw[i] - mean[j]) / stdv[j]);
}

__global__ void norm_targets_kernel(int n, const float* __restrict__ raw, const float* __restrict__ mean,
                                    const float* __restrict__ stdv, int nout, float* __restrict__ yt) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)n * DOUT) return;
  int j = (int)(i % DOUT);
  yt[i] = j < nout ? (raw[i] - mean[j]) / stdv[j] : 0.f;
}

// ------------------------------------------------------- BF16 tensor GEMM
// C(M x N) = sum_k A(m, k) B(k, n); A(m, k) = a[m*sam + k*sak], B(k, n) =
// b[k*sbk + n*sbn]; BF16 operands, FP32 accumulation on mma.sync.m16n8k16.
enum { EPI_HIDDEN = 0, EPI_OUT = 1, EPI_F32 = 2, EPI_DSILU = 3 };

struct GemmArgs {
  int M, N, K;
  const uint16_t* a;
  long long sam, sak;
  const uint16_t* b;
  long long sbk, sbn;
  const float* bias;   // EPI_HIDDEN, EPI_OUT
  const float* zin;    // EPI_DSILU: pre-activations (ldz)
  float* zout;         // EPI_HIDDEN: pre-activations out (may be null)
  long long ldz;
  float* outf;         // EPI_OUT, EPI_F32
  uint16_t* outh;      // EPI_HIDDEN, EPI_DSILU
  long long ldo;
};

constexpr int BM = 64, BN = 64, BK = 32, PAD = 8;

__device__ __forceinline__ void mma_bf16(float* d, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

template <int EPI>
__global__ void __launch_bounds__(128) mlp_gemm_kernel(GemmArgs g) {
  __shared__ __align__(16) uint16_t As[BM][BK + PAD];
  __shared__ __align__(16) uint16_t Bs[BN][BK + PAD];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int gq = lane >> 2, tq = lane & 3;
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.f;

  for (int k0 = 0; k0 < g.K; k0 += BK) {
    // A tile: As[m][k]
    if (g.sak == 1) {
      const int kk = tid & 31;
      for (int r = tid >> 5; r < BM; r += 4) {
        int m = m0 + r, k = k0 + kk;
        As[r][kk] = (m < g.M && k < g.K) ? g.a[(long long)m * g.sam + k] : (uint16_t)0;
      }
    } else {
      const int r = tid & 63;
      for (int kk = tid >> 6; kk < BK; kk += 2) {
        int m = m0 + r, k = k0 + kk;
        As[r][kk] = (m < g.M && k < g.K) ? g.a[(long long)m * g.sam + (long long)k * g.sak] : (uint16_t)0;
      }
    }
    // B tile: Bs[n][k]
    if (g.sbk == 1) {
      const int kk = tid & 31;
      for (int r = tid >> 5; r < BN; r += 4) {
        int n = n0 + r, k = k0 + kk;
        Bs[r][kk] = (n < g.N && k < g.K) ? g.b[(long long)n * g.sbn + k] : (uint16_t)0;
      }
    } else {
      const int r = tid & 63;
      for (int kk = tid >> 6; kk < BK; kk += 2) {
        int n = n0 + r, k = k0 + kk;
        Bs[r][kk] = (n < g.N && k < g.K) ? g.b[(long long)k * g.sbk + (long long)n * g.sbn] : (uint16_t)0;
      }
    }
    __syncthreads();
#pragma unroll
    for (int ks = 0; ks < BK; ks += 16) {
      uint32_t af[2][4], bfr[4][2];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int r = wm + i * 16 + gq;
        af[i][0] = *reinterpret_cast<const uint32_t*>(&As[r][ks + 2 * tq]);
        af[i][1] = *reinterpret_cast<const uint32_t*>(&As[r + 8][ks + 2 * tq]);
        af[i][2] = *reinterpret_cast<const uint32_t*>(&As[r][ks + 2 * tq + 8]);
        af[i][3] = *reinterpret_cast<const uint32_t*>(&As[r + 8][ks + 2 * tq + 8]);
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = wn + j * 8 + gq;
        bfr[j][0] = *reinterpret_cast<const uint32_t*>(&Bs[c][ks + 2 * tq]);
        bfr[j][1] = *reinterpret_cast<const uint32_t*>(&Bs[c][ks + 2 * tq + 8]);
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i][0], af[i][1], af[i][2], af[i][3], bfr[j][0], bfr[j][1]);
    }
    __syncthreads();
  }
  // epilogue
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int m = m0 + wm + i * 16 + gq + (r >> 1) * 8;
        const int n = n0 + wn + j * 8 + 2 * tq + (r & 1);
        if (m >= g.M || n >= g.N) continue;
        float v = acc[i][j][r];
        if (EPI == EPI_HIDDEN) {
          float z = v + g.bias[n];
          if (g.zout) g.zout[(long long)m * g.ldz + n] = z;
          g.outh[(long long)m * g.ldo + n] = f2bf(silu_f(z));
        } else if (EPI == EPI_OUT) {
          g.outf[(long long)m * g.ldo + n] = v + g.bias[n];
        } else if (EPI == EPI_F32) {
          g.outf[(long long)m * g.ldo + n] = v;
        } else {
          g.outh[(long long)m * g.ldo + n] = f2bf(v * dsilu_f(g.zin[(long long)m * g.ldz + n]));
        }
      }
}

template <int EPI>
int launch_gemm(const GemmArgs& g, cudaStream_t s) {
  if (g.M <= 0 || g.N <= 0) return MB_OK;
  dim3 grid((g.N + BN - 1) / BN, (g.M + BM - 1) / BM);
  mlp_gemm_kernel<EPI><<<grid, 128, 0, s>>>(g);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

// ------------------------------------------------------ assembly, targets
__device__ __forceinline__ void umat(int nor, const double* R, double U[4][4]) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) U[i][j] = 0.0;
  U[0][0] = 1.0;
  if (nor == 4)
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) U[1 + r][1 + c] = R[3 * c + r];  // column c = axis c
}

__constant__ int c_tri4[10][2] = {{0, 0}, {1, 0}, {1, 1}, {2, 0}, {2, 1}, {2, 2}, {3, 0}, {3, 1}, {3, 2}, {3, 3}};

__global__ void assemble_kernel(int npairs, const int* __restrict__ pf, const int* __restrict__ ps,
                                const int* __restrict__ pt, const double* __restrict__ frames,
                                const float* __restrict__ y, const float* __restrict__ params,
                                const int* __restrict__ first, const int* __restrict__ nor,
                                double* __restrict__ p) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npairs) return;
  const int f = pf[q], s = ps[q], t = pt[q];
  const float* pm = params + (long long)t * PER_TYPE;
  const float* yq = y + (long long)q * DOUT;
  double L[4][4];
  const int nr = nor[f], nc = nor[s];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) L[i][j] = 0.0;
  if (t == 0) {
    for (int k = 0; k < 10; ++k) {
      double v = (double)yq[k] * (double)pm[OFF_OUT_STD + k] + (double)pm[OFF_OUT_MEAN + k];
      L[c_tri4[k][0]][c_tri4[k][1]] = v;
      L[c_tri4[k][1]][c_tri4[k][0]] = v;
    }
  } else {
    for (int i = 0; i < nr; ++i)
      for (int j = 0; j < nc; ++j) {
        int k = i * nc + j;
        L[i][j] = (double)yq[k] * (double)pm[OFF_OUT_STD + k] + (double)pm[OFF_OUT_MEAN + k];
      }
  }
  double R[9];
  for (int k = 0; k < 9; ++k) R[k] = frames[9ll * q + k];
  double Uf[4][4], Us[4][4];
  umat(nr, R, Uf);
  umat(nc, R, Us);
  // B = Uf L Us^T
  double T[4][4], B[4][4];
  for (int i = 0; i < nr; ++i)
    for (int j = 0; j < nc; ++j) {
      double v = 0.0;
      for (int k = 0; k < nr; ++k) v += Uf[i][k] * L[k][j];
      T[i][j] = v;
    }
  for (int i = 0; i < nr; ++i)
    for (int j = 0; j < nc; ++j) {
      double v = 0.0;
      for (int k = 0; k < nc; ++k) v += T[i][k] * Us[j][k];
      B[i][j] = v;
    }
  const int fo = first[f], so = first[s];
  if (f == s) {
    for (int i = 0; i < nr; ++i)
      for (int j = 0; j <= i; ++j) p[mb_tri(fo + i, fo + j)] = B[i][j];
  } else if (fo > so) {
    for (int i = 0; i < nr; ++i)
      for (int j = 0; j < nc; ++j) p[mb_tri(fo + i, so + j)] = B[i][j];
  } else {
    for (int i = 0; i < nr; ++i)
      for (int j = 0; j < nc; ++j) p[mb_tri(so + j, fo + i)] = B[i][j];
  }
}

__global__ void targets_kernel(int npairs, const int* __restrict__ pf, const int* __restrict__ ps,
                               const int* __restrict__ pt, const double* __restrict__ frames,
                               const int* __restrict__ first, const int* __restrict__ nor,
                               const double* __restrict__ p, float* __restrict__ yraw) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npairs) return;
  const int f = pf[q], s = ps[q], t = pt[q];
  const int nr = nor[f], nc = nor[s], fo = first[f], so = first[s];
  double B[4][4];
  for (int i = 0; i < nr; ++i)
    for (int j = 0; j < nc; ++j) {
      int r = fo + i, c = so + j;
      B[i][j] = r >= c ? p[mb_tri(r, c)] : p[mb_tri(c, r)];
    }
  double R[9];
  for (int k = 0; k < 9; ++k) R[k] = frames[9ll * q + k];
  double Uf[4][4], Us[4][4];
  umat(nr, R, Uf);
  umat(nc, R, Us);
  // L = Uf^T B Us
  double T[4][4], L[4][4];
  for (int i = 0; i < nr; ++i)
    for (int j = 0; j < nc; ++j) {
      double v = 0.0;
      for (int k = 0; k < nr; ++k) v += Uf[k][i] * B[k][j];
      T[i][j] = v;
    }
  for (int i = 0; i < nr; ++i)
    for (int j = 0; j < nc; ++j) {
      double v = 0.0;
      for (int k = 0; k < nc; ++k) v += T[i][k] * Us[k][j];
      L[i][j] = v;
    }
  float* o = yraw + (long long)q * DOUT;
  for (int k = 0; k < DOUT; ++k) o[k] = 0.f;
  if (t == 0) {
    for (int k = 0; k < 10; ++k) o[k] = (float)L[c_tri4[k][0]][c_tri4[k][1]];
  } else {
    for (int i = 0; i < nr; ++i)
      for (int j = 0; j < nc; ++j) o[i * nc + j] = (float)L[i][j];
  }
}

// ----------------------------------------------------------------- training
__global__ void lossgrad_kernel(int n, int nout, const float* __restrict__ y, const float* __restrict__ yt,
                                uint16_t* __restrict__ dz, double* __restrict__ loss) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double l = 0.0;
  if (i < (long long)n * DOUT) {
    int j = (int)(i % DOUT);
    float r = j < nout ? y[i] - yt[i] : 0.f;
    l = (double)r * (double)r;
    dz[i] = f2bf(r * (2.0f / ((float)n * (float)nout)));
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0 && l != 0.0) atomicAdd(loss, l);
}

// db[j] = sum over rows of dz[row * ld + j]
__global__ void colsum_kernel(int rows, int cols, const uint16_t* __restrict__ dz, float* __restrict__ db) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cols) return;
  float s = 0.f;
  for (int r = 0; r < rows; ++r) s += bf2f(dz[(long long)r * cols + j]);
  db[j] = s;
}

__global__ void adam_kernel(long long n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, uint16_t* __restrict__ pbf, float lr, float b1, float b2, float c1,
                            float c2, float eps) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float gi = g[i];
  float mi = b1 * m[i] + (1.f - b1) * gi;
  float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  float w = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  p[i] = w;
  pbf[i] = f2bf(w);
}

__global__ void to_bf16_kernel(long long n, const float* __restrict__ p, uint16_t* __restrict__ pbf) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) pbf[i] = f2bf(p[i]);
}

int blocks_for(long long n, int tpb) { return (int)((n + tpb - 1) / tpb); }

}  // namespace

// ======================================================================
//                                   models
// ======================================================================
struct mb_guess_model {
  float* params = nullptr;  // NT * PER_TYPE floats
  uint16_t* wbf = nullptr;  // BF16 mirror of params
  bool owns = true;
};

extern "C" size_t mb_guess_blob_floats(void) { return (size_t)NT * PER_TYPE; }

extern "C" int mb_guess_model_create(const float* blob, mb_guess_model** out) {
  if (!blob || !out) return mb_set_error(MB_ERR_ARG, "mb_guess_model_create: bad args");
  *out = nullptr;
  const size_t nf = (size_t)NT * PER_TYPE;
  mb_guess_model* m = new mb_guess_model();
  cudaError_t e = cudaMalloc(&m->params, nf * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&m->wbf, nf * sizeof(uint16_t));
  if (e == cudaSuccess) e = cudaMemcpy(m->params, blob, nf * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(m->params);
    cudaFree(m->wbf);
    delete m;
    return mb_set_cuda_error(e, "mb_guess_model_create", __FILE__, __LINE__);
  }
  to_bf16_kernel<<<blocks_for((long long)nf, 256), 256>>>((long long)nf, m->params, m->wbf);
  MB_LAUNCH_CHECK();
  MB_CUDA(cudaDeviceSynchronize());
  *out = m;
  return MB_OK;
}

extern "C" int mb_guess_model_destroy(mb_guess_model* m) {
  if (!m) return MB_OK;
  if (m->owns) {
    cudaFree(m->params);
    cudaFree(m->wbf);
  }
  delete m;
  return MB_OK;
}

extern "C" int mb_guess_pairs_dev(int numat, const int* nat, const double* xyz, double rpair, int* counts_host,
                                  int max_pairs, int* pf, int* ps, int* pt, int* work, cudaStream_t s) {
  if (numat <= 0 || numat >= (1 << 21) || !nat || !xyz || !counts_host || !work)
    return mb_set_error(MB_ERR_ARG, "mb_guess_pairs_dev: bad args");
  const double r2 = rpair * rpair;
  int* counts = work;
  int* seg = work + NT;
  int* cursor = work + 2 * NT;
  MB_CUDA(cudaMemsetAsync(work, 0, sizeof(int) * 3 * NT, s));
  pairs_count_kernel<<<blocks_for(numat, 128), 128, 0, s>>>(numat, nat, xyz, r2, counts);
  MB_LAUNCH_CHECK();
  MB_CUDA(cudaMemcpyAsync(counts_host, counts, sizeof(int) * NT, cudaMemcpyDeviceToHost, s));
  MB_CUDA(cudaStreamSynchronize(s));
  long long tot = 0;
  int segh[NT];
  for (int t = 0; t < NT; ++t) {
    segh[t] = (int)tot;
    tot += counts_host[t];
  }
  if (!pf) return MB_OK;  // count only
  if (tot > max_pairs) return mb_set_error(MB_ERR_ARG, "mb_guess_pairs_dev: pair buffer too small");
  MB_CUDA(cudaMemcpyAsync(seg, segh, sizeof(int) * NT, cudaMemcpyHostToDevice, s));
  pairs_emit_kernel<<<blocks_for(numat, 128), 128, 0, s>>>(numat, nat, xyz, r2, seg, cursor, pf, ps, pt);
  MB_LAUNCH_CHECK();
  MB_CUDA(cudaStreamSynchronize(s));  // segh lives on this stack frame
  return MB_OK;
}

static size_t nbr_bytes(int numat) { return ((sizeof(int) * (size_t)numat * (NBR_MAX + 1)) + 255) & ~(size_t)255; }

// fws: mb_guess_features_ws_bytes(numat) bytes, 256-byte aligned: the
// neighbour counts and lists, then the atoms' long-range moments.
static int features_impl(int numat, const int* nat, const double* xyz, int npairs, const int* pf, const int* ps,
                         float* feat, double* frames, void* fws, cudaStream_t s) {
  int* nbr_count = (int*)fws;
  int* nbr = nbr_count + numat;
  double* mom = (double*)((char*)fws + nbr_bytes(numat));
  neighbours_kernel<<<blocks_for(numat, 128), 128, 0, s>>>(numat, xyz, nbr_count, nbr);
  MB_LAUNCH_CHECK();
  lr_moments_kernel<<<blocks_for(numat, 4), 128, 0, s>>>(numat, nat, xyz, mom);
  MB_LAUNCH_CHECK();
  features_kernel<<<blocks_for(npairs, 4), 128, 0, s>>>(numat, nat, xyz, npairs, pf, ps, nbr_count, nbr, mom, feat,
                                                        frames);
  MB_LAUNCH_CHECK();
  // an overflowing neighbour list is an error, not a silent truncation
  int mx = 0;
  std::vector<int> cnt(numat);
  MB_CUDA(cudaMemcpyAsync(cnt.data(), nbr_count, sizeof(int) * numat, cudaMemcpyDeviceToHost, s));
  MB_CUDA(cudaStreamSynchronize(s));
  for (int a = 0; a < numat; ++a) mx = cnt[a] > mx ? cnt[a] : mx;
  if (mx > NBR_MAX) return mb_set_error(MB_ERR_UNSUPPORTED, "learned guess: more than 512 atoms within 6 A of an atom");
  return MB_OK;
}

extern "C" size_t mb_guess_features_ws_bytes(int numat) {
  return nbr_bytes(numat) + sizeof(double) * NMOM * (size_t)numat;
}

// ws: mb_guess_features_ws_bytes(numat) bytes of device scratch, 256-byte
// aligned (neighbour lists and long-range moments).
extern "C" int mb_guess_features_dev(int numat, const int* nat, const double* xyz, int npairs, const int* pf,
                                     const int* ps, float* feat, double* frames, void* ws, cudaStream_t s) {
  if (npairs < 0 || numat <= 0 || numat >= (1 << 21) || !ws)
    return mb_set_error(MB_ERR_ARG, "mb_guess_features_dev: bad args");
  if (npairs == 0) return MB_OK;
  if (((uintptr_t)ws & 255) != 0) return mb_set_error(MB_ERR_ARG, "mb_guess_features_dev: ws must be 256-byte aligned");
  return features_impl(numat, nat, xyz, npairs, pf, ps, feat, frames, ws, s);
}

extern "C" int mb_guess_normalize_dev(const mb_guess_model* m, int type, int n, const float* raw, uint16_t* x,
                                      cudaStream_t s) {
  if (!m || type < 0 || type >= NT || n < 0) return mb_set_error(MB_ERR_ARG, "mb_guess_normalize_dev: bad args");
  if (n == 0) return MB_OK;
  const float* pm = m->params + (long long)type * PER_TYPE;
  normalize_kernel<<<blocks_for((long long)n * DIN, 256), 256, 0, s>>>(n, raw, pm + OFF_IN_MEAN, pm + OFF_IN_STD, x);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

extern "C" int mb_guess_norm_targets_dev(const mb_guess_model* m, int type, int n, const float* yraw, float* yt,
                                         cudaStream_t s) {
  if (!m || type < 0 || type >= NT || n < 0) return mb_set_error(MB_ERR_ARG, "mb_guess_norm_targets_dev: bad args");
  if (n == 0) return MB_OK;
  const float* pm = m->params + (long long)type * PER_TYPE;
  norm_targets_kernel<<<blocks_for((long long)n * DOUT, 256), 256, 0, s>>>(n, yraw, pm + OFF_OUT_MEAN,
                                                                           pm + OFF_OUT_STD, nout_of(type), yt);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

// Forward pass of one type's network on n normalised rows.  ws: 2 * n * HID
// BF16 values; zs (optional): 3 * n * HID floats of pre-activations (z1, z2,
// z3), kept for the backward pass; acts (optional): if given, the three hidden
// activations are written there (3 * n * HID BF16) instead of ws.
static int forward_impl(const float* params, const uint16_t* wbf, int type, int n, const uint16_t* x, float* y,
                        uint16_t* ws, float* zs, uint16_t* acts, cudaStream_t s) {
  const long long base = (long long)type * PER_TYPE;
  const uint16_t* W[4] = {wbf + base + OFF_W1, wbf + base + OFF_W2, wbf + base + OFF_W3, wbf + base + OFF_W4};
  const float* b[4] = {params + base + OFF_B1, params + base + OFF_B2, params + base + OFF_B3, params + base + OFF_B4};
  const uint16_t* in = x;
  int kin = DIN;
  for (int l = 0; l < 3; ++l) {
    uint16_t* out = acts ? acts + (long long)l * n * HID : ws + (long long)(l & 1) * n * HID;
    GemmArgs g{};
    g.M = n; g.N = HID; g.K = kin;
    g.a = in; g.sam = kin; g.sak = 1;
    g.b = W[l]; g.sbk = 1; g.sbn = kin;
    g.bias = b[l];
    g.zout = zs ? zs + (long long)l * n * HID : nullptr;
    g.ldz = HID;
    g.outh = out; g.ldo = HID;
    MB_TRY(launch_gemm<EPI_HIDDEN>(g, s));
    in = out;
    kin = HID;
  }
  GemmArgs g{};
  g.M = n; g.N = DOUT; g.K = HID;
  g.a = in; g.sam = HID; g.sak = 1;
  g.b = W[3]; g.sbk = 1; g.sbn = HID;
  g.bias = b[3];
  g.outf = y; g.ldo = DOUT;
  return launch_gemm<EPI_OUT>(g, s);
}

extern "C" int mb_guess_forward_dev(const mb_guess_model* m, int type, int n, const uint16_t* x, float* y, void* ws,
                                    cudaStream_t s) {
  if (!m || type < 0 || type >= NT || n < 0 || (n > 0 && (!x || !y || !ws)))
    return mb_set_error(MB_ERR_ARG, "mb_guess_forward_dev: bad args");
  if (n == 0) return MB_OK;
  return forward_impl(m->params, m->wbf, type, n, x, y, (uint16_t*)ws, nullptr, nullptr, s);
}

extern "C" int mb_guess_assemble_dev(const mb_guess_model* m, int npairs, const int* pf, const int* ps, const int* pt,
                                     const double* frames, const float* y, const int* first, const int* nor,
                                     double* p, cudaStream_t s) {
  if (!m || npairs < 0) return mb_set_error(MB_ERR_ARG, "mb_guess_assemble_dev: bad args");
  if (npairs == 0) return MB_OK;
  assemble_kernel<<<blocks_for(npairs, 128), 128, 0, s>>>(npairs, pf, ps, pt, frames, y, m->params, first, nor, p);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

extern "C" int mb_guess_targets_dev(int npairs, const int* pf, const int* ps, const int* pt, const double* frames,
                                    const int* first, const int* nor, const double* p, float* yraw, cudaStream_t s) {
  if (npairs < 0) return mb_set_error(MB_ERR_ARG, "mb_guess_targets_dev: bad args");
  if (npairs == 0) return MB_OK;
  targets_kernel<<<blocks_for(npairs, 128), 128, 0, s>>>(npairs, pf, ps, pt, frames, first, nor, p, yraw);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

// Grow-only device workspace of the prediction (a context keeps one, so a
// prediction allocates only when a molecule needs more room than any before).
struct mb_guess_ws {
  char* buf = nullptr;
  size_t bytes = 0;
};

static int ws_ensure(mb_guess_ws* w, size_t bytes) {
  if (bytes <= w->bytes) return MB_OK;
  if (w->buf) MB_CUDA(cudaFree(w->buf));
  w->buf = nullptr;
  w->bytes = 0;
  MB_CUDA(cudaMalloc((void**)&w->buf, bytes));
  w->bytes = bytes;
  return MB_OK;
}

extern "C" int mb_guess_ws_create(mb_guess_ws** out) {
  if (!out) return mb_set_error(MB_ERR_ARG, "mb_guess_ws_create: null");
  *out = new mb_guess_ws();
  return MB_OK;
}

extern "C" int mb_guess_ws_destroy(mb_guess_ws* w) {
  if (w) {
    if (w->buf) cudaFree(w->buf);
    delete w;
  }
  return MB_OK;
}

// Whole prediction for one molecule into a packed density p (device, mpack
// doubles, overwritten: pairs beyond 6 A are zero).  Two host synchronisations
// (pair counts, neighbour-list check); buffers from the grow-only workspace.
extern "C" int mb_guess_predict_density_ws(const mb_guess_model* m, int numat, const int* nat, const double* xyz,
                                           const int* first, const int* nor, int norbs, double* p, mb_guess_ws* w,
                                           cudaStream_t s) {
  if (!m || !w || numat <= 0 || numat >= (1 << 21) || norbs <= 0 || !p)
    return mb_set_error(MB_ERR_ARG, "mb_guess_predict_density_ws: bad args");
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  const double r2 = 36.0;
  MB_TRY(ws_ensure(w, 256));
  int* work = (int*)w->buf;
  int counts[NT];
  MB_CUDA(cudaMemsetAsync(work, 0, sizeof(int) * 3 * NT, s));
  pairs_count_kernel<<<blocks_for(numat, 128), 128, 0, s>>>(numat, nat, xyz, r2, work);
  MB_LAUNCH_CHECK();
  MB_CUDA(cudaMemcpyAsync(counts, work, sizeof(int) * NT, cudaMemcpyDeviceToHost, s));
  MB_CUDA(cudaStreamSynchronize(s));
  long long tot = 0;
  int maxc = 0, segh[NT];
  for (int t = 0; t < NT; ++t) {
    segh[t] = (int)tot;
    tot += counts[t];
    maxc = counts[t] > maxc ? counts[t] : maxc;
  }
  const size_t b_work = 256;
  const size_t b_pairs = sizeof(int) * 3 * (size_t)tot;
  const size_t b_frames = sizeof(double) * 9 * (size_t)tot;
  const size_t b_feat = sizeof(float) * DIN * (size_t)tot;
  const size_t b_y = sizeof(float) * DOUT * (size_t)tot;
  const size_t b_x = sizeof(uint16_t) * DIN * (size_t)maxc;
  const size_t b_ws = sizeof(uint16_t) * 2 * HID * (size_t)maxc;
  const size_t b_nbr = mb_guess_features_ws_bytes(numat);
  MB_TRY(ws_ensure(w, b_work + al(b_pairs) + al(b_frames) + al(b_feat) + al(b_y) + al(b_x) + al(b_ws) + al(b_nbr)));
  char* cur = w->buf;
  work = (int*)cur; cur += b_work;
  int* pf = (int*)cur;
  int* ps = pf + tot;
  int* pt = ps + tot;
  cur += al(b_pairs);
  double* frames = (double*)cur; cur += al(b_frames);
  float* feat = (float*)cur; cur += al(b_feat);
  float* y = (float*)cur; cur += al(b_y);
  uint16_t* x = (uint16_t*)cur; cur += al(b_x);
  uint16_t* mlp_ws = (uint16_t*)cur; cur += al(b_ws);
  void* fws = cur;
  // emit the pairs type by type
  MB_CUDA(cudaMemcpyAsync(work + NT, segh, sizeof(int) * NT, cudaMemcpyHostToDevice, s));
  MB_CUDA(cudaMemsetAsync(work + 2 * NT, 0, sizeof(int) * NT, s));
  pairs_emit_kernel<<<blocks_for(numat, 128), 128, 0, s>>>(numat, nat, xyz, r2, work + NT, work + 2 * NT, pf, ps, pt);
  MB_LAUNCH_CHECK();
  MB_TRY(features_impl(numat, nat, xyz, (int)tot, pf, ps, feat, frames, fws, s));  // syncs: segh is safe
  long long off = 0;
  for (int t = 0; t < NT; ++t) {
    if (counts[t] == 0) continue;
    MB_TRY(mb_guess_normalize_dev(m, t, counts[t], feat + off * DIN, x, s));
    MB_TRY(forward_impl(m->params, m->wbf, t, counts[t], x, y + off * DOUT, mlp_ws, nullptr, nullptr, s));
    off += counts[t];
  }
  MB_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * (size_t)norbs * (norbs + 1) / 2, s));
  return mb_guess_assemble_dev(m, (int)tot, pf, ps, pt, frames, y, first, nor, p, s);
}

// The same with a workspace of its own (allocated and freed in the call).
extern "C" int mb_guess_predict_density_dev(const mb_guess_model* m, int numat, const int* nat, const double* xyz,
                                            const int* first, const int* nor, int norbs, double* p,
                                            cudaStream_t s) {
  mb_guess_ws w;
  int rc = mb_guess_predict_density_ws(m, numat, nat, xyz, first, nor, norbs, p, &w, s);
  cudaError_t e = cudaStreamSynchronize(s);
  if (w.buf) cudaFree(w.buf);
  if (rc == MB_OK && e != cudaSuccess) rc = mb_set_cuda_error(e, "mb_guess_predict_density_dev", __FILE__, __LINE__);
  return rc;
}

// ------------------------------------------------------------ purification
// McWeeny purification of a predicted total density P: D = P/2 is replaced
// by 3 D^2 - 2 D^3 (steps times), which pulls D's eigenvalues towards 0 and 1
// -- a closed-shell density matrix -- with FP64 GEMMs.
namespace {
__global__ void unpack_half_kernel(int n, const double* __restrict__ pk, double* __restrict__ d) {
  long long nn = (long long)n * n;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nn; q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % n), j = (int)(q / n);
    int r = i > j ? i : j, c = i > j ? j : i;
    d[q] = pk[mb_tri(r, c)] * 0.5;
  }
}
__global__ void mcweeny_kernel(long long nn, const double* __restrict__ d2, const double* __restrict__ d3,
                               double* __restrict__ d) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nn; q += (long long)gridDim.x * blockDim.x)
    d[q] = 3.0 * d2[q] - 2.0 * d3[q];
}
__global__ void pack_twice_kernel(int n, const double* __restrict__ d, double* __restrict__ pk) {
  long long mp = (long long)n * (n + 1) / 2;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < mp; q += (long long)gridDim.x * blockDim.x) {
    int r = (int)((sqrt(8.0 * (double)q + 1.0) - 1.0) * 0.5);
    while ((long long)r * (r + 1) / 2 > q) --r;
    while ((long long)(r + 1) * (r + 2) / 2 <= q) ++r;
    int c = (int)(q - (long long)r * (r + 1) / 2);
    pk[q] = d[r + (long long)c * n] + d[c + (long long)r * n];  // 2 * the symmetric part
  }
}
}  // namespace

extern "C" int mb_dgemm_dev(char transa, char transb, int m, int n, int k, double alpha, const double* a, int lda,
                            const double* b, int ldb, double beta, double* c, int ldc, cudaStream_t stream);

extern "C" size_t mb_guess_purify_ws_bytes(int n) { return sizeof(double) * 3 * (size_t)n * n; }

extern "C" int mb_guess_purify_dev(int n, double* p, int steps, void* ws, cudaStream_t s) {
  if (n <= 0 || !p || steps < 0 || (steps > 0 && !ws)) return mb_set_error(MB_ERR_ARG, "mb_guess_purify_dev: bad args");
  if (steps == 0) return MB_OK;
  const long long nn = (long long)n * n;
  double* d = (double*)ws;
  double* d2 = d + nn;
  double* d3 = d2 + nn;
  const int grid = 148 * 8;
  unpack_half_kernel<<<grid, 256, 0, s>>>(n, p, d);
  MB_LAUNCH_CHECK();
  for (int it = 0; it < steps; ++it) {
    MB_TRY(mb_dgemm_dev('N', 'N', n, n, n, 1.0, d, n, d, n, 0.0, d2, n, s));
    MB_TRY(mb_dgemm_dev('N', 'N', n, n, n, 1.0, d2, n, d, n, 0.0, d3, n, s));
    mcweeny_kernel<<<grid, 256, 0, s>>>(nn, d2, d3, d);
    MB_LAUNCH_CHECK();
  }
  pack_twice_kernel<<<grid, 256, 0, s>>>(n, d, p);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

extern "C" size_t mb_gemm_split_ws_bytes(int m, int n, int k);
extern "C" int mb_gemm_split_ws(char transa, char transb, int m, int n, int k, double alpha, const double* a, int lda,
                                const double* b, int ldb, double beta, double* c, int ldc, void* ws, size_t ws_bytes,
                                int* err_dev, cudaStream_t stream);

// The same purification with the two products on the tensor cores (two BF16
// planes per operand, three products accumulated in FP32: about 1e-5 of
// |A||B| per element): the result only seeds the SCF, which converges to the
// same fixed point from it.  tc_ws: mb_gemm_split_ws_bytes(n, n, n) bytes, 1024-byte aligned;
// err_dev: the GEMM pipeline's error flag (zeroed by the caller, read after
// the stream is synchronised).
extern "C" int mb_guess_purify_split_dev(int n, double* p, int steps, void* ws, void* tc_ws, size_t tc_ws_bytes,
                                         int* err_dev, cudaStream_t s) {
  if (n <= 0 || !p || steps < 0 || (steps > 0 && (!ws || !tc_ws || !err_dev)))
    return mb_set_error(MB_ERR_ARG, "mb_guess_purify_split_dev: bad args");
  if (steps == 0) return MB_OK;
  const long long nn = (long long)n * n;
  double* d = (double*)ws;
  double* d2 = d + nn;
  double* d3 = d2 + nn;
  const int grid = 148 * 8;
  unpack_half_kernel<<<grid, 256, 0, s>>>(n, p, d);
  MB_LAUNCH_CHECK();
  for (int it = 0; it < steps; ++it) {
    MB_TRY(mb_gemm_split_ws('N', 'N', n, n, n, 1.0, d, n, d, n, 0.0, d2, n, tc_ws, tc_ws_bytes, err_dev, s));
    MB_TRY(mb_gemm_split_ws('N', 'N', n, n, n, 1.0, d2, n, d, n, 0.0, d3, n, tc_ws, tc_ws_bytes, err_dev, s));
    mcweeny_kernel<<<grid, 256, 0, s>>>(nn, d2, d3, d);
    MB_LAUNCH_CHECK();
  }
  pack_twice_kernel<<<grid, 256, 0, s>>>(n, d, p);
  MB_LAUNCH_CHECK();
  return MB_OK;
}

// ======================================================================
//                                  trainer
// ======================================================================
struct mb_guess_trainer {
  mb_guess_model view;  // aliases params / wbf (owns = false)
  float* params = nullptr;
  uint16_t* wbf = nullptr;
  float *grads = nullptr, *mom = nullptr, *vel = nullptr;
  int max_rows = 0;
  float* zs = nullptr;       // 3 * max_rows * HID
  uint16_t* acts = nullptr;  // 3 * max_rows * HID
  float* y = nullptr;        // max_rows * DOUT
  uint16_t* dz = nullptr;    // 2 * max_rows * HID
  double* loss = nullptr;
  long long steps[NT] = {0, 0, 0, 0, 0};
};

static void trainer_free(mb_guess_trainer* t) {
  void* ptrs[] = {t->params, t->wbf, t->grads, t->mom, t->vel, t->zs, t->acts, t->y, t->dz, t->loss};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  delete t;
}

extern "C" int mb_guess_trainer_create(const float* blob, int max_rows, mb_guess_trainer** out) {
  if (!blob || max_rows <= 0 || !out) return mb_set_error(MB_ERR_ARG, "mb_guess_trainer_create: bad args");
  *out = nullptr;
  const size_t nf = (size_t)NT * PER_TYPE, mr = (size_t)max_rows;
  mb_guess_trainer* t = new mb_guess_trainer();
  t->max_rows = max_rows;
  cudaError_t e = cudaSuccess;
#define TALLOC(ptr, bytes) if (e == cudaSuccess) e = cudaMalloc((void**)&(ptr), (bytes))
  TALLOC(t->params, nf * sizeof(float));
  TALLOC(t->wbf, nf * sizeof(uint16_t));
  TALLOC(t->grads, nf * sizeof(float));
  TALLOC(t->mom, nf * sizeof(float));
  TALLOC(t->vel, nf * sizeof(float));
  TALLOC(t->zs, 3 * mr * HID * sizeof(float));
  TALLOC(t->acts, 3 * mr * HID * sizeof(uint16_t));
  TALLOC(t->y, mr * DOUT * sizeof(float));
  TALLOC(t->dz, 2 * mr * HID * sizeof(uint16_t));
  TALLOC(t->loss, sizeof(double));
#undef TALLOC
  if (e == cudaSuccess) e = cudaMemcpy(t->params, blob, nf * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(t->grads, 0, nf * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(t->mom, 0, nf * sizeof(float));
  if (e == cudaSuccess) e = cudaMemset(t->vel, 0, nf * sizeof(float));
  if (e != cudaSuccess) {
    trainer_free(t);
    return mb_set_cuda_error(e, "mb_guess_trainer_create", __FILE__, __LINE__);
  }
  to_bf16_kernel<<<blocks_for((long long)nf, 256), 256>>>((long long)nf, t->params, t->wbf);
  MB_LAUNCH_CHECK();
  MB_CUDA(cudaDeviceSynchronize());
  t->view.params = t->params;
  t->view.wbf = t->wbf;
  t->view.owns = false;
  *out = t;
  return MB_OK;
}

extern "C" int mb_guess_trainer_destroy(mb_guess_trainer* t) {
  if (t) {
    cudaDeviceSynchronize();
    trainer_free(t);
  }
  return MB_OK;
}

extern "C" const mb_guess_model* mb_guess_trainer_model(mb_guess_trainer* t) { return t ? &t->view : nullptr; }

// Replaces the normalisation statistics of one type (host arrays; DIN, DIN,
// DOUT, DOUT floats).
extern "C" int mb_guess_trainer_set_norm(mb_guess_trainer* t, int type, const float* in_mean, const float* in_std,
                                         const float* out_mean, const float* out_std) {
  if (!t || type < 0 || type >= NT) return mb_set_error(MB_ERR_ARG, "mb_guess_trainer_set_norm: bad args");
  float* pm = t->params + (long long)type * PER_TYPE;
  MB_CUDA(cudaMemcpy(pm + OFF_IN_MEAN, in_mean, sizeof(float) * DIN, cudaMemcpyHostToDevice));
  MB_CUDA(cudaMemcpy(pm + OFF_IN_STD, in_std, sizeof(float) * DIN, cudaMemcpyHostToDevice));
  MB_CUDA(cudaMemcpy(pm + OFF_OUT_MEAN, out_mean, sizeof(float) * DOUT, cudaMemcpyHostToDevice));
  MB_CUDA(cudaMemcpy(pm + OFF_OUT_STD, out_std, sizeof(float) * DOUT, cudaMemcpyHostToDevice));
  return MB_OK;
}

// One training step on n rows of one type: forward, MSE loss over the type's
// valid outputs, backward, and (update != 0) an Adam step with learning rate
// lr.  x: n x DIN BF16 (normalised), yt: n x DOUT normalised targets.
// loss_out (optional) synchronises and returns the batch loss.
extern "C" int mb_guess_trainer_step(mb_guess_trainer* t, int type, int n, const uint16_t* x, const float* yt,
                                     float lr, int update, double* loss_out, cudaStream_t s) {
  if (!t || type < 0 || type >= NT || n <= 0 || n > t->max_rows || !x || !yt)
    return mb_set_error(MB_ERR_ARG, "mb_guess_trainer_step: bad args");
  const long long base = (long long)type * PER_TYPE;
  const long long nh = (long long)n * HID;
  float* zs = t->zs;
  uint16_t* acts = t->acts;
  MB_TRY(forward_impl(t->params, t->wbf, type, n, x, t->y, nullptr, zs, acts, s));
  MB_CUDA(cudaMemsetAsync(t->loss, 0, sizeof(double), s));
  uint16_t* dzA = t->dz;
  uint16_t* dzB = t->dz + (long long)t->max_rows * HID;
  lossgrad_kernel<<<blocks_for((long long)n * DOUT, 256), 256, 0, s>>>(n, nout_of(type), t->y, yt, dzA, t->loss);
  MB_LAUNCH_CHECK();
  const uint16_t* Wbf[4] = {t->wbf + base + OFF_W1, t->wbf + base + OFF_W2, t->wbf + base + OFF_W3,
                            t->wbf + base + OFF_W4};
  float* gW[4] = {t->grads + base + OFF_W1, t->grads + base + OFF_W2, t->grads + base + OFF_W3,
                  t->grads + base + OFF_W4};
  float* gb[4] = {t->grads + base + OFF_B1, t->grads + base + OFF_B2, t->grads + base + OFF_B3,
                  t->grads + base + OFF_B4};
  // layer l (0-based, 3 = output): dz_l has width nw[l]; its input a_{l-1}
  const int nw[4] = {HID, HID, HID, DOUT};
  const int kin[4] = {DIN, HID, HID, HID};
  uint16_t* dz = dzA;
  for (int l = 3; l >= 0; --l) {
    const uint16_t* ain = l == 0 ? x : acts + (long long)(l - 1) * nh;
    // dW_l (nw x kin) = dz^T a_in
    GemmArgs g{};
    g.M = nw[l]; g.N = kin[l]; g.K = n;
    g.a = dz; g.sam = 1; g.sak = nw[l];
    g.b = ain; g.sbk = kin[l]; g.sbn = 1;
    g.outf = gW[l]; g.ldo = kin[l];
    MB_TRY(launch_gemm<EPI_F32>(g, s));
    colsum_kernel<<<blocks_for(nw[l], 128), 128, 0, s>>>(n, nw[l], dz, gb[l]);
    MB_LAUNCH_CHECK();
    if (l > 0) {
      // dz_{l-1} = (dz W_l) * silu'(z_{l-1})
      uint16_t* dzn = dz == dzA ? dzB : dzA;
      GemmArgs h{};
      h.M = n; h.N = kin[l]; h.K = nw[l];
      h.a = dz; h.sam = nw[l]; h.sak = 1;
      h.b = Wbf[l]; h.sbk = kin[l]; h.sbn = 1;
      h.zin = zs + (long long)(l - 1) * nh; h.ldz = HID;
      h.outh = dzn; h.ldo = HID;
      MB_TRY(launch_gemm<EPI_DSILU>(h, s));
      dz = dzn;
    }
  }
  if (update) {
    long long st = ++t->steps[type];
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)st), c2 = 1.f - powf(b2, (float)st);
    const long long nt = TRAIN_END - TRAIN_BEGIN;
    adam_kernel<<<blocks_for(nt, 256), 256, 0, s>>>(nt, t->params + base + TRAIN_BEGIN, t->grads + base + TRAIN_BEGIN,
                                                    t->mom + base + TRAIN_BEGIN, t->vel + base + TRAIN_BEGIN,
                                                    t->wbf + base + TRAIN_BEGIN, lr, b1, b2, c1, c2, 1e-8f);
    MB_LAUNCH_CHECK();
  }
  if (loss_out) {
    double l = 0.0;
    MB_CUDA(cudaMemcpyAsync(&l, t->loss, sizeof(double), cudaMemcpyDeviceToHost, s));
    MB_CUDA(cudaStreamSynchronize(s));
    *loss_out = l / ((double)n * nout_of(type));
  }
  return MB_OK;
}

extern "C" int mb_guess_trainer_get(mb_guess_trainer* t, float* params_host, float* grads_host) {
  if (!t) return mb_set_error(MB_ERR_ARG, "mb_guess_trainer_get: null trainer");
  MB_CUDA(cudaDeviceSynchronize());
  const size_t nf = (size_t)NT * PER_TYPE;
  if (params_host) MB_CUDA(cudaMemcpy(params_host, t->params, nf * sizeof(float), cudaMemcpyDeviceToHost));
  if (grads_host) MB_CUDA(cudaMemcpy(grads_host, t->grads, nf * sizeof(float), cudaMemcpyDeviceToHost));
  return MB_OK;
}
