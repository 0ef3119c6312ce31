// Shared helpers for the mopac_gpu_b200 CUDA sources (sm_100a only).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "mopac_b200.h"

// Record a CUDA failure in the library's last-error slot and return MB_ERR_CUDA.
int mb_set_cuda_error(cudaError_t e, const char* what, const char* file, int line);
int mb_set_error(int code, const char* msg);

#define MB_CUDA(call)                                                        \
  do {                                                                       \
    cudaError_t _e = (call);                                                 \
    if (_e != cudaSuccess) return mb_set_cuda_error(_e, #call, __FILE__, __LINE__); \
  } while (0)

// Every kernel launch of the library is followed by MB_LAUNCH_CHECK, which
// also counts it (mb_launch_count()).
void mb_count_launch();
#define MB_LAUNCH_CHECK()                                                    \
  do {                                                                       \
    mb_count_launch();                                                       \
    cudaError_t _e = cudaGetLastError();                                     \
    if (_e != cudaSuccess) return mb_set_cuda_error(_e, "kernel launch", __FILE__, __LINE__); \
  } while (0)

// Kernel-family ids for the opt-in event timing (mb_kstats_*).
#define MB_KSTAT_TRIDIAG 0   // one tridiag_panel launch
#define MB_KSTAT_FOCK 1      // one fock2_kernel launch
#define MB_KSTAT_DENSITY 2   // one packed SYRK (density) launch
#define MB_KSTAT_EIGH 3      // one full eigensolve
#define MB_KSTAT_PSEUDO 4    // one pseudo-diagonalisation
#define MB_KSTAT_IDS 8
void mb_kstat_mark(int id, cudaStream_t s, bool begin);

// cudaMallocAsync from the device's default pool, which on first use per
// device is told to keep freed memory (release threshold: unlimited), so the
// library's per-call scratch is not unmapped and remapped at every
// synchronisation.  Process-local; changes no device setting.
cudaError_t mb_malloc_async(void** p, size_t bytes, cudaStream_t s);
template <class T>
inline cudaError_t mb_malloc_async(T** p, size_t bytes, cudaStream_t s) {
  return mb_malloc_async((void**)p, bytes, s);
}

#define MB_TRY(expr)            \
  do {                          \
    int _rc = (expr);           \
    if (_rc != MB_OK) return _rc; \
  } while (0)

// Packed lower triangle, row-major: element (r, c) with r >= c, 0-based.
__host__ __device__ __forceinline__ long long mb_tri(long long r, long long c) {
  return r * (r + 1) / 2 + c;
}

// Unrounded-product-free arithmetic: these keep the operation order of the
// reference's Fortran loops with one rounding per operation (no FMA).
#define DMUL(a, b) __dmul_rn((a), (b))
#define DADD(a, b) __dadd_rn((a), (b))
#define DSUB(a, b) __dsub_rn((a), (b))

// Per-atom layout shared by the dense kernels.  Atoms are 0-based; `first`
// is the 0-based first orbital, `nor` the orbital count (1 or 4), `lim` the
// pair count (1 or 10), `wrow` the offset of the atom's first two-centre W
// block and `cum` the prefix sum of `lim` over lower-numbered atoms, so the W
// block of pair (a, b), b < a, starts at wrow[a] + lim[a] * cum[b] and the
// one-centre block at wrow[a] + lim[a] * cum[a].
struct MbAtoms {
  int numat;
  const int* first;
  const int* nor;
  const int* lim;
  const long long* wrow;
  const int* cum;
};

// Integrals of many molecules in one launch (device pointers): molecule m
// owns atoms atom_off[m] .. atom_off[m+1]-1 of the concatenated tables
// (molecule-local first/wrow/cum), pairs pair_off[m] .. pair_off[m+1]-1 of
// enuc_pairs, and its packed H and W at hoff[m], woff[m].
struct MbHcoreBatch {
  int nmol;
  long long npair_tot, natom_tot;
  const long long* pair_off;
  const long long* atom_off;
  const long long* hoff;
  const long long* woff;
  const int* nat;
  const double* coord;
  const int* first;
  const int* nor;
  const int* lim;
  const long long* wrow;
  const int* cum;
  double* h;
  double* w;
  double* enuc_pairs;
  double* enuclr;
};

