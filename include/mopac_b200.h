/*
 * mopac_b200.h -- C ABI of libmopac_b200.so, the B200 (sm_100a) build of
 * MOPAC's semiempirical SCF hot path.
 *
 * Three layers, all plain C types (no torch, no C++):
 *
 *  (1) The reference GPU layer's bind(C) symbols with identical signatures
 *      (src/gpu/cuda_wrappers.cu in the reference), so a Fortran build that
 *      links the reference's wrappers links this library instead.  Host
 *      pointers, synchronous, like the originals; the arithmetic runs in this
 *      library's own kernels.
 *  (2) Fortran-callable shims (by-reference arguments, gfortran mangling) for
 *      the routines iter calls: fock2_, helect_, cnvg_, density_for_gpu_,
 *      eigenvectors_lapack_, diag_for_gpu_.
 *  (3) A device-resident native API (mb_*): an SCF context keeps H, W, F, P,
 *      C and the eigenvalues in HBM across iterations and returns int status
 *      codes.  Device-pointer kernel entry points (mb_*_dev) are exported for
 *      callers that manage their own device memory.
 *
 * Packed matrices follow MOPAC: lower triangle by rows, element (i, j), i >= j
 * (1-based) at i*(i-1)/2 + j, identical to the column-major upper triangle.
 * Square matrices are column-major.  Orbital and atom indices passed as
 * nfirst/nlast are 1-based like the reference; everything else is 0-based.
 *
 * Thread safety: one context must not be used from two threads at once
 * (the reference is not thread-safe either, README.md:254-255); separate
 * contexts are independent.
 */
#ifndef MOPAC_B200_H
#define MOPAC_B200_H

#include <stddef.h>
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

/* CUDA stream handle without pulling in cuda_runtime.h */
#ifndef __CUDA_RUNTIME_H__
typedef struct CUstream_st* cudaStream_t;
#endif

/* ---------------------------------------------------------------- status */
#define MB_OK 0
#define MB_ERR_ARG 1          /* bad argument or size                         */
#define MB_ERR_CUDA 2         /* CUDA runtime error (message in mb_last_error) */
#define MB_ERR_NOCONV 3       /* SCF did not reach self-consistence in itrmax  */
#define MB_ERR_TIMEOUT 4      /* a bounded device-side wait gave up            */
#define MB_ERR_UNSUPPORTED 5  /* element or option outside this build          */
#define MB_ERR_NUMERIC 6      /* NaN/Inf detected or eigensolver failure       */
#define MB_ERR_NOMEM 7        /* device allocation failed                      */

int mb_version(void);                 /* 10000*major + 100*minor + patch       */
long long mb_launch_count(void);      /* kernels this library has launched     */
/* Opt-in CUDA-event timing per kernel family, recorded on the launching
 * stream: 0 Householder panel, 1 Fock build, 2 density, 3 full eigensolve,
 * 4 pseudo-diagonalisation.  mb_kstats_read syncs, returns and clears id. */
void mb_kstats_enable(int on);
int mb_kstats_read(int id, long long* count, double* total_ms);
const char* mb_last_error(void);      /* thread-local text of the last failure */

/* ------------------------------------------------ (3) device-resident API */

/* Device-side atom layout used by the dense kernels (see mb_atoms_create). */
typedef struct MbAtomsDev {
  int numat;
  const int* first;      /* 0-based first orbital of each atom               */
  const int* nor;        /* orbitals on the atom (1 or 4)                    */
  const int* lim;        /* orbital pairs on the atom (1 or 10)              */
  const long long* wrow; /* offset of the atom's first two-centre W block    */
  const int* cum;        /* prefix sum of lim over lower-numbered atoms      */
} MbAtomsDev;

typedef struct mb_ctx mb_ctx; /* opaque SCF context */

typedef struct mb_scf_opts {
  int pseudo;        /* 1: pseudo-diagonalise once newdg is set (reference's
                        commented-out path, SCF/iter.F90:847-861); 0: full
                        diagonalisation every iteration like the fork     */
  int itrmax;        /* iteration cap (ITRY), reference default 2000      */
  double scfcrt;     /* SCF criterion, reference default 1e-4 kcal/mol    */
  int precision;     /* 0: all FP64; 1: density and Fmo GEMMs in split BF16
                        precision on the tensor cores until max|dP| <
                        switch_pl, FP64 after (convergence is only
                        declared in FP64)                                 */
  double switch_pl;  /* precision switch threshold (default 1e-4)         */
  int verbose;       /* print one line per iteration to stderr            */
  int pulay;         /* 1: Pulay's converger once newdg is set, like the
                        PULAY keyword (SCF/iter.F90:135, :815-831); cnvg is
                        then skipped (:899) and the shift is -8 / 0 (:417) */
  int guess;         /* 1: start from the density given by mb_ctx_set_guess
                        or predicted by mb_ctx_guess, entered like an OLDENS
                        density (SCF/iter.F90:151-158); 0: the standard
                        diagonal guess                                     */
  double finish_dp;  /* FP64 finish (an addition to iter): once iter's test
                        (SCF/iter.F90:675-690) passes in FP64, convergence
                        is accepted only when the last density update moved
                        no element of P by more than finish_dp; until then
                        the loop goes on in FP64 with both of the rotation
                        sweep's thresholds (bigeps and 0.05 max|Fmo|) at 0,
                        every occupied-virtual pair rotated, and, from its first
                        iteration, the orbital energies of the current
                        vectors (diag C^T F C) in the rotation angles.  It
                        takes the SCF to its self-consistent point instead
                        of stopping inside iter's criterion.  < 0
                        (default): 1e-7 when precision = 1, off when
                        precision = 0; 0: off                              */
  int finish_max;    /* cap on the iterations the finish adds (default 40) */
  double bshift;     /* -n for the SHIFT=n keyword (SCF/iter.F90:119, :131);
                        default -80 (no keyword).  0 (SHIFT=0) turns the
                        level shift off and lets newdg switch on as soon as
                        the density change falls below trans (:136)       */
  int camp;          /* 1: the CAMP keyword (SCF/iter.F90:134): Camp-King's
                        interp (matrix/interp.F90) on the vectors from the
                        third iteration, a full diagonalisation in every
                        iteration; an interpolated pass (interp's mode 3)
                        builds the rotated vectors' density without Pulay,
                        diagonalisation or cnvg and is not counted.
                        Independently of it, iter's forced switch-on of all
                        convergers (:351-372) runs when niter passes
                        itrmax - 10: Pulay and Camp-King on, bshift = 4.44,
                        the count restarts.  Default 0                    */
} mb_scf_opts;

typedef struct mb_scf_result {
  double escf;       /* heat of formation from iter, kcal/mol (no post-SCF
                        geometry terms)                                  */
  double ee;         /* electronic energy, eV                              */
  int niter;
  int converged;
  int n_full_diag;   /* full eigensolves performed                         */
  int n_pseudo_diag; /* pseudo-diagonalisations performed                  */
  double pl;         /* last max|dP_ii|                                    */
  double t_fock_ms, t_diag_ms, t_density_ms, t_other_ms; /* device-timed  */
  double t_total_ms; /* CUDA events on the context stream around the SCF   */
  int n_pulay;       /* Pulay extrapolation steps taken                    */
  int n_split;       /* iterations whose density / Fmo GEMMs ran in the
                        split BF16 precision (opts.precision = 1)          */
  int n_finish;      /* iterations the FP64 finish added                   */
  double dp;         /* max|P_k - P_(k-1)| of the last density update
                        (computed when the finish is on, else -1)          */
  int n_interp;      /* Camp-King interpolated passes (interp mode 3)      */
  int forced_on;     /* 1 when iter forced all convergers on (niter passed
                        itrmax - 10, SCF/iter.F90:351-372)                 */
  int exit_split;    /* 1 when the exit diagonalisation (SCF/iter.F90 label
                        600) was solved as the occupied and virtual blocks
                        of C^T F C after the FP64 finish (an addition to
                        iter: the two blocks' eigenvalues differ from the
                        whole matrix's by at most ||B||_F^2 / gap, accepted
                        below 1e-8 eV, and a first-order rotation takes the
                        coupling B out of the vectors); 0: the full
                        eigensolve, counted in n_full_diag                 */
  double exit_coupling; /* ||C_v^T F C_o||_F at the exit (eV) when the split
                        was tried, else -1                                 */
} mb_scf_result;

void mb_scf_opts_default(mb_scf_opts* o);

/* numat atoms with atomic numbers nat (H, C, O in this build); coordinates
 * in Angstrom (numat x 3, host).  Computes nothing yet. */
int mb_ctx_create(int numat, const int* nat, const double* coord, mb_ctx** out);
int mb_ctx_destroy(mb_ctx* ctx);
/* The atomic term of the heat of formation, sum over atoms of the
 * experimental heat of atomisation minus eisol in kcal/mol
 * (interface/mopac_api_initialize.F90:340-350); NaN for an element outside
 * this build.  What iter adds to (ee + enuclr) * fpc_9. */
double mb_atheat(int numat, const int* nat);
int mb_ctx_norbs(const mb_ctx* ctx);
long long mb_ctx_n2elec(const mb_ctx* ctx);
int mb_ctx_nclose(const mb_ctx* ctx);

/* One-electron matrix H, two-electron integrals W and core-core energy from
 * the coordinates, on the GPU (hcore, integrals/hcore.F90:150-297). */
int mb_ctx_hcore(mb_ctx* ctx);
/* Or supply them (host pointers): h[mpack], w[n2elec]. */
int mb_ctx_set_hw(mb_ctx* ctx, const double* h, const double* w, double enuclr);
/* Copy out H (mpack), W (n2elec), enuclr to host. */
int mb_ctx_get_hw(mb_ctx* ctx, double* h, double* w, double* enuclr);

/* Closed-shell RHF SCF (iter, SCF/iter.F90) from the standard diagonal guess
 * (moldat.F90:731-760).  The whole loop runs on the device; only scalars
 * cross to the host each iteration.  Work arrays are allocated in the
 * context on first use and kept for later calls (the pseudo-diagonalisation,
 * the split-precision planes, Pulay's histories, and for an SCF that ends in
 * the FP64 finish the split exit diagonalisation's 2 n^2 + ~(3/2)(k^2 + v^2)
 * + 2 k v doubles, k = nclose, v = norbs - nclose). */
int mb_scf_run(mb_ctx* ctx, const mb_scf_opts* opts, mb_scf_result* res);

/* Starting density for opts.guess = 1: a host packed total density (mpack)
 * such as a previous SCF's P -- the reference reads one with OLDENS
 * (SCF/iter.F90:151-158, den_in_out) -- or the learned guess (below). */
int mb_ctx_set_guess(mb_ctx* ctx, const double* p);

/* Results to host: density P (mpack), eigenvectors C (norbs x norbs,
 * column-major), eigenvalues (norbs), Fock matrix F (mpack). */
int mb_ctx_get_density(mb_ctx* ctx, double* p);
int mb_ctx_get_vectors(mb_ctx* ctx, double* c, double* eigs);
int mb_ctx_get_fock(mb_ctx* ctx, double* f);
/* Device pointers owned by the context (valid until destroy). */
int mb_ctx_device_ptrs(mb_ctx* ctx, double** h, double** w, double** f, double** p,
                       double** c, double** eigs);
int mb_ctx_atoms_dev(mb_ctx* ctx, MbAtomsDev* out);

/* Cartesian gradient of the SCF energy at the context's density (dcart,
 * forces/dcart.F90:16-300, for a molecule, RHF, the default finite
 * difference: every pair's energy as dhc forms it, forces/dhc.F90, with atom
 * jj moved 0.5e-4 A along all axes and atom ii 1e-4 A along each).  dxyz:
 * host array of 3*numat doubles, kcal/mol/A, atom-major.  Post-SCF
 * corrections (PM7 dispersion, hydrogen bonds) are not included. */
int mb_ctx_gradient(mb_ctx* ctx, double* dxyz);

/* dfock2 (forces/dfock2.F90:16-279) on device arrays: f (in/out), ptot, p
 * packed (mpack), w the derivative integrals of the pairs (nati, jj) in
 * partner order, mb_dfock2_w_len values (100 / 10 / 1 per heavy-heavy /
 * heavy-light / light-light pair); nfirst, nlast host, 1-based; nati
 * 1-based.  Bit-identical to the reference's loop.  mb_dfock2_w_len returns
 * -1 for bad arguments or d orbitals. */
long long mb_dfock2_w_len(int numat, const int* nfirst, const int* nlast, int nati);
int mb_dfock2_dev(int numat, const int* nfirst, const int* nlast, int nati, double* f, const double* ptot,
                  const double* p, const double* w, cudaStream_t stream);
/* The same on device arrays: nat_d/coord_d (A) as for mb_hcore_dev, p the
 * packed density; ws of mb_dcart_ws_bytes(numat) bytes (3 doubles per
 * atom pair); dxyz_dev 3*numat doubles. */
size_t mb_dcart_ws_bytes(int numat);
int mb_dcart_dev(const int* nat_d, const double* coord_d, const MbAtomsDev* at, int numat,
                 const double* p, double* dxyz_dev, void* ws, size_t ws_bytes, cudaStream_t stream);

/* --------------------------------------------- device-pointer kernels */
/* Atom layout on the device from host nfirst/nlast (1-based). */
int mb_atoms_create(int numat, const int* nfirst, const int* nlast, MbAtomsDev* out);
int mb_atoms_destroy(MbAtomsDev* atoms);

/* F = start + two-centre + one-centre terms (fock2 mode 2 with fock1).
 * start = H (use_shift = 0) or H + shift*PA + 1e-16*i, F_ii -= shift.
 * Bit-identical to the reference loop order.  All pointers device. */
int mb_fock2_dev(const MbAtomsDev* atoms, double* f, const double* h, const double* ptot,
                 const double* pa, const double* w, double shift, int use_shift,
                 cudaStream_t stream);

/* The same Fock build with a caller-owned device workspace of at least
 * mb_fock2_ws_bytes(numat) bytes, 256-byte aligned (mb_fock2_dev takes one
 * from the stream-ordered allocator per call).  The workspace holds every
 * atom's staged partner contributions (10 numat^2 doubles); calls that
 * overlap in time need separate workspaces. */
size_t mb_fock2_ws_bytes(int numat);
int mb_fock2_ws(const MbAtomsDev* atoms, double* f, const double* h, const double* ptot,
                const double* pa, const double* w, double shift, int use_shift, void* ws,
                size_t ws_bytes, cudaStream_t stream);

/* helect: sum_{i>j} P(H+F) + 0.5 sum_i P(H+F), written to *out (device). */
int mb_helect_dev(int n, const double* p, const double* h, const double* f, double* out,
                  cudaStream_t stream);

/* Self-test of the bounded mbarrier wait the tcgen05 GEMM uses: waits
 * limit_ns (1 ns .. 0.1 s, else MB_ERR_ARG) on a barrier that never
 * completes and writes out_dev[0] = 1 (the wait gave up) and out_dev[1] =
 * nanoseconds waited.  No reference counterpart: it exercises this library's
 * failure path without faulting or hanging anything. */
int mb_selftest_bounded_wait(unsigned long long limit_ns, long long* out_dev, cudaStream_t stream);

/* helect without any device allocation.  No counterpart in the reference: it
 * exists for callers that cannot allocate device memory where they need the
 * energy (a host arena that owns all device memory, stream capture, hard
 * latency loops).  Scratch is a fixed 256 KiB array inside the library, so
 * n <= 16384 (larger n: MB_ERR_ARG); calls share that array and must not
 * overlap on the GPU; the first call on a device resolves the array's address
 * and should happen outside stream capture.  That address is cached per
 * device for the life of the process: a caller that resets the device
 * (cudaDeviceReset, which destroys the primary context) leaves the cached
 * address stale, so it must not call this entry point afterwards. */
int mb_helect_noalloc(int n, const double* p, const double* h, const double* f, double* out,
                      cudaStream_t stream);

/* cnvg (SCF/cnvg.F90) for RHF.  pnew is extrapolated in place, p and p1 are
 * the history; *pl_out (device) receives max|dP_ii|.  Bit-identical. */
int mb_cnvg_dev(int norbs, double* pnew, double* p, double* p1, int niter, double* pl_out,
                cudaStream_t stream);

/* One step of Pulay's converger, pulay(f, p, n, fppf, fock, emat, lfock,
 * nfock, msize, start, pl) (SCF/pulay.F90:16-180), on device histories.
 * f, p: packed n x n (device); f is replaced by the extrapolated Fock matrix
 * once two entries are stored.  fppf, fock: device histories of mfock
 * entries in the reference's layouts (commutator slot l is the block
 * fppf[l*linear ...], Fock entry i of slot l is fock[l + i*mfock]).  emat:
 * host, column-major ldemat x ldemat (ldemat >= mfock + 1).  lfock, nfock,
 * start (0/1), pl: host scalars with the reference's meaning.  ws: device,
 * 256-byte aligned, mb_pulay_ws_bytes(n) bytes.  mfock <= 16.  Synchronises
 * the stream once (the B matrix is inverted on the host). */
size_t mb_pulay_ws_bytes(int n);
int mb_pulay_ws(int n, double* f, const double* p, double* fppf, double* fock, int mfock,
                double* emat, int ldemat, int* lfock, int* nfock, int* start, double* pl, void* ws,
                cudaStream_t stream);
/* osinv(a, n, d) (matrix/osinv.F90): in-place Gauss-Jordan inverse with full
 * pivoting of the column-major n x n host matrix a; returns d (0 when a pivot
 * is below 1e-8). */
double mb_osinv(double* a, int n);

/* Split-precision GEMM on the tcgen05 tensor cores: C = alpha*op(A)*op(B) +
 * beta*C (column-major, BLAS argument meaning), each FP64 operand split into
 * two BF16 planes and three BF16 products accumulated in FP32 (relative error
 * ~1e-5 of |A||B|).  ws: device, 1024-byte aligned, mb_gemm_split_ws_bytes
 * bytes.  err_dev: device int the kernel sets to 1 if a pipeline wait ran out
 * (results are then not written); the caller zeroes and reads it. */
size_t mb_gemm_split_ws_bytes(int m, int n, int k);
int mb_gemm_split_ws(char transa, char transb, int m, int n, int k, double alpha, const double* a,
                     int lda, const double* b, int ldb, double beta, double* c, int ldc, void* ws,
                     size_t ws_bytes, int* err_dev, cudaStream_t stream);
/* Density with the same split arithmetic: packed P = occ * C_occ C_occ^T
 * (lower tiles only, written straight into the packed layout). */
size_t mb_density_split_ws_bytes(int n, int nocc);
int mb_density_split_ws(int n, int nocc, double occ, const double* c, int ldc, double* p, void* ws,
                        size_t ws_bytes, int* err_dev, cudaStream_t stream);

/* ----------------------------------------------- batched small molecules */
/* Many closed-shell molecules (n <= 128 basis functions, n * nocc <= 11008)
 * in one persistent launch, one CTA per molecule SCF at a time (iter with a
 * full diagonalisation every iteration, SCF/iter.F90:16-1107; Fock and cnvg
 * bit-identical to the oracle's).  numat[m] atoms of molecule m; nat and
 * coord (Angstrom, 3 per atom) concatenated over the molecules, host arrays.
 * Integrals are computed on the GPU at creation. */
typedef struct mb_batch mb_batch;
int mb_batch_create(int nmol, const int* numat, const int* nat, const double* coord, mb_batch** out);
int mb_batch_destroy(mb_batch* batch);
int mb_batch_nmol(const mb_batch* batch);
/* Runs every molecule's SCF; per molecule escf (kcal/mol, iter's), niter,
 * converged (host arrays of nmol, each optional); *t_ms: CUDA-event time of
 * the launch.  The launch sequence is captured into a CUDA graph on the first
 * run of a configuration and replayed after that. */
int mb_batch_run(mb_batch* batch, const mb_scf_opts* opts, double* escf, int* niter, int* converged,
                 double* t_ms);
int mb_batch_get_density(mb_batch* batch, int m, double* p);
/* Launch configuration: back-transformation block size nb (4, 8 or 16
 * reflectors per compact-WY block) and CTAs per SM (0: as many as fit).
 * mb_batch_autotune times all six on this batch (two runs each) and keeps the
 * fastest; every configuration gives the same SCFs up to FP64 rounding. */
int mb_batch_set_config(mb_batch* batch, int nb, int per_sm);
int mb_batch_get_config(const mb_batch* batch, int* nb, int* grid);
int mb_batch_autotune(mb_batch* batch, const mb_scf_opts* opts, int* nb, int* per_sm, double* ms);
/* Phase timing (off by default): SM cycles summed over all CTAs of the last
 * run, out[8] = Fock, energy and control, Householder, bisection, inverse
 * iteration, back-transformation, density, cnvg. */
int mb_batch_set_phase_timing(mb_batch* batch, int on);
int mb_batch_phase_cycles(mb_batch* batch, unsigned long long* out);
int mb_batch_get_hw(mb_batch* batch, int m, double* h, double* w, double* enuclr);

/* ------------------------------------------------ MOZYME (sparse blocks) */
/* Pair-block storage of P, H, F (MOZYME/fillij.F90:20-230, first call,
 * molecular): for atom i in order, partners j < i with r^2 < cutof2 (block
 * iorbs(i) x iorbs(j), i's orbitals outer), then i's lower triangle.  Device
 * arrays; pair entries of atom i are pair_ptr[i] .. pair_ptr[i+1]-1, partners
 * ascending, the diagonal block last; pair_off = the reference's nijbo. */
typedef struct MbMzLayout {
  int numat;
  long long mpack, npairs;
  const int* iorbs;
  const int* pair_ptr;
  const int* pair_i;
  const int* pair_j;
  const long long* pair_off;
  /* two-electron integrals of the stored pairs: entry e's block (100, 10 or
   * 1 values for a pair, ilim^2 for an atom's own entry) at pair_woff[e], nw
   * in all -- the dense W's order with the pairs outside cutof2 left out */
  const long long* pair_woff;
  long long nw;
  /* every stored partner of atom a, both directions, ascending:
   * nbr_atom[nbr_ptr[a] ..], with the pair entry of (max, min) in nbr_entry */
  const int* nbr_ptr;
  const int* nbr_atom;
  const long long* nbr_entry;
  double cutof1, cutof2;
  const int* first;   /* 0-based first orbital of each atom */
  int norbs;
} MbMzLayout;
/* Occupied LMOs on the device: cocc as in MOZYME_C plus, per atom, the LMOs
 * containing it (ascending) and the offset of its coefficients in cocc. */
typedef struct MbMzLmos {
  int nlmo;
  const int* atom_ptr;
  const int* atom_lmo;
  const int* atom_coff;
  const double* cocc;
  /* the reference's own arrays: ncf (atoms per LMO), nncf (0-based start in
   * icocc), icocc (1-based atom numbers), ncocc (0-based start in cocc) */
  const int* ncf;
  const int* nncf;
  const int* icocc;
  const int* ncocc;
  long long nentries;  /* length of icocc (icocc_dim) */
  long long ncoeff;    /* length of cocc (cocc_dim) */
} MbMzLmos;
/* Builds the layout (host coordinates in Angstrom, cutoffs squared, as
 * cutof1/cutof2 in fillij); nijbo (optional, host numat x numat) receives the
 * reference's table: offset, -2 (cutof2 <= r^2 < cutof1) or -1. */
int mb_mz_layout_create(int numat, const int* iorbs, const double* coord, double cutof1, double cutof2,
                        MbMzLayout* out, long long* nijbo);
int mb_mz_layout_destroy(MbMzLayout* layout);
/* hcore_for_MOZYME (MOZYME/hcore_for_MOZYME.F90, molecular, mode 0) on the
 * layout: h (mpack) the one-electron matrix in pair blocks, w (nw) the stored
 * pairs' two-centre integrals and every atom's one-centre block,
 * *enuclr_dev the core-core energy over every atom pair (pairs not stored:
 * outer2's monopole in the cutof2-cutof1 band, outer1's feathered point
 * charge beyond).  nat, coord: device (atomic numbers; Angstrom).  ws:
 * mb_mz_hcore_ws_bytes(layout) bytes of device scratch.  Any cutoff: a far
 * pair inside PM7's 7 A feathering radius takes outer1's or outer2's
 * diagonal terms (MOZYME/outer1.F90, outer2.F90), one beyond it the rotated
 * core attraction, which is the same point charge there. */
size_t mb_mz_hcore_ws_bytes(const MbMzLayout* layout);
int mb_mz_hcore_dev(const MbMzLayout* layout, const int* nat, const double* coord, double* h, double* w,
                    double* enuclr, void* ws, cudaStream_t stream);
/* idiag (host, norbs): 1-based position of each orbital's diagonal element,
 * as iter_for_MOZYME.F90:183-190. */
int mb_mz_idiag(const MbMzLayout* layout, long long* idiag);
/* Uploads LMOs given in the reference's arrays (host; icocc 1-based atoms,
 * nncf/ncocc 0-based starts).  icocc_dim and cocc_dim are the arrays'
 * lengths: the space between one LMO's end and the next LMO's start (and,
 * for the last, up to these lengths) is where diagg2 may grow the LMO. */
int mb_mz_lmos_create(int numat, const int* iorbs, int nlmo, const int* ncf, const int* nncf,
                      const int* icocc, const int* ncocc, const double* cocc, long long icocc_dim,
                      long long cocc_dim, MbMzLmos* out);
/* Rebuilds the per-atom index after diagg2 has grown LMOs (mb_mz_density_dev
 * reads it). */
int mb_mz_lmos_refresh(int numat, const int* iorbs_host, MbMzLmos* lmos);
/* The same index built on the device, in place, on `stream` (iorbs_dev: a
 * device array, e.g. MbMzLayout.iorbs): each atom's LMOs ascending, as the
 * host version orders them.  Synchronises the stream once to report
 * malformed LMOs (MB_ERR_ARG). */
int mb_mz_lmos_refresh_dev(int numat, const int* iorbs_dev, MbMzLmos* lmos, cudaStream_t stream);
int mb_mz_lmos_destroy(MbMzLmos* lmos);
/* density_for_MOZYME(p, mode, nclose, partp) (MOZYME/density_for_MOZYME.F90:16):
 * mode 0: P = 2 sum_LMO c c^T; -1: P = -2 (sum - partp/2); 1: P = 2 (sum +
 * partp/2); other: P = sum + partp/2.  Bit-identical to the reference's
 * loop. */
int mb_mz_density_dev(const MbMzLayout* layout, const MbMzLmos* lmos, int mode, const double* partp,
                      double* p, cudaStream_t stream);
/* buildf(f, partf, 0) -> fock2z (MOZYME/buildf.F90:16, fock2z.F90:669-1293),
 * whole-F mode, direct and semi-direct (the reference's defaults), s/p atoms:
 * F = H + the two-electron terms of the stored pairs (w: their integrals in
 * pair_woff order), the point-charge monopole qe(b) ev a0 / r of every
 * other pair, then each atom's one-centre terms.  coord: device, numat x 3
 * Angstrom.  Needs cutof2 >= 49 (7 A), where the reference's feathering
 * weight is exactly zero for every pair outside the cutoff, so its dipole
 * terms vanish (mb_mz_fock_nat_dev takes shorter cutoffs).  Bit-identical
 * to the reference's loop. */
size_t mb_mz_fock_ws_bytes(const MbMzLayout* layout);
int mb_mz_fock_dev(const MbMzLayout* layout, const double* coord, const double* w, const double* ptot,
                   const double* h, double* f, void* ws, cudaStream_t stream);
/* The same with the atomic numbers (device, numat ints), which a cutoff
 * below 7 A needs: a pair outside cutof2 but inside PM7's 7 A feathering
 * radius takes fock2z's feathered monopole and, inside cutof1, its dipole
 * terms (MOZYME/fock2z.F90:440-634); mb_mz_fock_dev (nat = NULL) refuses
 * such cutoffs with MB_ERR_UNSUPPORTED. */
int mb_mz_fock_nat_dev(const MbMzLayout* layout, const int* nat, const double* coord, const double* w,
                       const double* ptot, const double* h, double* f, void* ws, cudaStream_t stream);

/* diagg1 (MOZYME/diagg1.F90:16-503): F psi for every virtual LMO, the virtual
 * LMO energies eigv, the occupied-virtual interaction list (fmo) -- rebuilt
 * when idiagg <= 5 or even, recomputed on the previous list otherwise -- and,
 * when idiagg <= 2 or divisible by 4, the occupied LMO energies eigs.  All
 * cutoffs and orders as the reference; fao and p in the block storage.
 * state[4] (host, in/out): fref, safety, oldlim, tiny of the previous call
 * (start with 10, 1, 0, 0).  nfmo (device, nvir), ifmo (device, 2 x cap,
 * 1-based LMO numbers) and fmo (device, cap) carry the list between calls;
 * *nij: capacity in, entries out (MB_ERR_UNSUPPORTED if a rebuilt list would
 * not fit, where the reference truncates).  *eigs_done: 1 if eigs was
 * computed.  *sumt: the sum of |fmo| over the evaluated pairs (a fixed-order
 * parallel sum; diagnostic only in the reference).  Bit-identical fmo, eigv,
 * eigs and tiny. */
size_t mb_mz_diagg1_ws_bytes(const MbMzLayout* layout, const MbMzLmos* occ, const MbMzLmos* vir);
int mb_mz_diagg1_dev(const MbMzLayout* layout, const MbMzLmos* occ, const MbMzLmos* vir, const double* fao,
                     const double* p, int idiagg, double* state, int* nfmo, int* ifmo, double* fmo,
                     long long* nij, double* eigv, double* eigs, int* eigs_done, double* sumt, void* ws,
                     cudaStream_t stream);

/* diagg2 (MOZYME/diagg2.F90:16-359): the 2x2 rotations of diagg1's list in
 * list order, with the reference's growth of LMOs by atoms whose new
 * coefficients exceed thresh and its rejection of rotations that would
 * overflow an LMO's space (retried with alpha <- (alpha + 1)/2 when the
 * last two calls rejected equally often).  Rotations touching disjoint LMO
 * pairs commute, so the list runs in dependency levels, each level's
 * rotations in parallel: bit-identical coefficients and atom lists.
 * occ/vir are modified in place (call mb_mz_lmos_refresh on occ before the
 * next density).  eigs/eigv: occupied / virtual LMO energies (device);
 * ctl[5] (host): damping constant, shift, thresh, diagg1's tiny, bigeps;
 * nrejct[2] (host, in/out) the rejection counts of the last two calls.
 * *sumb: the sum of |beta| (fixed-order, diagnostic in the reference). */
int mb_mz_diagg2_dev(const MbMzLayout* layout, MbMzLmos* occ, MbMzLmos* vir, const int* ifmo,
                     const double* fmo, long long nij, const double* eigs, const double* eigv, int idiagg,
                     const double* ctl, int* nrejct, double* sumb, long long* nrej, cudaStream_t stream);

/* helecz() (MOZYME/helecz.F90:16): sum p(h+f) with diagonal elements
 * weighted 1/2; *out (device).  Fixed-order parallel reduction. */
size_t mb_mz_helecz_ws_bytes(void);
int mb_mz_helecz_ws(long long mpack, int norbs, const long long* idiag, const double* p,
                    const double* h, const double* f, double* out, double* ws, cudaStream_t stream);
/* cnvgz(pnew, p, p1, p2, p3, niter, idiag) (MOZYME/cnvgz.F90:16), device
 * arrays; use3 = use_three_point_extrap; *pmax_out (device) = max|pnew - p|
 * before extrapolation.  Bit-identical. */
size_t mb_mz_cnvgz_ws_bytes(void);
int mb_mz_cnvgz_ws(int norbs, long long mpack, double* pnew, double* p, double* p1, double* p2,
                   double* p3, int niter, const long long* idiag, int use3, double* pmax_out, void* ws,
                   cudaStream_t stream);
/* The routines iter_for_MOZYME calls between the kernels above.
 * check (MOZYME/check.F90): renormalises every LMO in place; norm2[nlmo]
 * (device) receives the squared norms before the scaling and *error (host,
 * optional; synchronises) their summed |1 - norm2| (the reference stops above
 * 0.1).  iorbs: device, per atom. */
int mb_mz_check_dev(const MbMzLmos* lmos, const int* iorbs, double* norm2, double* error,
                    cudaStream_t stream);
/* tidy's compression step (MOZYME/tidy.F90:66-107): every LMO drops the
 * atoms whose squared coefficients sum to thresh (1e-13 in iter_for_MOZYME)
 * or less, keeping the order of the rest, within its own storage; call
 * mb_mz_lmos_refresh afterwards.  The reference's repacking of the storage
 * is not restated: every LMO keeps its own space.  iorbs: device. */
int mb_mz_tidy_dev(MbMzLmos* lmos, const int* iorbs, double thresh, cudaStream_t stream);
/* eimp (MOZYME/eimp.F90): p's first element of every stored off-diagonal
 * block becomes the block's sum of squared f elements. */
int mb_mz_eimp_dev(const MbMzLayout* layout, double* p, const double* f, cudaStream_t stream);
/* hbonds (MOZYME/hbonds.F90), called by addhb with cutoff 1, 0.1, 0.01, 1e-3
 * on its first four calls: (virtual, occupied) LMO pairs (1-based, ifmo[2e],
 * ifmo[2e+1]; fmo[e] = 0.1) around stored atom pairs with sum F^2 > cutoff
 * and sum P^2 < 1e-10, in the reference's order; at most cap entries.
 * Synchronises the stream. */
int mb_mz_hbonds_dev(const MbMzLayout* layout, const MbMzLmos* occ, const MbMzLmos* vir,
                     const double* f, const double* p, double cutoff, long long cap, int* ifmo,
                     double* fmo, long long* nij, cudaStream_t stream);

/* The whole MOZYME SCF on the device, iter_for_MOZYME
 * (MOZYME/iter_for_MOZYME.F90:218-630) for a closed-shell system with every
 * atom in the SCF (no partial SCF, no setupk): from the starting LMOs occ and
 * vir (updated in place) and the pair-block integrals (h, w from
 * mb_mz_hcore_dev; coord device, Angstrom), per iteration tidy's
 * compression, check, eimp,
 * diagg1 + diagg2 + density, addhb every third iteration (four at most),
 * cnvgz while the three-point extrapolation is on, buildf, helecz, isitsc's
 * 1SCF test (diagg1's tiny below 5 scfcrt and |dE| below scfcrt on two
 * consecutive iterations) and the shift control.  p and f (device, mpack)
 * are the working density and Fock matrix and hold the last ones on return.
 * iorbs_host: orbitals per atom (host).  MB_ERR_NOCONV after itrmax
 * iterations.  tidy's repacking of the storage is not restated: every LMO
 * needs spare atom slots (the space mb_mz_lmos_create leaves after it); a
 * rotation that would overflow one is rejected. */
typedef struct mb_mz_scf_opts {
  double scfcrt;   /* selcon, kcal/mol (default 1e-2)                       */
  int itrmax;      /* iteration cap (default 2000)                           */
  long long cap;   /* capacity of the interaction lists (0: 300 norbs)       */
  int verbose;     /* one line per iteration to stderr                       */
  const int* nat;  /* atomic numbers on the device, or NULL; needed for a
                      cutoff below 7 A (mb_mz_fock_nat_dev)                  */
} mb_mz_scf_opts;
typedef struct mb_mz_scf_result {
  double escf;          /* heat of formation, kcal/mol (no post-SCF terms)   */
  double ee;            /* electronic energy, eV                             */
  int niter, converged;
  double t_total_ms;    /* CUDA events on the stream around the SCF          */
  long long nrejected;  /* rotations diagg2 rejected for want of space       */
} mb_mz_scf_result;
void mb_mz_scf_opts_default(mb_mz_scf_opts* o);
int mb_mz_scf_run(const MbMzLayout* layout, const int* iorbs_host, MbMzLmos* occ, MbMzLmos* vir,
                  const double* coord, const double* w, const double* h, double enuclr, double atheat,
                  const mb_mz_scf_opts* opts, double* p, double* f, mb_mz_scf_result* res,
                  cudaStream_t stream);

/* P (packed) = occ * C[:, 0:nocc] C[:, 0:nocc]^T, FP64. */
int mb_density_dev(int n, int nocc, double occ, const double* c, int ldc, double* p,
                   cudaStream_t stream);

/* density_for_GPU (matrix/density_for_GPU.F90:16-130) with every occupation
 * it handles: ndubl doubly occupied MOs, MOs ndubl+1..nsingl holding fract
 * electrons, occ = 2 (RHF) or 1 (one spin of UHF); mode 2 forbids the
 * positron equivalent (:32).  iopc selects the reference's form: 2 or 3 the
 * two DGEMMs (2*sign*G2 + frac*sign*G1 + cst*I), 4 occ*C_d C_d^T, 5 that
 * below fract 0.01 and the explicit sums sign*(occ*G2 + frac*G1) + cst*I
 * above; 6 (no reference iopc) the explicit sums at any fract, which is
 * densit (matrix/densit.F90).  c: n x n column-major device matrix of all
 * MOs (ldc >= n); p: packed device output.  FP64 on the DMMA engine. */
int mb_density_occ_dev(int n, int ndubl, int nsingl, double occ, double fract, int mode, int iopc,
                       const double* c, int ldc, double* p, cudaStream_t stream);

/* Full eigensolve of a packed symmetric matrix after adding i*1e-10 to
 * diagonal element i (eigenvectors_LAPACK.F90:53-55; the packed input is
 * modified like the reference's xmat).  Ascending eigenvalues, vectors in
 * columns.  Returns MB_ERR_NUMERIC if the solver fails. */
int mb_eigh_packed_dev(int n, double* fpacked, double* c, double* eigs, cudaStream_t stream);
/* The same with a caller-owned workspace (mb_eigh_ws_bytes(n) bytes, 256-byte
 * aligned) and no host synchronisation: perturb = 1 adds the i*1e-10
 * diagonal; *status_dev (device int) is set nonzero if inverse iteration
 * fails. */
size_t mb_eigh_ws_bytes(int n);
int mb_eigh_ws(int n, double* fpacked, int perturb, double* c, double* eigs, void* ws, int* status_dev,
               cudaStream_t stream);

/* Pseudo-diagonalisation (diag_for_GPU.F90): Fmo = C_v^T F C_o and the
 * ordered 2x2 rotation sweep on C.  *nrot_out (host) gets the rotations
 * applied.  Bit-identical rotation arithmetic. */
int mb_pseudo_diag_dev(int n, int nocc, const double* fpacked, double* c, const double* eigs,
                       long long* nrot_out, cudaStream_t stream);

/* FP64 GEMM, column-major: C = alpha*op(A)*op(B) + beta*C. */
int mb_dgemm_dev(char transa, char transb, int m, int n, int k, double alpha, const double* a,
                 int lda, const double* b, int ldb, double beta, double* c, int ldc,
                 cudaStream_t stream);

/* ------------------------------------------------ learned initial guess
 * No counterpart in the reference (which starts from moldat.F90:731-760 or an
 * OLDENS density): an atom-pair MLP predicts each pair's density block in a
 * local frame from radial/angular descriptors within 6 A and each centre's
 * long-range electrostatic environment (reference charges).  Five pair types
 * (0 heavy atom's own block, 1 hydrogen's own block, 2 heavy-heavy,
 * 3 heavy-hydrogen, 4 hydrogen-hydrogen), each with its own network
 * DIN -> 128 -> 128 -> 128 -> 16 (SiLU), BF16 weights and activations, FP32
 * accumulation.  The parameter blob is NTYPES consecutive blocks of
 * MB_GUESS_PER_TYPE floats: in_mean[DIN], in_std[DIN], W1[128][DIN], b1[128],
 * W2[128][128], b2, W3[128][128], b3, W4[16][128], b4[16], out_mean[16],
 * out_std[16]. */
#define MB_GUESS_DIN 356
#define MB_GUESS_HID 128
#define MB_GUESS_DOUT 16
#define MB_GUESS_NTYPES 5
#define MB_GUESS_PER_TYPE 81528
typedef struct mb_guess_model mb_guess_model;
size_t mb_guess_blob_floats(void);
int mb_guess_model_create(const float* blob, mb_guess_model** out);
int mb_guess_model_destroy(mb_guess_model* model);
/* Predicts the context's starting density on the device (H and O only; other
 * elements return MB_ERR_UNSUPPORTED and the caller keeps the standard guess),
 * then applies purify_steps McWeeny purifications (1 recommended) with the
 * split-precision products of mb_guess_purify_split_dev.  Use with
 * opts.guess = 1. */
int mb_ctx_guess(mb_ctx* ctx, const mb_guess_model* model, int purify_steps);
/* McWeeny purification of a packed total density p (device, mpack): D = p/2,
 * D <- 3 D^2 - 2 D^3 steps times (FP64 GEMMs), p = 2 D.  It moves D's
 * eigenvalues towards 0 and 1, i.e. towards a closed-shell density, which
 * keeps iter's first density change small.  ws: mb_guess_purify_ws_bytes(n)
 * bytes of device scratch. */
size_t mb_guess_purify_ws_bytes(int n);
int mb_guess_purify_dev(int n, double* p, int steps, void* ws, cudaStream_t stream);
/* The same with both products of each step as three-product BF16 splits on
 * the tensor cores (mb_gemm_split_ws's accuracy, about 1e-5 of |A||B|; the
 * result only seeds the SCF).  tc_ws: mb_gemm_split_ws_bytes(n, n, n) bytes, 1024-byte aligned;
 * err_dev: device int, zeroed by the caller, nonzero after the stream is
 * synchronised if a tensor-core pipeline wait expired. */
int mb_guess_purify_split_dev(int n, double* p, int steps, void* ws, void* tc_ws, size_t tc_ws_bytes, int* err_dev,
                              cudaStream_t stream);
/* The steps, on device pointers.  Pairs: counts_host[NTYPES] receives the
 * per-type counts; with pf == NULL only counting is done; otherwise pf/ps/pt
 * (first atom, second atom, type) are filled type by type (order inside a
 * type is unspecified).  work: 15 ints of device scratch. */
int mb_guess_pairs_dev(int numat, const int* nat, const double* xyz, double rpair, int* counts_host,
                       int max_pairs, int* pf, int* ps, int* pt, int* work, cudaStream_t stream);
/* Frames (npairs x 9 doubles, axes as columns) and raw descriptors (npairs x
 * DIN floats).  ws: mb_guess_features_ws_bytes(numat) bytes of device scratch
 * (per-atom neighbour lists within 6 A, at most 512 per atom; more returns
 * MB_ERR_UNSUPPORTED).  Synchronises the stream. */
size_t mb_guess_features_ws_bytes(int numat);
int mb_guess_features_dev(int numat, const int* nat, const double* xyz, int npairs, const int* pf,
                          const int* ps, float* feat, double* frames, void* ws, cudaStream_t stream);
/* Raw descriptors -> normalised BF16 rows (uint16 bit patterns). */
int mb_guess_normalize_dev(const mb_guess_model* model, int type, int n, const float* raw,
                           unsigned short* x, cudaStream_t stream);
/* Raw local blocks -> normalised targets (unused slots 0). */
int mb_guess_norm_targets_dev(const mb_guess_model* model, int type, int n, const float* yraw,
                              float* yt, cudaStream_t stream);
/* Network of one type on n rows: y (n x 16, normalised).  ws: 2*n*128 BF16. */
int mb_guess_forward_dev(const mb_guess_model* model, int type, int n, const unsigned short* x,
                         float* y, void* ws, cudaStream_t stream);
/* Local blocks (network output) -> packed density p (pairs not listed are
 * left untouched); first (0-based) and nor per atom as in MbAtomsDev. */
int mb_guess_assemble_dev(const mb_guess_model* model, int npairs, const int* pf, const int* ps,
                          const int* pt, const double* frames, const float* y, const int* first,
                          const int* nor, double* p, cudaStream_t stream);
/* Training targets: each pair's block of a packed density in its frame (npairs x 16, raw). */
int mb_guess_targets_dev(int npairs, const int* pf, const int* ps, const int* pt,
                         const double* frames, const int* first, const int* nor, const double* p,
                         float* yraw, cudaStream_t stream);
/* All of the above for one molecule: p (mpack) is overwritten.  The _ws form
 * takes its buffers from a grow-only workspace (mb_guess_ws_create; contexts
 * keep one), the _dev form allocates and frees its own. */
typedef struct mb_guess_ws mb_guess_ws;
int mb_guess_ws_create(mb_guess_ws** out);
int mb_guess_ws_destroy(mb_guess_ws* ws);
int mb_guess_predict_density_ws(const mb_guess_model* model, int numat, const int* nat,
                                const double* xyz, const int* first, const int* nor, int norbs,
                                double* p, mb_guess_ws* ws, cudaStream_t stream);
int mb_guess_predict_density_dev(const mb_guess_model* model, int numat, const int* nat,
                                 const double* xyz, const int* first, const int* nor, int norbs,
                                 double* p, cudaStream_t stream);
/* Training on the device: FP32 master weights, BF16 copies for the GEMMs,
 * Adam.  mb_guess_trainer_model returns a model view of the current weights. */
typedef struct mb_guess_trainer mb_guess_trainer;
int mb_guess_trainer_create(const float* blob, int max_rows, mb_guess_trainer** out);
int mb_guess_trainer_destroy(mb_guess_trainer* trainer);
const mb_guess_model* mb_guess_trainer_model(mb_guess_trainer* trainer);
int mb_guess_trainer_set_norm(mb_guess_trainer* trainer, int type, const float* in_mean,
                              const float* in_std, const float* out_mean, const float* out_std);
/* Forward, MSE over the type's valid outputs, backward; update != 0 applies
 * an Adam step (lr).  loss_out (optional) synchronises and returns the loss. */
int mb_guess_trainer_step(mb_guess_trainer* trainer, int type, int n, const unsigned short* x,
                          const float* yt, float lr, int update, double* loss_out,
                          cudaStream_t stream);
/* Copies the parameter blob and the last step's gradients (same layout) to host. */
int mb_guess_trainer_get(mb_guess_trainer* trainer, float* params, float* grads);

/* ------------------------------------------- electronic-state exchange */
/* DENOUT / OLDENS density restart file, den_in_out (SCF/iter.F90:1133-1227):
 * one record "norbs, numat, pa(mpack)" with pa the alpha density (P/2 for a
 * closed shell); formatted = 0 writes gfortran's unformatted sequential
 * layout (4-byte length markers), 1 list-directed text (DENOUTF).  Reading
 * tries *formatted first (0 if formatted is NULL) and the other format
 * second; on return *formatted says which one was read.  A file for another
 * system fails with "Density file read in does not match current data set",
 * an unreadable one with "Density Restart File missing or corrupt". */
int mb_den_write(const char* path, int norbs, int numat, const double* pa, int formatted);
int mb_den_read(const char* path, int norbs, int numat, double* pa, int* formatted);
/* struct mopac_state (include/mopac.h:123-132) save and load,
 * mopac_save / mopac_load (interface/mopac_api_saveload.F90:26-78): save
 * gives mpack, uhf (0) and pa = P/2 of the context's current density (pa NULL:
 * size query); load makes pa the starting density of the next mb_scf_run with
 * opts.guess = 1 (mpack 0: nothing to load; a state of another size or a UHF
 * state: "Attempting to load incompatible MOPAC state"). */
int mb_ctx_save_state(mb_ctx* ctx, int* mpack, int* uhf, double* pa);
int mb_ctx_load_state(mb_ctx* ctx, int mpack, int uhf, const double* pa, const double* pb);

/* ------------------------------------- (1) reference bind(C) symbols */
/* src/gpu/cuda_wrappers.cu:192 (cublas_interfaces.F90:9-21) */
void call_gemm_cublas(char tra, char trb, int m, int n, int k, double alpha, const double* A,
                      int lda, const double* B, int ldb, double beta, double* C, int ldc);
/* src/gpu/cuda_wrappers.cu:229 */
void call_syrk_cublas(char uplo, char tra, int n, int k, double alpha, const double* A, int lda,
                      double beta, double* C, int ldc);
/* src/gpu/cuda_wrappers.cu:272, :372 -- one GPU here: same as the above */
void call_gemm_cublas_2gpu(char tra, char trb, int m, int n, int k, double alpha, const double* A,
                           int lda, const double* B, int ldb, double beta, double* C, int ldc);
void call_syrk_cublas_2gpu(char uplo, char tra, int n, int k, double alpha, const double* A,
                           int lda, double beta, double* C, int ldc);
/* src/gpu/cuda_wrappers.cu:469 (eigenvectors_cuda.F90:9-20): full symmetric
 * eigensolve, upper triangle of A (lda x n, column-major) on entry,
 * eigenvectors on exit, eigenvalues in W, info = 0 on success. */
void mopac_cuda_dsyevd(int n, double* A, int lda, double* W, int* info);
/* src/gpu/cuda_wrappers.cu:547: rotation sweep of diag_for_GPU; lumo is
 * 1-based; ci0/ca0 are unused (as in the reference). */
void call_rot_cuda_gpu(const double* fmo, const double* eig, double* vector, const double* ci0,
                       const double* ca0, int nocc, int lumo, int n, double bigeps, double tiny);
void call_rot_cuda_2gpu_gpu(const double* fmo, const double* eig, double* vector,
                            const double* ci0, const double* ca0, int nocc, int lumo, int n,
                            double bigeps, double tiny);
/* src/gpu/cuda_wrappers.cu:71, :115, :58, :158, :176, :830 */
void getGPUInfo(bool* hasGpu, bool* hasDouble, int* nDevices, char (*name)[256], int* name_size,
                size_t* totalMem, int* clockRate, int* major, int* minor);
void setDevice(int idevice, bool* stat);
void set_mozyme_gpu_pair(int dev0, int dev1);
void create_handle(void);
void destroy_handle(void);
void mopac_cuda_destroy_resources(void);

/* ------------------------------------------ (2) Fortran-level shims */
/* fock2(f, ptot, p, w, wj, wk, numat, nfirst, nlast, mode), SCF/fock2.F90:16;
 * host arrays, mode 2 only (fock1 included), numat > 0. */
void fock2_(double* f, const double* ptot, const double* p, const double* w, const double* wj,
            const double* wk, const int* numat, const int* nfirst, const int* nlast,
            const int* mode);
/* helect(n, p, h, f), integrals/helect.F90:16 */
double helect_(const int* n, const double* p, const double* h, const double* f);
/* dfock2(f, ptot, p, w, numat, nfirst, nlast, nati), forces/dfock2.F90:16
 * (called at forces/deri1.F90:107): the two-centre Fock-matrix derivative
 * of atom nati (1-based) added to f; host arrays, s and sp atoms. */
void dfock2_(double* f, const double* ptot, const double* p, const double* w, const int* numat,
             const int* nfirst, const int* nlast, const int* nati);
/* cnvg(pnew, p, p1, niter, pl), SCF/cnvg.F90:16 (RHF).  norbs comes from
 * molkst_C in the reference; a Fortran host sets it once with mb_set_norbs. */
void cnvg_(double* pnew, double* p, double* p1, const int* niter, double* pl);
void mb_set_norbs_(const int* norbs);
/* pulay(f, p, n, fppf, fock, emat, lfock, nfock, msize, start, pl),
 * SCF/pulay.F90:16; host arrays; start is a Fortran LOGICAL (4 bytes).
 * npulay comes from molkst_C in the reference (default 10, which this shim
 * assumes); a Fortran host with another value sets it with mb_set_npulay. */
void pulay_(double* f, const double* p, const int* n, double* fppf, double* fock, double* emat,
            int* lfock, int* nfock, const int* msize, int* start, double* pl);
void mb_set_npulay_(const int* npulay);
/* density_for_GPU(c, fract, ndubl, nsingl, occ, mpack, norbs, mode, pp, iopc),
 * matrix/density_for_GPU.F90:16: every occupation (closed shell, fractional,
 * one UHF spin) and every iopc it takes (2..5), through mb_density_occ_dev;
 * c holds all norbs MOs (the positron equivalent reads the virtual ones) */
void density_for_gpu_(const double* c, const double* fract, const int* ndubl, const int* nsingl,
                      const double* occ, const int* mpack, const int* norbs, const int* mode,
                      double* pp, const int* iopc);
/* eigenvectors_LAPACK(eigenvecs, xmat, eigvals, ndim),
 * matrix/eigenvectors_LAPACK.F90:16; modifies xmat like the reference */
void eigenvectors_lapack_(double* eigenvecs, double* xmat, double* eigvals, const int* ndim);
/* diag_for_GPU(fao, vector, nocc, eig, norbs, mpack), matrix/diag_for_GPU.F90:16 */
void diag_for_gpu_(const double* fao, double* vector, const int* nocc, const double* eig,
                   const int* norbs, const int* mpack);

/* MOZYME's routines read module MOZYME_C and common_arrays_C, which a C
 * library cannot see; the host registers them (by reference, Fortran-style),
 * then calls the shims with the reference's argument lists.  Each call stages
 * the registered host arrays through the device kernels and writes the
 * results back into them. */
/* After fillij and hcore_for_MOZYME: the atoms (iorbs, coord in Angstrom),
 * fillij's cutoffs (squared), H in pair blocks (mpack) and the stored pairs'
 * two-electron integrals (nw, the layout's order). */
int mb_mz_bind_system_(const int* numat, const int* iorbs, const double* coord, const double* cutof1,
                       const double* cutof2, const double* h, const double* w, const long long* nw);
/* Whenever the LMO arrays are (re)allocated or repacked: MOZYME_C's ncf,
 * nncf, icocc, ncocc, cocc and nce, nnce, icvir, ncvir, cvir with their
 * dimensions, common_arrays_C's p and eigs, and fmo_dim.  The pointers are
 * kept and read / written by the shims. */
int mb_mz_bind_lmos_(const int* nocc, int* ncf, int* nncf, int* icocc, int* ncocc, double* cocc,
                     const long long* icocc_dim, const long long* cocc_dim, const int* nvir, int* nce,
                     int* nnce, int* icvir, int* ncvir, double* cvir, const long long* icvir_dim,
                     const long long* cvir_dim, double* p, double* eigs, const long long* fmo_dim);
/* MOZYME_C's shift and thresh, read at every diagg_ call. */
int mb_mz_bind_controls_(const double* shift, const double* thresh);
/* density_for_MOZYME(p, mode, nclose_loc, partp), MOZYME/density_for_MOZYME.F90:16 */
void density_for_mozyme_(double* p, const int* mode, const int* nclose_loc, const double* partp);
/* buildf(f, partf, mode), MOZYME/buildf.F90:16; P is the registered p; mode 0
 * (whole F) only, other modes report MB_ERR_UNSUPPORTED */
void buildf_(double* f, const double* partf, const int* mode);
/* diagg(fao, nocc, nvir, idiagg, partp, indi), MOZYME/diagg.F90: diagg1,
 * diagg2 and density_for_MOZYME(p, indi, nocc, partp); diagg1's and diagg2's
 * saved state is kept by the library between calls */
void diagg_(const double* fao, const int* nocc, const int* nvir, const int* idiagg, double* partp,
            const int* indi);

#ifdef __cplusplus
}
#endif
#endif /* MOPAC_B200_H */
