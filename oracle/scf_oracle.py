"""CPU oracle for the PM7 dense SCF path (test infrastructure only).

Only tests/, __graft_entry__.smoke() and the CPU legs of bench.py may import
this module; the product package never does.  It is the checker, not the
thing measured or shipped.

What it restates:
  * ``iter`` (SCF/iter.F90:16-1107) for closed-shell RHF with the default
    keywords (no UHF, no C.I., id = 0), Camp-King optional (``camp``,
    oracle/campking_oracle.py, and iter's forced switch-on): level-shift control
    (:273-325), Fock build (:553), energy (:641-659), convergence test
    (:675-690), full diagonalisation (:849) or, in ``pseudo`` mode, the
    pseudo-diagonalisation the reference comments out (:847-861), density
    (:897), ``cnvg`` (:899-901) and the exit diagonalisation (:1052-1106);
  * ``eigenvectors_LAPACK`` (matrix/eigenvectors_LAPACK.F90:53-121): adds
    i*1e-10 to diagonal element i, then LAPACK dsyevd (numpy.linalg.eigh calls
    the same LAPACK driver);
  * ``density_for_GPU`` iopc 5 (matrix/density_for_GPU.F90:102-108):
    P = 2 C_occ C_occ^T;
  * ``diag_for_GPU`` (matrix/diag_for_GPU.F90:101-206): Fmo = C_v^T F C_o and
    the ordered 2x2 rotation sweep.
The integral, Fock, energy and extrapolation kernels live in the C part
(mopac_oracle.c) and are reached through ctypes.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

FPC9 = 23.060547830619029
EV = 27.211386245988


def build() -> str:
    """Compile the C oracle (gcc, -ffp-contract=off) into oracle/_build."""
    src = os.path.join(_HERE, "mopac_oracle.c")
    if (not os.path.exists(_LIB_PATH)) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        i32p = np.ctypeslib.ndpointer(np.int32, flags="C")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
        L.orc_layout.argtypes = [ctypes.c_int, i32p, i32p, i32p]
        L.orc_layout.restype = ctypes.c_int
        L.orc_n2elec.argtypes = [ctypes.c_int, i32p]
        L.orc_n2elec.restype = ctypes.c_longlong
        L.orc_hcore.argtypes = [ctypes.c_int, i32p, f64p, f64p, f64p, ctypes.POINTER(ctypes.c_double)]
        L.orc_fock2.argtypes = [ctypes.c_int, i32p, i32p, f64p, f64p, f64p, f64p]
        L.orc_helect.argtypes = [ctypes.c_int, f64p, f64p, f64p]
        L.orc_helect.restype = ctypes.c_double
        L.orc_cnvg.argtypes = [ctypes.c_int, f64p, f64p, f64p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.orc_pdiag.argtypes = [ctypes.c_int, i32p, f64p]
        L.orc_atheat.argtypes = [ctypes.c_int, i32p]
        L.orc_atheat.restype = ctypes.c_double
        L.orc_disp_pm7.argtypes = [ctypes.c_int, i32p, f64p]
        L.orc_disp_pm7.restype = ctypes.c_double
        L.orc_param.argtypes = [ctypes.c_int, ctypes.c_char_p]
        L.orc_param.restype = ctypes.c_double
        f64f = np.ctypeslib.ndpointer(np.float64, flags="F")
        L.orc_rot_sweep.argtypes = [ctypes.c_int, ctypes.c_int, f64f, f64p, f64f, ctypes.c_double, ctypes.c_double]
        L.orc_rot_sweep.restype = ctypes.c_longlong
        _lib = L
    return _lib


# ---------------------------------------------------------------- packing
def tri_index(n: int):
    """(row, col) of packed lower-triangle storage, row-major: i(i-1)/2 + j."""
    return np.tril_indices(n)


def unpack(p: np.ndarray, n: int) -> np.ndarray:
    a = np.zeros((n, n))
    r, c = tri_index(n)
    a[r, c] = p
    a[c, r] = p
    return a


def pack(a: np.ndarray) -> np.ndarray:
    r, c = tri_index(a.shape[0])
    return np.ascontiguousarray(a[r, c])


def diag_index(n: int) -> np.ndarray:
    i = np.arange(1, n + 1)
    return i * (i + 1) // 2 - 1


# ---------------------------------------------------------------- system
@dataclass
class System:
    nat: np.ndarray          # atomic numbers (int32)
    coord: np.ndarray        # (numat, 3) Angstrom
    nfirst: np.ndarray = field(default=None)  # 1-based
    nlast: np.ndarray = field(default=None)
    norbs: int = 0
    nclose: int = 0
    h: np.ndarray = field(default=None)
    w: np.ndarray = field(default=None)
    enuclr: float = 0.0
    atheat: float = 0.0
    pdiag: np.ndarray = field(default=None)

    @property
    def numat(self) -> int:
        return int(self.nat.shape[0])

    @property
    def mpack(self) -> int:
        return self.norbs * (self.norbs + 1) // 2


def make_system(nat, coord, integrals: bool = True) -> System:
    L = lib()
    nat = np.ascontiguousarray(nat, dtype=np.int32)
    coord = np.ascontiguousarray(coord, dtype=np.float64).reshape(-1, 3)
    n = nat.shape[0]
    nfirst = np.zeros(n, np.int32)
    nlast = np.zeros(n, np.int32)
    norbs = L.orc_layout(n, nat, nfirst, nlast)
    if norbs < 0:
        raise ValueError("oracle supports H, C and O only")
    tore = {1: 1, 6: 4, 8: 6}
    nelec = int(sum(tore[int(z)] for z in nat))
    if nelec % 2:
        raise ValueError("closed-shell RHF needs an even electron count")
    s = System(nat=nat, coord=coord, nfirst=nfirst, nlast=nlast, norbs=norbs, nclose=nelec // 2)
    s.pdiag = np.zeros(norbs)
    L.orc_pdiag(n, nat, s.pdiag)
    s.atheat = L.orc_atheat(n, nat)
    if integrals:
        hcore(s)
    return s


def hcore(s: System) -> None:
    L = lib()
    n2 = L.orc_n2elec(s.numat, s.nat)
    s.h = np.zeros(s.mpack)
    s.w = np.zeros(n2)
    e = ctypes.c_double(0.0)
    L.orc_hcore(s.numat, s.nat, s.coord.reshape(-1), s.h, s.w, ctypes.byref(e))
    s.enuclr = e.value


def fock2(s: System, f: np.ndarray, ptot: np.ndarray, pa: np.ndarray) -> None:
    lib().orc_fock2(s.numat, s.nfirst, s.nlast, f, ptot, pa, s.w)


def helect(n: int, p, h, f) -> float:
    return lib().orc_helect(n, p, h, f)


def cnvg(norbs: int, pnew, p, p1, niter: int) -> float:
    pl = ctypes.c_double(0.0)
    lib().orc_cnvg(norbs, pnew, p, p1, niter, ctypes.byref(pl))
    return pl.value


def disp_correction(s: System) -> float:
    return lib().orc_disp_pm7(s.numat, s.nat, s.coord.reshape(-1))


def eigenvectors_lapack(f: np.ndarray, n: int):
    """eigenvectors_LAPACK.F90:53-121; perturbs f in place like the reference."""
    f[diag_index(n)] += np.arange(1, n + 1) * 1.0e-10
    a = unpack(f, n)
    w, v = np.linalg.eigh(a, UPLO="U")
    return np.asfortranarray(v), w


def density(c: np.ndarray, nclose: int) -> np.ndarray:
    co = c[:, :nclose]
    return pack(2.0 * (co @ co.T))


def density_for_gpu(c: np.ndarray, fract: float, ndubl: int, nsingl: int, occ: float, mode: int,
                    iopc: int) -> np.ndarray:
    """matrix/density_for_GPU.F90:16-130 (iopc 2..5) and matrix/densit.F90
    (iopc 6 here: the explicit sums at any fract).  c: (norbs, norbs), column
    k = MO k.  Returns the packed lower triangle (= dtrttp('u') of the
    symmetric result)."""
    n = c.shape[0]
    if iopc == 4 or (iopc == 5 and fract < 1.0e-2):           # :96-106 (dsyrk)
        cd = c[:, :ndubl]
        return pack(occ * (cd @ cd.T))
    if ndubl != 0 and nsingl > n // 2 and mode != 2:           # :32-43 positron equivalent
        sign, frac, cst = -1.0, occ - fract, occ
        nl2, nu2, nl1, nu1 = nsingl + 1, n, ndubl + 1, nsingl
    else:                                                      # :44-54 electron equivalent
        sign, frac, cst = 1.0, fract, 0.0
        nl2, nu2, nl1, nu1 = 1, ndubl, ndubl + 1, nsingl
    c2 = c[:, nl2 - 1:nu2] if nu2 >= nl2 else c[:, :0]
    c1 = c[:, nl1 - 1:nu1] if nu1 >= nl1 else c[:, :0]
    g2, g1 = c2 @ c2.T, c1 @ c1.T
    if iopc in (2, 3):                                         # :57-87 (two dgemm)
        x = (2.0 * sign) * g2
        x = (frac * sign) * g1 + x
    else:                                                      # :107-124, densit.F90:37-48
        x = (occ * g2 + g1 * frac) * sign
    x[np.diag_indices(n)] = cst + x[np.diag_indices(n)]
    return pack(x)


def fmo_block(f: np.ndarray, c: np.ndarray, nocc: int) -> np.ndarray:
    """diag_for_GPU.F90:101-150: Fmo (nvirt x nocc) = C_v^T F C_o."""
    n = c.shape[0]
    F = unpack(f, n)
    if nocc < n - nocc:
        return c[:, nocc:].T @ (F @ c[:, :nocc])
    return (F @ c[:, nocc:]).T @ c[:, :nocc]


def rotation_sweep(c: np.ndarray, fmo: np.ndarray, eig: np.ndarray, nocc: int,
                   bigeps: float = 1.5e-7, tiny: float | None = None) -> int:
    """diag_for_GPU.F90:151-206 (CPU branch) in C (orc_rot_sweep): the same
    rotations in the same order as ``rotation_sweep_py``, bit for bit, with
    the rows of c split over threads.  c must be Fortran-ordered (n x n)."""
    if tiny is None:
        tiny = float(np.max(np.abs(fmo))) * 0.05
    assert c.flags.f_contiguous and c.dtype == np.float64
    fmo = np.asfortranarray(fmo, dtype=np.float64)
    eig = np.ascontiguousarray(eig, dtype=np.float64)
    return int(lib().orc_rot_sweep(c.shape[0], nocc, fmo, eig, c, float(bigeps), float(tiny)))


def rotation_sweep_py(c: np.ndarray, fmo: np.ndarray, eig: np.ndarray, nocc: int,
                      bigeps: float = 1.5e-7, tiny: float | None = None) -> int:
    """diag_for_GPU.F90:151-206 (CPU branch).  Rotates columns of c in place in
    the reference order (occupied i outer, virtual j inner); returns the count
    of rotations applied."""
    n = c.shape[0]
    if tiny is None:
        tiny = float(np.max(np.abs(fmo))) * 0.05
    done = 0
    for i in range(nocc):
        for jv in range(n - nocc):
            x = fmo[jv, i]
            if abs(x) < tiny:
                continue
            a = eig[i]
            b = eig[nocc + jv]
            d = a - b
            if abs(x / d) < bigeps:
                continue
            e = np.copysign(np.sqrt(4.0 * x * x + d * d), d)
            alpha = np.sqrt(0.5 * (1.0 + d / e))
            beta = -np.copysign(np.sqrt(1.0 - alpha * alpha), x)
            ci = c[:, i].copy()
            cj = c[:, nocc + jv].copy()
            c[:, i] = alpha * ci + beta * cj
            c[:, nocc + jv] = alpha * cj - beta * ci
            done += 1
    return done


def pseudo_diag(f, c, nocc, eig, bigeps: float = 1.5e-7, tiny: float | None = None):
    fmo = fmo_block(f, c, nocc)
    return rotation_sweep(c, fmo, eig, nocc, bigeps=bigeps, tiny=tiny)


# ---------------------------------------------------------------- pulay
def osinv(a: np.ndarray, n: int):
    """matrix/osinv.F90: in-place Gauss-Jordan inverse with full pivoting of
    the column-major n x n matrix stored flat in a; returns the clamped
    determinant d (0 when a pivot falls below 1e-8)."""
    tol = 1.0e-8
    d = 1.0
    L = [0] * (n + 1)
    M = [0] * (n + 1)
    A = a  # 1-based helper below
    def g(i):
        return A[i - 1]
    def s_(i, v):
        A[i - 1] = v
    nk = -n
    for k in range(1, n + 1):
        nk = nk + n
        L[k] = k
        M[k] = k
        kk = nk + k
        biga = g(kk)
        for j in range(k, n + 1):
            iz = n * (j - 1)
            for i in range(k, n + 1):
                ij = iz + i
                if abs(biga) - abs(g(ij)) >= 0.0:
                    continue
                biga = g(ij)
                L[k] = i
                M[k] = j
        j = L[k]
        if j - k > 0:
            ki = k - n
            for i in range(1, n + 1):
                ki = ki + n
                holo = -g(ki)
                ji = ki - k + j
                s_(ki, g(ji))
                s_(ji, holo)
        i = M[k]
        if i - k > 0:
            jp = n * (i - 1)
            for j in range(1, n + 1):
                jk = nk + j
                ji = jp + j
                holo = -g(jk)
                s_(jk, g(ji))
                s_(ji, holo)
        if abs(biga) - tol < 0.0:
            return 0.0
        for i in range(1, n + 1):
            if i - k == 0:
                continue
            ik = nk + i
            s_(ik, g(ik) / (-biga))
        for i in range(1, n + 1):
            ik = nk + i
            ij = i - n
            if i - k != 0:
                for j in range(1, n + 1):
                    ij = ij + n
                    if j - k == 0:
                        continue
                    kj = ij - i + k
                    s_(ij, g(ik) * g(kj) + g(ij))
        kj = k - n
        for j in range(1, n + 1):
            kj = kj + n
            if j - k == 0:
                continue
            s_(kj, g(kj) / biga)
        d = min(d * biga, 1.0e10)
        s_(kk, 1.0 / biga)
    k = n
    while True:
        k = k - 1
        if k <= 0:
            break
        i = L[k]
        if i - k > 0:
            jq = n * (k - 1)
            jr = n * (i - 1)
            for j in range(1, n + 1):
                jk = jq + j
                holo = g(jk)
                ji = jr + j
                s_(jk, -g(ji))
                s_(ji, holo)
        j = M[k]
        if j - k <= 0:
            continue
        ki = k - n
        for i in range(1, n + 1):
            ki = ki + n
            holo = g(ki)
            ji = ki + j - k
            s_(ki, -g(ji))
            s_(ji, holo)
    return d


class PulayState:
    """Storage iter hands to pulay (SCF/pulay.F90:16).  As in the reference
    (setup_mopac_arrays.F90:148, iter.F90:826-831) the commutator history is
    ``pold`` and the Fock history is ``pold2``, both npulay*mpack long: slot l
    of the commutators is the planar block fppf[l*linear:(l+1)*linear], entry
    i of Fock slot l sits at fock[l + i*mfock] (interleaved).  iter's cnvg
    uses the first mpack (resp. norbs) elements of the same two arrays."""

    def __init__(self, n: int, npulay: int = 10):
        self.n = n
        self.linear = n * (n + 1) // 2
        self.mfock = npulay
        self.fppf = np.zeros(npulay * self.linear)
        self.fock = np.zeros(npulay * self.linear)
        self.emat = np.zeros((npulay + 1, npulay + 1))
        self.start = True
        self.lfock = 0
        self.nfock = 0


def commutator_packed(p: np.ndarray, f: np.ndarray, n: int) -> np.ndarray:
    """sym_commute + pack_matrix (SCF/pulay.F90:219-247, 181-191): M = P F,
    element (i, j), i <= j, becomes M(i, j) - M(j, i), packed 'U' by columns
    (the same index as MOPAC's lower-triangle-by-rows layout)."""
    P = unpack(p, n)
    F = unpack(f, n)
    m = P @ F
    r, c = tri_index(n)          # r >= c: packed slot of (row c, col r) in 'U'
    return np.ascontiguousarray(m[c, r] - m[r, c])


def pulay(st: PulayState, f: np.ndarray, p: np.ndarray):
    """SCF/pulay.F90:16-180.  f is replaced by the extrapolated Fock matrix
    when at least two entries are stored; returns pl = |[P,F]|^2 / linear."""
    lin = st.linear
    if st.start:
        st.nfock = 1
        st.lfock = 1
        st.start = False
    else:
        if st.nfock < st.mfock:
            st.nfock += 1
        st.lfock = st.lfock + 1 if st.lfock != st.mfock else 1
    l0 = st.lfock - 1
    st.fock[l0::st.mfock][:lin] = f[:lin]
    st.fppf[l0 * lin:(l0 + 1) * lin] = commutator_packed(p, f, st.n)
    nf = st.nfock
    e = st.emat
    cur = st.fppf[l0 * lin:(l0 + 1) * lin]
    for i in range(nf):
        e[nf, i] = -1.0
        e[i, nf] = -1.0
        e[l0, i] = float(np.dot(st.fppf[i * lin:(i + 1) * lin], cur))
        e[i, l0] = e[l0, i]
    pl = e[l0, l0] / lin
    e[nf, nf] = 0.0
    if e[l0, l0] < 1.0e-20:
        return pl
    const = 1.0 / e[l0, l0]
    e[:nf, :nf] *= const
    ev = list(e[:nf + 1, :nf + 1].ravel())   # row i of emat -> column i of evec
    const = 1.0 / const
    e[:nf, :nf] *= const
    d = osinv(ev, nf + 1)
    if abs(d) < 1.0e-6:
        st.start = True
        return pl
    if nf < 2:
        return pl
    il = nf * (nf + 1)
    coeffs = [-ev[il + j] for j in range(nf)]
    hist = st.fock[:lin * st.mfock].reshape(lin, st.mfock)
    out = np.zeros(lin)
    for j in range(nf):
        out = out + coeffs[j] * hist[:, j]
    f[:lin] = out
    return pl


# ---------------------------------------------------------------- iter
@dataclass
class ScfResult:
    escf: float             # heat of formation from iter, kcal/mol (no post-SCF terms)
    ee: float               # electronic energy, eV
    eigs: np.ndarray
    c: np.ndarray
    p: np.ndarray
    niter: int
    converged: bool
    history: list
    n_finish: int = 0
    n_interp: int = 0       # interpolated iterations (Camp-King's mode 3)
    forced_on: bool = False  # iter forced all convergers on (niter > itrmax - 10)


def iter_scf(s: System, pseudo: bool = False, scfcrt: float = 1.0e-4, itrmax: int = 2000,
             gnorm: float = 0.0, trace: bool = False, pulay_on: bool = False,
             p_guess: np.ndarray | None = None, finish_dp: float = 0.0,
             finish_max: int = 40, shift_kw: float | None = None, camp: bool = False) -> ScfResult:
    """Closed-shell restatement of iter (SCF/iter.F90), 1SCF settings
    (last = 1, nscf = 0, fulscf = .true.).

    p_guess: a starting total density (packed).  It enters like a density
    read with OLDENS (iter.F90:151-158: pa = p/2, pold = 2*pa); pold2, which
    that branch leaves as allocated, starts as the diagonal of p.

    shift_kw: the SHIFT=n keyword (iter.F90:131-136): bshift = -n; SHIFT=0
    switches the level shift off and allows newdg from the first iteration.

    finish_dp > 0 adds the FP64 finish of the device SCF (mb_scf_opts
    finish_dp): once iter's test (:675-690) passes, convergence is accepted
    only when the last density update moved no element of P by more than
    finish_dp (max|P_k - P_(k-1)| over all mpack elements); otherwise the
    loop goes on, at most finish_max more iterations, and in those
    iterations the rotation sweep's relative threshold bigeps
    (diag_for_GPU.F90:33) and its absolute one, tiny = 0.05 max|Fmo|
    (:151-152), are both 0: every occupied-virtual pair is rotated.

    camp: the CAMP keyword (iter.F90:134): Camp-King's interp on the alpha
    vectors from the third iteration (:781-798), a full diagonalisation in
    every iteration, and an interpolated iteration (interp's mode 3) neither
    counts nor tests convergence (:342-343, :662) and skips Pulay, the
    diagonalisation and cnvg (:800, :888).  Without it iter still forces all
    convergers on when niter passes itrmax - 10 (:351-372): Pulay and
    Camp-King on, a constant shift (bshift = 4.44), iredy = -4, and the
    iteration count restarts.  The pseudo-diagonalisation takes its rotation angles from
    the orbital energies of the last full diagonalisation, which carry that
    iteration's level shift (-8 eV on the virtuals with Pulay); at its first
    iteration the finish replaces them by the energies of the current
    vectors, diag(C^T F C).  With finish_dp = 0 this is iter unchanged."""
    n = s.norbs
    mpack = s.mpack
    nclose = s.nclose
    h, w = s.h, s.w
    enrgy = FPC9
    # -- first-call setup (iter.F90:123-221) --
    shift = 1.0
    shfmax = 20.0
    newdg = False
    plchek = 0.005
    pl = 1.0
    bshift = -80.0 if shift_kw is None else -float(shift_kw)
    ten = bshift
    tenold = ten
    shfto = 0.0
    shftbo = 0.0
    shiftb = 0.0
    oknewd = abs(bshift) < 0.001
    okpuly = pulay_on
    pst = PulayState(s.norbs) if pulay_on else None
    halfe = False
    camkin = bool(camp)
    allcon = okpuly or camkin           # iter.F90:142
    modea = 1 if camkin else 0          # label 180 (:322-330)
    ck = None                           # interp's state, made on its first call
    trans = 0.2
    na1el = nclose
    nb1el = nclose
    ihomo = max(1, nclose)
    p = np.zeros(mpack)
    pa = np.zeros(mpack)
    w1 = na1el / (na1el + 1.0e-6 + nb1el)
    random = 1.0
    dix = diag_index(n)
    for i in range(n):
        j = dix[i]
        p[j] = s.pdiag[i]
        pa[j] = p[j] * w1 * random
        random = 1.0 / random
    if p_guess is not None:
        p = np.array(p_guess, dtype=np.float64)
        pa = p * 0.5
    if p_guess is not None and pst is None:
        pold = pa * 2.0
        pold2 = pold[dix].copy()
    elif pst is not None:
        # pold and pold2 are the heads of pulay's two history arrays
        pold = pst.fppf[:mpack]
        pold[:] = pa if p_guess is None else pa * 2.0
        pold2 = pst.fock[:n]
        pold2[:] = pold[dix]
    else:
        pold = pa.copy()
        pold2 = pold[dix].copy()
    gs = True
    selcon = scfcrt
    if gs:
        selcon = min(min(scfcrt * 100.0, 0.1), max(scfcrt * gnorm ** 3, scfcrt))
    pltest = 0.05 * np.sqrt(abs(selcon))
    iredy = 1
    niter = 0
    eold = 1.0e2
    ready = False
    diff = 0.0
    scorr = 0.0
    eigs = np.zeros(n)
    c = np.zeros((n, n), order="F")
    history = []
    ramp = np.arange(1, mpack + 1) * 1.0e-16
    f = None
    converged = False
    dp = np.inf          # max|P_k - P_(k-1)| of the last density update
    n_finish = 0         # iterations the finish added after iter's test passed
    refreshed = False    # orbital energies refreshed for the finish
    n_interp = 0                        # interpolated passes (interp mode 3)
    forced_on = False
    while True:  # label 250
        incitr = modea != 3
        if incitr:
            niter += 1
        if niter > itrmax:
            break
        if niter > itrmax - 10 and not allcon:
            # SWITCH ON ALL CONVERGERS (:351-372), then label 180
            okpuly = True
            camkin = not halfe
            allcon = True
            bshift = 4.44
            iredy = -4
            eold = 100.0
            newdg = False
            if pst is None:
                # pulay's histories start at pold and pold2 (the same arrays
                # in the reference): carry cnvg's heads over
                pst = PulayState(s.norbs)
                pst.fppf[:mpack] = pold
                pst.fock[:n] = pold2
                pold = pst.fppf[:mpack]
                pold2 = pst.fock[:n]
            pst.start = True
            niter = 0
            modea = 1 if camkin else 0
            forced_on = True
            if trace:
                history.append(dict(niter=0, escf=None, pl=pl, shift=shift, newdg=newdg, allcon=True))
            continue
        if abs(shift) > 1.0e-10 and bshift != 0.0:
            if niter > 1:
                if newdg and not (halfe or camkin):
                    if diff > 0.0:
                        shift = 1.0
                        if diff > 1:
                            newdg = False
                    else:
                        shift = -0.1
                else:
                    if ihomo < n:
                        shift = ten + eigs[ihomo] - eigs[ihomo - 1] + shift
                    else:
                        shift = 0.0
                if diff > 0.0:
                    if shift > 4.0:
                        shfmax = 4.5
                    if shift > shfmax:
                        shfmax = max(shfmax - 0.5, 0.0)
                shift = max(-20.0, min(shfmax, shift))
                if abs(shift - shfmax) < 1.0e-5:
                    shfmax = shfmax + 0.01
                if okpuly or abs(bshift - 4.44) < 1.0e-5:
                    shift = -8.0
                    if newdg:
                        shift = 0.0
            tenold = ten
            if pl > plchek:
                shftbo = shiftb
                shfto = shift
            else:
                shiftb = shftbo
                shift = shfto
            eigs[ihomo:] = eigs[ihomo:] + shift
            f = h + shift * pa + ramp
            f[dix] = f[dix] - shift
        else:
            f = h.copy()
        while True:  # label 320
            fock2(s, f, p, pa)
            ee = helect(n, pa, h, f) * 2.0
            escf = (ee + s.enuclr) * enrgy + s.atheat + scorr
            if not incitr:      # an interpolated point: no energy test (:662)
                break
            diff = escf - eold
            if diff > 0:
                ten = ten - 1.0
            else:
                ten = ten * 0.975 + 0.05
            sellim = max(selcon, 1.0e-15 * max(abs(ee), 1.0))
            conv = niter > 4 and (pl == 0.0 or (pl < pltest and abs(diff) < sellim)) and ready
            if conv and finish_dp > 0.0 and dp > finish_dp and n_finish < finish_max:
                n_finish += 1
                conv = False
            if conv:
                if abs(shift) < 1.0e-10:
                    converged = True
                    break
                shift = 0.0
                shiftb = 0.0
                f = h.copy()
                continue
            break
        if converged:
            break
        if incitr:
            ready = iredy > 0 and (abs(diff) < sellim * 10.0 or pl == 0.0)
            iredy += 1
            eold = escf
        if trace:
            history.append(dict(niter=niter, escf=escf, pl=pl, shift=shift, newdg=newdg, mode=modea))
        if niter > 2 and camkin:        # :781-798 (makea is always true for RHF)
            if ck is None:
                from oracle.campking_oracle import CampKing
                ck = CampKing(n)
            modea = ck.interp(na1el, n - na1el, modea, escf / enrgy, f, c)
            if modea == 3:
                n_interp += 1
        p_before = p
        if modea == 3:                  # interpolated vectors: no Pulay, no diagonalisation, no cnvg
            p = density(c, nclose)
            dp = float(np.max(np.abs(p - p_before)))
            pa = p * 0.5
            oknewd = pl < sellim or oknewd
            newdg = (pl < trans and oknewd) or newdg
            if pl < trans * 0.3333:
                oknewd = True
            continue
        if newdg and okpuly and iredy > 1:
            pl = pulay(pst, f, pa)
        if newdg and pseudo and not (halfe or camkin):
            if n_finish > 0 and not refreshed:
                # the finish refreshes the orbital energies the rotation
                # angles use: eigs from the last full diagonalisation carry
                # that iteration's level shift
                eigs = np.einsum("ij,ij->j", c, unpack(f, n) @ c)
                refreshed = True
            if n_finish > 0:    # the finish rotates every occupied-virtual pair
                pseudo_diag(f, c, na1el, eigs, bigeps=0.0, tiny=0.0)
            else:
                pseudo_diag(f, c, na1el, eigs)
        else:
            c, eigs = eigenvectors_lapack(f, n)
        p = density(c, nclose)
        if not (newdg and okpuly):
            pl = cnvg(n, p, pold, pold2, niter)
        dp = float(np.max(np.abs(p - p_before)))
        pa = p * 0.5
        oknewd = pl < sellim or oknewd
        newdg = (pl < trans and oknewd) or newdg
        if pl < trans * 0.3333:
            oknewd = True
    # -- label 600 --
    ee = helect(n, pa, h, f) * 2.0
    fcopy = f.copy()
    c, eigs = eigenvectors_lapack(fcopy, n)
    escf = (ee + s.enuclr) * enrgy + s.atheat
    return ScfResult(escf=escf, ee=ee, eigs=eigs, c=c, p=p, niter=niter, converged=converged,
                     history=history, n_finish=n_finish, n_interp=n_interp, forced_on=forced_on)


def exit_block_diag(f: np.ndarray, c: np.ndarray, nocc: int, tol_ev: float = 1.0e-8):
    """The device SCF's exit diagonalisation after the FP64 finish (an
    addition to iter's label 600, which calls eigenvectors_LAPACK on the whole
    F): F gets the reference's perturbation i * 1e-10 (in place, as
    eigenvectors_lapack does), M = C^T F C is split into its occupied and
    virtual diagonal blocks, each block is diagonalised, and the first-order
    rotation X = B' / (e_o - e_v) with B' = Q_v^T B Q_o, B = M[nocc:, :nocc],
    takes the remaining coupling out of the vectors.  Returns (c, eigs,
    ||B||_F), or (None, None, ||B||_F) when the eigenvalue bound
    ||B||_F^2 / gap exceeds tol_ev and the whole matrix must be solved."""
    n = c.shape[0]
    f[diag_index(n)] += np.arange(1, n + 1) * 1.0e-10
    ff = unpack(f, n)
    m = c.T @ (ff @ c)
    b = m[nocc:, :nocc]
    b2 = float(np.sum(b * b))
    if not b2 <= tol_ev * 1.0e3:
        return None, None, np.sqrt(b2)
    ea, qa = np.linalg.eigh(0.5 * (m[:nocc, :nocc] + m[:nocc, :nocc].T))
    ed, qd = np.linalg.eigh(0.5 * (m[nocc:, nocc:] + m[nocc:, nocc:].T))
    gap = ed[0] - ea[-1]
    if not (gap > 0.0 and b2 <= tol_ev * gap):
        return None, None, np.sqrt(b2)
    x = (qd.T @ b @ qa) / (ea[None, :] - ed[:, None])
    co = c[:, :nocc] @ qa
    cv = c[:, nocc:] @ qd
    cn = np.hstack([co + cv @ x, cv - co @ x.T])
    return np.asfortranarray(cn), np.concatenate([ea, ed]), np.sqrt(b2)


# ---------------------------------------------------------------- fixed point
def roothaan_step(s: System, p: np.ndarray):
    """One plain SCF step from the total density p: F(p) = H + fock2
    (iter.F90:553), the heat at p (:641-659), the full diagonalisation with
    the reference's perturbation (eigenvectors_LAPACK.F90:53-121) and the
    closed-shell density of its eigenvectors (density_for_GPU.F90:102-108).
    Returns (new density, eigenvalues of F(p), heat of formation at p)."""
    f = s.h.copy()
    fock2(s, f, p, p * 0.5)
    ee = helect(s.norbs, p * 0.5, s.h, f) * 2.0
    heat = (ee + s.enuclr) * FPC9 + s.atheat
    c, e = eigenvectors_lapack(f, s.norbs)
    return density(c, s.nclose), e, heat


def fixed_point_certificate(s: System, p: np.ndarray, steps: int = 3) -> dict:
    """How far a density p is from the oracle's self-consistent point P*.

    Runs ``steps`` plain steps P_k = T(P_(k-1)) from P_0 = p and records
    r_k = max|P_k - P_(k-1)|.  Near P* the step is a contraction with factor
    rho (estimated as the largest r_(k+1)/r_k), so max|p - P*| <= r_1/(1 - rho);
    for water clusters rho is about 0.6 and the bound matches the true
    distance to within a few percent.  Also returns the orbital energies of
    F(p) (what iter's exit diagonalisation gives for a converged p) and the
    heat at p and at P_steps."""
    rs, heats = [], []
    pk = p
    eigs0 = None
    for k in range(steps):
        pn, e, heat = roothaan_step(s, pk)
        if k == 0:
            eigs0 = e
        heats.append(heat)
        rs.append(float(np.max(np.abs(pn - pk))))
        pk = pn
    ratios = [rs[k + 1] / rs[k] for k in range(len(rs) - 1) if rs[k] > 0.0]
    rho = max(ratios) if ratios else 0.0
    bound = rs[0] / (1.0 - rho) if rho < 1.0 else float("inf")
    return dict(r=rs, rho=rho, bound=bound, eigs=eigs0, heat_at_p=heats[0], heat_last=heats[-1], p_last=pk)


# ---------------------------------------------------------------- gradients
def _pair_system(nat2, xyz2) -> System:
    """The two atoms alone (electron count not checked: dhc's diatomic need
    not be closed shell)."""
    L = lib()
    nat2 = np.ascontiguousarray(nat2, dtype=np.int32)
    xyz2 = np.ascontiguousarray(xyz2, dtype=np.float64).reshape(2, 3)
    nfirst, nlast = np.zeros(2, np.int32), np.zeros(2, np.int32)
    norbs = L.orc_layout(2, nat2, nfirst, nlast)
    s = System(nat=nat2, coord=xyz2, nfirst=nfirst, nlast=nlast, norbs=norbs, nclose=0)
    hcore(s)
    return s


def _pair_energy(nat2, x1, x2, p_loc, pa_loc) -> float:
    """forces/dhc.F90 for a molecule, RHF: the diatomic's energy with its
    density blocks fixed.  Built from the whole two-atom system, so it also
    holds the one-centre terms; those do not depend on the geometry and drop
    out of every difference dcart takes."""
    s = _pair_system(nat2, np.vstack([x1, x2]))
    f = s.h.copy()
    fock2(s, f, p_loc, pa_loc)
    return 2.0 * helect(s.norbs, pa_loc, s.h, f) + s.enuclr


def dcart(s: System, p: np.ndarray) -> np.ndarray:
    """forces/dcart.F90:60-300 for a molecule (id = 0), RHF, the default
    finite difference (no FORCE keyword): for every pair (ii, jj), jj < ii,
    atom jj moves chnge/2 along all three axes (:283-286), then atom ii moves
    chnge along each axis in turn (:292-296); deriv = (aa - ee) fpc_9 / chnge
    (:297) is subtracted from ii's gradient and added to jj's.  Returns
    (numat, 3) kcal/mol/A, accumulated in the reference's order."""
    chnge = 1.0e-4
    chnge2 = chnge * 0.5
    n = s.numat
    P = unpack(p, s.norbs)
    dxyz = np.zeros((n, 3))
    for ii in range(n):
        for jj in range(ii):
            idx = np.concatenate([np.arange(s.nfirst[jj] - 1, s.nlast[jj]),
                                  np.arange(s.nfirst[ii] - 1, s.nlast[ii])])
            p_loc = pack(P[np.ix_(idx, idx)])
            pa_loc = 0.5 * p_loc
            nat2 = s.nat[[jj, ii]]
            x1 = s.coord[jj] + chnge2
            x2 = s.coord[ii].copy()
            aa = _pair_energy(nat2, x1, x2, p_loc, pa_loc)
            for k in range(3):
                x2[k] = x2[k] + chnge
                ee = _pair_energy(nat2, x1, x2, p_loc, pa_loc)
                x2[k] = x2[k] - chnge2
                x2[k] = x2[k] - chnge2
                deriv = (aa - ee) * FPC9 / chnge
                dxyz[ii, k] = dxyz[ii, k] - deriv
                dxyz[jj, k] = dxyz[jj, k] + deriv
    return dxyz


# ---------------------------------------------------------------- properties
def mulliken_charges(s: System, p: np.ndarray) -> np.ndarray:
    """NDDO net charges: core charge minus the diagonal density on the atom."""
    tore = {1: 1.0, 6: 4.0, 8: 6.0}
    pd = p[diag_index(s.norbs)]
    q = np.zeros(s.numat)
    for a in range(s.numat):
        q[a] = tore[int(s.nat[a])] - pd[s.nfirst[a] - 1:s.nlast[a]].sum()
    return q


def heat_of_formation(s: System, res: ScfResult) -> float:
    """Final heat = iter's escf + the PM7 post-SCF dispersion term (compfg)."""
    return res.escf + disp_correction(s)
