// Electronic-state exchange with stock MOPAC: density restart files and the
// C API's state record.
//
//  * mb_den_write / mb_den_read restate den_in_out (SCF/iter.F90:1133-1227),
//    the DENOUT / OLDENS file: one sequential record "norbs, numat, pa(mpack)"
//    (pa = the alpha density, P/2 for a closed shell), unformatted by default
//    (gfortran's layout: a 4-byte little-endian length before and after the
//    record) or list-directed text with DENOUTF.  Reading tries the format
//    asked for first and the other one second, like the reference; a file
//    for another system fails with the reference's message, and so does a
//    missing or corrupt one.
//  * mb_ctx_save_state / mb_ctx_load_state mirror mopac_save / mopac_load
//    (interface/mopac_api_saveload.F90:26-78) for struct mopac_state
//    (include/mopac.h:123-132): mpack, uhf, pa, pb.  Loading a state is the
//    API's OLDENS: the next mb_scf_run with opts.guess = 1 starts from it.
//
// Host code only (no kernels); the context functions copy through the
// context's density buffers.
#include <ctype.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "mb_common.cuh"

extern "C" int mb_ctx_get_density(mb_ctx* c, double* p);
extern "C" int mb_ctx_set_guess(mb_ctx* c, const double* p);
extern "C" int mb_ctx_norbs(const mb_ctx* c);

namespace {

// Record payload size limit of one gfortran record without subrecords.
constexpr long long kMaxRecord = 2147483647LL;

int write_unformatted(FILE* f, int norbs, int numat, const double* pa, long long mpack) {
  const long long bytes = 8 + 8 * mpack;
  if (bytes > kMaxRecord)
    return mb_set_error(MB_ERR_UNSUPPORTED, "mb_den_write: density record above 2 GiB (gfortran subrecords)");
  const int32_t marker = (int32_t)bytes;
  const int32_t hdr[2] = {norbs, numat};
  if (fwrite(&marker, 4, 1, f) != 1 || fwrite(hdr, 4, 2, f) != 2 ||
      fwrite(pa, 8, (size_t)mpack, f) != (size_t)mpack || fwrite(&marker, 4, 1, f) != 1)
    return mb_set_error(MB_ERR_ARG, "mb_den_write: write failed");
  return MB_OK;
}

int write_formatted(FILE* f, int norbs, int numat, const double* pa, long long mpack) {
  if (fprintf(f, " %12d %12d\n", norbs, numat) < 0) return mb_set_error(MB_ERR_ARG, "mb_den_write: write failed");
  for (long long i = 0; i < mpack; ++i) {
    // 17 significant digits: the value reads back bit for bit
    if (fprintf(f, " %24.17E%s", pa[i], (i % 3 == 2 || i == mpack - 1) ? "\n" : "") < 0)
      return mb_set_error(MB_ERR_ARG, "mb_den_write: write failed");
  }
  return MB_OK;
}

// Readers return 0 when the file is not in their format, 1 when the header
// (norbs, numat) was read but the densities were not (short record), 2 when
// everything was read.  Like the Fortran read, the header comes first.
int read_unformatted(const std::vector<unsigned char>& buf, long long mpack, int* norbs, int* numat, double* pa) {
  if (buf.size() < 16) return 0;
  int32_t m1 = 0;
  memcpy(&m1, buf.data(), 4);
  if (m1 < 8 || (size_t)m1 + 8 > buf.size()) return 0;
  int32_t m2 = 0;
  memcpy(&m2, buf.data() + 4 + m1, 4);
  if (m2 != m1) return 0;
  int32_t hdr[2];
  memcpy(hdr, buf.data() + 4, 8);
  *norbs = hdr[0];
  *numat = hdr[1];
  // Fortran reads mpack values out of the record: the record must hold them
  if ((long long)m1 < 8 + 8 * mpack) return 1;
  memcpy(pa, buf.data() + 12, 8 * (size_t)mpack);
  return 2;
}

// One list-directed value: handles Fortran's D exponent and r*c repeats.
struct ListReader {
  const char* p;
  const char* end;
  double rep_val = 0.0;
  long long rep_left = 0;
  bool next(double* v) {
    if (rep_left > 0) {
      --rep_left;
      *v = rep_val;
      return true;
    }
    while (p < end && (isspace((unsigned char)*p) || *p == ',')) ++p;
    if (p >= end) return false;
    const char* s = p;
    while (p < end && !isspace((unsigned char)*p) && *p != ',') ++p;
    std::string tok(s, p);
    for (char& ch : tok)
      if (ch == 'd' || ch == 'D') ch = 'E';
    size_t star = tok.find('*');
    if (star != std::string::npos) {
      char* e1 = nullptr;
      long long r = strtoll(tok.c_str(), &e1, 10);
      if (e1 != tok.c_str() + star || r <= 0) return false;
      char* e2 = nullptr;
      double val = strtod(tok.c_str() + star + 1, &e2);
      if (*e2 != '\0') return false;
      rep_val = val;
      rep_left = r - 1;
      *v = val;
      return true;
    }
    char* e = nullptr;
    *v = strtod(tok.c_str(), &e);
    return *e == '\0' && !tok.empty();
  }
};

int read_formatted(const std::vector<unsigned char>& buf, long long mpack, int* norbs, int* numat, double* pa) {
  ListReader r{(const char*)buf.data(), (const char*)buf.data() + buf.size()};
  double a = 0.0, b = 0.0;
  if (!r.next(&a) || !r.next(&b)) return 0;
  if (a != (double)(long long)a || b != (double)(long long)b) return 0;
  *norbs = (int)a;
  *numat = (int)b;
  for (long long i = 0; i < mpack; ++i)
    if (!r.next(&pa[i])) return 1;
  return 2;
}

}  // namespace

extern "C" int mb_den_write(const char* path, int norbs, int numat, const double* pa, int formatted) {
  if (!path || norbs <= 0 || numat <= 0 || !pa) return mb_set_error(MB_ERR_ARG, "mb_den_write: bad args");
  const long long mpack = (long long)norbs * (norbs + 1) / 2;
  FILE* f = fopen(path, formatted ? "w" : "wb");
  if (!f) return mb_set_error(MB_ERR_ARG, "mb_den_write: cannot open the density file");
  int rc = formatted ? write_formatted(f, norbs, numat, pa, mpack) : write_unformatted(f, norbs, numat, pa, mpack);
  if (fclose(f) != 0 && rc == MB_OK) rc = mb_set_error(MB_ERR_ARG, "mb_den_write: close failed");
  return rc;
}

// Reads pa (mpack = norbs(norbs+1)/2 values) for a system of norbs orbitals
// and numat atoms.  *formatted (optional): in, the format to try first
// (0 unformatted, 1 text); out, the one that was read.
extern "C" int mb_den_read(const char* path, int norbs, int numat, double* pa, int* formatted) {
  if (!path || norbs <= 0 || numat <= 0 || !pa) return mb_set_error(MB_ERR_ARG, "mb_den_read: bad args");
  const long long mpack = (long long)norbs * (norbs + 1) / 2;
  std::vector<unsigned char> buf;
  {
    FILE* f = fopen(path, "rb");
    if (!f) return mb_set_error(MB_ERR_ARG, "Density Restart File missing or corrupt");
    unsigned char chunk[1 << 16];
    size_t got;
    while ((got = fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + got);
    fclose(f);
  }
  int want = formatted ? *formatted : 0;
  std::vector<double> tmp((size_t)mpack);
  for (int attempt = 0; attempt < 2; ++attempt) {
    const int fmt = attempt == 0 ? want : !want;
    int on = 0, oa = 0;
    const int got = fmt ? read_formatted(buf, mpack, &on, &oa, tmp.data())
                        : read_unformatted(buf, mpack, &on, &oa, tmp.data());
    if (got == 0) continue;
    // den_in_out compares the sizes (for plausible header values) before it
    // looks at the read status
    if (on > 0 && on < 100000 && (on != norbs || oa != numat))
      return mb_set_error(MB_ERR_ARG, "Density file read in does not match current data set");
    if (got == 1) continue;
    memcpy(pa, tmp.data(), sizeof(double) * (size_t)mpack);
    if (formatted) *formatted = fmt;
    return MB_OK;
  }
  return mb_set_error(MB_ERR_ARG, "Density Restart File missing or corrupt");
}

// mopac_save: the context's current density as the alpha density P/2.
// pa may be NULL to query mpack.
extern "C" int mb_ctx_save_state(mb_ctx* c, int* mpack, int* uhf, double* pa) {
  if (!c || !mpack) return mb_set_error(MB_ERR_ARG, "mb_ctx_save_state: bad args");
  const int n = mb_ctx_norbs(c);
  *mpack = (int)((long long)n * (n + 1) / 2);
  if (uhf) *uhf = 0;
  if (!pa) return MB_OK;
  MB_TRY(mb_ctx_get_density(c, pa));
  for (int i = 0; i < *mpack; ++i) pa[i] *= 0.5;
  return MB_OK;
}

// mopac_load: a saved state becomes the starting density (opts.guess = 1).
extern "C" int mb_ctx_load_state(mb_ctx* c, int mpack, int uhf, const double* pa, const double* pb) {
  if (!c) return mb_set_error(MB_ERR_ARG, "mb_ctx_load_state: null context");
  const int n = mb_ctx_norbs(c);
  if (mpack <= 0) return MB_OK;  // no state: the standard guess stays
  if (mpack != (int)((long long)n * (n + 1) / 2) || uhf != 0)
    return mb_set_error(MB_ERR_ARG, "Attempting to load incompatible MOPAC state");
  if (!pa) return mb_set_error(MB_ERR_ARG, "mb_ctx_load_state: null pa");
  (void)pb;
  std::vector<double> p((size_t)mpack);
  for (int i = 0; i < mpack; ++i) p[i] = pa[i] * 2.0;
  return mb_ctx_set_guess(c, p.data());
}
