/* A plain-C client of libmopac_b200.so through include/mopac_b200.h only, the
 * way a Fortran host's iso_c_binding interfaces reach it: library version,
 * error reporting, and a DENOUT -> OLDENS density file round trip (host-only
 * entry points, so it runs without a GPU).  Exit code 0 on success. */
#include <stdio.h>
#include <string.h>

#include "mopac_b200.h"

int main(int argc, char** argv) {
  const char* path = argc > 1 ? argv[1] : "c_abi_client.den";
  if (mb_version() < 100) return 1;
  enum { NORBS = 6, NUMAT = 3, MPACK = NORBS * (NORBS + 1) / 2 };
  double pa[MPACK], back[MPACK];
  for (int i = 0; i < MPACK; ++i) pa[i] = 0.01 * (i + 1) - 0.1;
  for (int formatted = 0; formatted < 2; ++formatted) {
    if (mb_den_write(path, NORBS, NUMAT, pa, formatted) != MB_OK) {
      fprintf(stderr, "write: %s\n", mb_last_error());
      return 2;
    }
    int fmt = 0;
    if (mb_den_read(path, NORBS, NUMAT, back, &fmt) != MB_OK || fmt != formatted) {
      fprintf(stderr, "read: %s\n", mb_last_error());
      return 3;
    }
    if (memcmp(pa, back, sizeof(pa)) != 0) return 4;
  }
  /* a file for another system is refused with the reference's message */
  if (mb_den_read(path, NORBS + 1, NUMAT, back, NULL) != MB_ERR_ARG) return 5;
  if (strstr(mb_last_error(), "does not match current data set") == NULL) return 6;
  printf("c_abi_client ok\n");
  return 0;
}
