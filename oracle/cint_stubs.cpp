// Link stubs for the libcint entry points src/AO_ints/ThreeCenterIntegrals.cpp references.  libcint is
// not in this image, so the integral generators cannot run; these abort if reached.  The oracle only
// calls the file's GEMM-only functions.
#include <cstdio>
#include <cstdlib>

extern "C" {
#include "cint.h"

static void no_libcint(const char* name) {
  std::fprintf(stderr, "oracle: %s needs libcint, which this build does not link\n", name);
  std::abort();
}

FINT CINTcgto_cart(const FINT, const FINT*) {
  no_libcint("CINTcgto_cart");
  return 0;
}
FINT cint3c2e_cart(double*, FINT*, FINT*, FINT, FINT*, FINT, double*, CINTOpt*) {
  no_libcint("cint3c2e_cart");
  return 0;
}
FINT cint2c2e_cart(double*, FINT*, FINT*, FINT, FINT*, FINT, double*, CINTOpt*) {
  no_libcint("cint2c2e_cart");
  return 0;
}
}
