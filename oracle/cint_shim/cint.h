/* Compile-only stand-in for libcint's header, for building src/AO_ints/ThreeCenterIntegrals.cpp into the
 * oracle without libcint (absent from this image).  Only the names that file uses are declared; the
 * numeric values are arbitrary placeholders, NOT libcint's, because nothing that reaches libcint is
 * ever called: the oracle uses the file's GEMM-only functions (transformRiThreeCenterAoLegs), and
 * oracle/cint_stubs.cpp makes every libcint entry point abort if it were reached. */
#ifndef RR_ORACLE_CINT_SHIM_H
#define RR_ORACLE_CINT_SHIM_H

typedef int FINT;
typedef struct RrOracleCintOpt CINTOpt;

enum {
  CHARGE_OF = 0, PTR_COORD = 1, ATOM_OF = 0, ANG_OF = 1, NPRIM_OF = 2, NCTR_OF = 3, PTR_EXP = 5, PTR_COEFF = 6,
  ATM_SLOTS = 6, BAS_SLOTS = 8, PTR_ENV_START = 20
};

FINT CINTcgto_cart(const FINT bas_id, const FINT* bas);

#endif
