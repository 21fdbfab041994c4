/*
 * Minimal CFITSIO stand-in used ONLY to compile mappraiser.c into the test
 * oracle.  NOT product code.  MLmap (mappraiser/src/mappraiser.c:336-342)
 * hands its I/Q/U/Cond/Hits maps to write_map(); the oracle's write_map
 * (shim_fits.c) stores them as raw native-endian arrays so tests can read them.
 */
#ifndef ORACLE_SHIM_FITSIO_H
#define ORACLE_SHIM_FITSIO_H
#define TINT    31
#define TLONG   41
#define TDOUBLE 82
#define TSTRING 16
#endif
