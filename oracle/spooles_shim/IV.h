/* Declaration-only stand-in for the SPOOLES header IV.h (the SPOOLES
 * sources are not available).  The sparse-Schur path that needs SPOOLES is
 * never taken for problems with nBlock <= 5 or m <= 100; every entry point
 * is stubbed in spooles_stub.cpp and aborts if reached. */
#include "spooles_types.h"
