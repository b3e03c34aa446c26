/* Project-written configuration header for the oracle build of the reference
 * PMG path (replaces the CMake-generated apbscfg.h).  Quiet mode, no FETK
 * components, no MPI. */
#ifndef ORACLE_APBSCFG_H
#define ORACLE_APBSCFG_H
#define PACKAGE_STRING "APBS 3.4.1 (reference oracle build)"
#define VAPBSQUIET 1
#define HAVE_TIME_FUNC 1
#define DOUBLE_EPSILON 2.2204460492503131e-16
#define FLOAT_EPSILON 1.1920928955078125e-07
#endif
