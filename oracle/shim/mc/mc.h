/* Project-written empty stand-in for FETK's mc/mc.h (oracle build only).
 * The PMG solve path never uses the MC finite-element types; HAVE_MC is not
 * defined, so the reference headers only include this file unconditionally
 * from vclist.h. */
#ifndef ORACLE_MC_SHIM_H
#define ORACLE_MC_SHIM_H
#endif
