/* Empty compile-environment stand-in for SuiteSparse's umfpack.h.
 * GEFEL/cc.cpp includes this header unconditionally, but every UMFPACK call
 * in that file sits under INC_CHMD, which the checker build never defines.
 * Test infrastructure only (used by oracle/build_ref.py). */
#ifndef SIFEL_REF_COMPAT_UMFPACK_H
#define SIFEL_REF_COMPAT_UMFPACK_H
#endif
