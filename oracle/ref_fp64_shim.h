// Forced-include shim for the FP64 oracle build of the reference library.
// The reference's drnum.h defines FR12/FR13/FR14/FR23/GLOBAL_EPS/MAX_REAL/MIN_REAL
// only in its single-precision branch (drnum.h:62-70); its double branch
// (drnum.h:72-81) leaves them undefined although fluxes/ausmplus.h:47 and
// reconstruction/vanalbada.h:31 use them.  The values below are the ones of the
// single-precision branch, so both precisions evaluate the same expressions.
// Test infrastructure only.
#ifndef DN_ORACLE_FP64_SHIM_H
#define DN_ORACLE_FP64_SHIM_H
#define MAX_REAL numeric_limits<real>::max()
#define MIN_REAL numeric_limits<real>::min()
#define FR12 real(0.5)
#define FR13 real(0.3333333)
#define FR14 real(0.25)
#define FR23 real(0.6666666)
#define GLOBAL_EPS real(1e-10)
#endif
