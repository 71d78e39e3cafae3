/* Links the reference's own objects against the portable exp/log/cbrt of the CUDA build
 * (inria-internship-project-sw2d-enzyme_b200/csrc/portable_math.h): with
 * -Wl,--wrap=exp,--wrap=log(,--wrap=cbrt) every call the reference makes to them lands here.  The
 * reference sources are not modified; only the libm they are linked with changes.
 * TEST INFRASTRUCTURE (oracle/_ref/libsw2d_ref_pm.so). */
#include "../inria-internship-project-sw2d-enzyme_b200/csrc/portable_math.h"

double __wrap_exp(double x) { return sw2d_exp(x); }
double __wrap_log(double x) { return sw2d_log(x); }
double __wrap_cbrt(double x) { return sw2d_cbrt(x); }
