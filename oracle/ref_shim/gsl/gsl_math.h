/* Build shim (test infrastructure): the reference includes this header for
 * declarations it does not use on the fixed-grid path. */
#ifndef Y3_REF_SHIM_GSL_MATH_H
#define Y3_REF_SHIM_GSL_MATH_H
#include <math.h>
#endif
