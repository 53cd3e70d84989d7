/* Build shim (test infrastructure): the reference includes this header but
 * uses none of its names on the fixed-GL path. */
#ifndef Y3_REF_SHIM_SECTION_NAMES_H
#define Y3_REF_SHIM_SECTION_NAMES_H
#define COSMOLOGICAL_PARAMETERS_SECTION "cosmological_parameters"
#define DISTANCES_SECTION "distances"
#define MASS_FUNCTION_SECTION "mass_function"
#endif
