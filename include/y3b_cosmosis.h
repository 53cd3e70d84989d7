/*
 * y3b_cosmosis.h -- the CosmoSIS module boundary of the y3b engine.
 *
 * Each of NumCountsSel.so, Shear1hMisSel.so, NumCountsFastMass.so and
 * Shear1hFastMass.so exports the three symbols that CosmoSIS dlopen()s, with
 * the reference's module labels, ini keys and DataBlock sections:
 *
 *   setup    replaces DEFINE_COSMOSIS_SCALAR_EVALUATOR_MODULE's setup,
 *            src/utils/module_macros.hh:79-83 (NumCounts.cc:14-19,
 *            Shear1hMis.cc:20-25): reads the module section (label) --
 *            bin_index, zt_low, zt_high, lnm_low, lnm_high, n_lnm (96),
 *            n_z (64); shear adds r_perp, lob_centers, method, stencil_h.
 *            Returns NULL on failure (the reference prints and returns a
 *            half-built module, CosmoSISScalarEvaluatorModule.hh:67-79).
 *   execute  replaces module_macros.hh:85-91 and
 *            CosmoSISScalarEvaluatorModule.hh:111-136: set_sample + evaluate
 *            over the grid, then put <output>/vals.  Returns 0 on success and
 *            a non-zero DATABLOCK_STATUS on any failure; it never throws
 *            (the reference always returns DBS_SUCCESS and lets
 *            std::out_of_range cross the C boundary).
 *   cleanup  replaces module_macros.hh:93-98; returns 0.
 *
 * With the option engine = fused in its section, a number-count module
 * (NumCountsSel.so / NumCountsFastMass.so) computes the whole integral
 * itself -- the lambda_t / lambda_obs / z_obs stage that sel_function.py
 * tabulates into S_stack included -- on the engine's fixed nested
 * Gauss-Legendre nodes (y3b_engine_eval, one parameter point per execute),
 * in precision = mixed (default) or fp64.  It then reads the sel_function
 * options (lam_min, lam_max, zob_min, zob_max, sigma_z per bin; from its own
 * section or the sel_function section), the lognormal MOR from
 * cluster_mor/{A, B, C, sigma_intr, M_pivot} and P(lambda_obs | lambda_true)
 * from the plob_ltr_params section (the default projection table when absent), and
 * with write_s_stack = T also writes sel_function/{lnM, z, S_stack}.
 *
 * The DataBlock is CosmoSIS's opaque c_datablock.  The modules call only the
 * C accessors declared below, which the host process provides at load time
 * (libcosmosis inside CosmoSIS; libdatablock_shim.so in the tests).
 */
#ifndef Y3B_COSMOSIS_H
#define Y3B_COSMOSIS_H

#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef void c_datablock;
typedef int DATABLOCK_STATUS;
#define DBS_SUCCESS 0

/* Module entry points (one set per module .so). */
void* setup(c_datablock* options);
DATABLOCK_STATUS execute(c_datablock* block, void* module);
int cleanup(void* module);

/* CosmoSIS C DataBlock accessors used by the modules (resolved from the host
 * process).  Arrays returned through pointer-to-pointer arguments are malloc()ed. */
bool c_datablock_has_value(c_datablock* s, const char* section, const char* name);
DATABLOCK_STATUS c_datablock_get_int(c_datablock* s, const char* section,
                                     const char* name, int* val);
DATABLOCK_STATUS c_datablock_get_double(c_datablock* s, const char* section,
                                        const char* name, double* val);
DATABLOCK_STATUS c_datablock_get_string(c_datablock* s, const char* section,
                                        const char* name, char** val);
DATABLOCK_STATUS c_datablock_get_int_array_1d(c_datablock* s, const char* section,
                                              const char* name, int** val, int* size);
DATABLOCK_STATUS c_datablock_get_double_array_1d(c_datablock* s, const char* section,
                                                 const char* name, double** val,
                                                 int* size);
DATABLOCK_STATUS c_datablock_get_array_ndim(c_datablock* s, const char* section,
                                            const char* name, int* ndim);
DATABLOCK_STATUS c_datablock_get_double_array_shape(c_datablock* s, const char* section,
                                                    const char* name, int ndims,
                                                    int* extents);
DATABLOCK_STATUS c_datablock_get_double_array(c_datablock* s, const char* section,
                                              const char* name, double* val, int ndims,
                                              int* extents);
DATABLOCK_STATUS c_datablock_put_double_array_1d(c_datablock* s, const char* section,
                                                 const char* name, const double* val,
                                                 int size);
DATABLOCK_STATUS c_datablock_put_double_array(c_datablock* s, const char* section,
                                              const char* name, const double* val,
                                              int ndims, const int* extents);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif
