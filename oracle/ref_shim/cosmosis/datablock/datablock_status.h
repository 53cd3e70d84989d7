/*
 * Build shim (test infrastructure): the status and type enumerations of the
 * CosmoSIS DataBlock C API, as far as the reference's fixed-GL module headers
 * use them.  Only the names matter to those headers; the values are this
 * shim's own.
 */
#ifndef Y3_REF_SHIM_DATABLOCK_STATUS_H
#define Y3_REF_SHIM_DATABLOCK_STATUS_H

typedef enum {
  DBS_SUCCESS = 0,
  DBS_DATABLOCK_NULL,
  DBS_SECTION_NULL,
  DBS_SECTION_NOT_FOUND,
  DBS_NAME_NULL,
  DBS_NAME_NOT_FOUND,
  DBS_NAME_ALREADY_EXISTS,
  DBS_VALUE_NULL,
  DBS_WRONG_VALUE_TYPE,
  DBS_MEMORY_ALLOC_FAILURE,
  DBS_SIZE_NULL,
  DBS_SIZE_NONPOSITIVE,
  DBS_SIZE_INSUFFICIENT,
  DBS_NDIM_NONPOSITIVE,
  DBS_NDIM_OVERFLOW,
  DBS_NDIM_MISMATCH,
  DBS_EXTENTS_NULL,
  DBS_EXTENTS_MISMATCH,
  DBS_LOGIC_ERROR,
  DBS_USED_DEFAULT
} DATABLOCK_STATUS;

typedef enum {
  DBT_INT,
  DBT_DOUBLE,
  DBT_COMPLEX,
  DBT_STRING,
  DBT_BOOL,
  DBT_INT1D,
  DBT_DOUBLE1D,
  DBT_COMPLEX1D,
  DBT_STRING1D,
  DBT_BOOL1D,
  DBT_INTND,
  DBT_DOUBLEND,
  DBT_COMPLEXND,
  DBT_UNKNOWN
} datablock_type_t;

#ifdef __cplusplus
extern "C" {
#endif
static inline const char* datablock_status_str(DATABLOCK_STATUS s)
{
  switch (s) {
    case DBS_SUCCESS: return "success";
    case DBS_SECTION_NOT_FOUND: return "section not found";
    case DBS_NAME_NOT_FOUND: return "name not found";
    case DBS_WRONG_VALUE_TYPE: return "wrong value type";
    default: return "datablock error";
  }
}
#ifdef __cplusplus
}
#endif

#endif
