// datablock_shim.cpp -- a standalone in-memory DataBlock that implements the
// CosmoSIS C accessors the y3b modules call (y3b_cosmosis.h), plus the put /
// create functions a host needs to drive setup/execute/cleanup without
// CosmoSIS (the tests, or a sampler that embeds the modules directly).
// Section and key names are case-insensitive, as in CosmoSIS.
#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "y3b_cosmosis.h"

namespace {

enum Kind { kInt, kDouble, kString, kIntArr, kDoubleArr };

struct Value {
  Kind kind;
  int i = 0;
  double d = 0.0;
  std::string s;
  std::vector<int> ia;
  std::vector<double> da;
  std::vector<int> ext;  // for double arrays
};

struct Block {
  std::map<std::pair<std::string, std::string>, Value> v;
};

std::string
lower(const char* s)
{
  std::string o(s ? s : "");
  for (auto& c : o) c = (char)std::tolower((unsigned char)c);
  return o;
}

Value*
find(c_datablock* b, const char* sec, const char* name)
{
  auto* blk = static_cast<Block*>(b);
  if (!blk || !sec || !name) return nullptr;
  auto it = blk->v.find({lower(sec), lower(name)});
  return it == blk->v.end() ? nullptr : &it->second;
}

void
put(c_datablock* b, const char* sec, const char* name, Value val)
{
  static_cast<Block*>(b)->v[{lower(sec), lower(name)}] = std::move(val);
}

constexpr DATABLOCK_STATUS kNotFound = 4;
constexpr DATABLOCK_STATUS kWrongType = 5;

}  // namespace

extern "C" {
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

c_datablock*
y3b_datablock_new(void)
{
  return new Block();
}

void
y3b_datablock_free(c_datablock* b)
{
  delete static_cast<Block*>(b);
}

bool
c_datablock_has_value(c_datablock* s, const char* section, const char* name)
{
  return find(s, section, name) != nullptr;
}

DATABLOCK_STATUS
c_datablock_get_int(c_datablock* s, const char* section, const char* name, int* val)
{
  Value* v = find(s, section, name);
  if (!v) return kNotFound;
  if (v->kind != kInt) return kWrongType;
  *val = v->i;
  return DBS_SUCCESS;
}

DATABLOCK_STATUS
c_datablock_get_double(c_datablock* s, const char* section, const char* name, double* val)
{
  Value* v = find(s, section, name);
  if (!v) return kNotFound;
  if (v->kind == kDouble)
    *val = v->d;
  else if (v->kind == kInt)
    *val = v->i;
  else
    return kWrongType;
  return DBS_SUCCESS;
}

DATABLOCK_STATUS
c_datablock_get_string(c_datablock* s, const char* section, const char* name, char** val)
{
  Value* v = find(s, section, name);
  if (!v) return kNotFound;
  if (v->kind != kString) return kWrongType;
  *val = static_cast<char*>(std::malloc(v->s.size() + 1));
  std::memcpy(*val, v->s.c_str(), v->s.size() + 1);
  return DBS_SUCCESS;
}

DATABLOCK_STATUS
c_datablock_get_int_array_1d(c_datablock* s, const char* section, const char* name, int** val,
                             int* size)
{
  Value* v = find(s, section, name);
  if (!v) return kNotFound;
  if (v->kind != kIntArr) return kWrongType;
  *size = (int)v->ia.size();
  *val = static_cast<int*>(std::malloc(sizeof(int) * std::max<size_t>(1, v->ia.size())));
  std::copy(v->ia.begin(), v->ia.end(), *val);
  return DBS_SUCCESS;
}

DATABLOCK_STATUS
c_datablock_get_double_array_1d(c_datablock* s, const char* section, const char* name,
                                double** val, int* size)
{
  Value* v = find(s, section, name);
  if (!v) return kNotFound;
  if (v->kind != kDoubleArr || v->ext.size() != 1) return kWrongType;
  *size = (int)v->da.size();
  *val = static_cast<double*>(std::malloc(sizeof(double) * std::max<size_t>(1, v->da.size())));
  std::copy(v->da.begin(), v->da.end(), *val);
  return DBS_SUCCESS;
}

DATABLOCK_STATUS
c_datablock_get_array_ndim(c_datablock* s, const char* section, const char* name, int* ndim)
{
  Value* v = find(s, section, name);
  if (!v) return kNotFound;
  if (v->kind == kIntArr) {
    *ndim = 1;
    return DBS_SUCCESS;
  }
  if (v->kind != kDoubleArr) return kWrongType;
  *ndim = (int)v->ext.size();
  return DBS_SUCCESS;
}

DATABLOCK_STATUS
c_datablock_get_double_array_shape(c_datablock* s, const char* section, const char* name,
                                   int ndims, int* extents)
{
  Value* v = find(s, section, name);
  if (!v) return kNotFound;
  if (v->kind != kDoubleArr || (int)v->ext.size() != ndims) return kWrongType;
  for (int i = 0; i < ndims; ++i) extents[i] = v->ext[i];
  return DBS_SUCCESS;
}

DATABLOCK_STATUS
c_datablock_get_double_array(c_datablock* s, const char* section, const char* name,
                             double* val, int ndims, int* extents)
{
  Value* v = find(s, section, name);
  if (!v) return kNotFound;
  if (v->kind != kDoubleArr || (int)v->ext.size() != ndims) return kWrongType;
  for (int i = 0; i < ndims; ++i)
    if (extents[i] != v->ext[i]) return kWrongType;
  std::copy(v->da.begin(), v->da.end(), val);
  return DBS_SUCCESS;
}

DATABLOCK_STATUS
c_datablock_put_double_array_1d(c_datablock* s, const char* section, const char* name,
                                const double* val, int size)
{
  Value v;
  v.kind = kDoubleArr;
  v.da.assign(val, val + size);
  v.ext = {size};
  put(s, section, name, std::move(v));
  return DBS_SUCCESS;
}

DATABLOCK_STATUS
c_datablock_put_double_array(c_datablock* s, const char* section, const char* name,
                             const double* val, int ndims, const int* extents)
{
  Value v;
  v.kind = kDoubleArr;
  size_t n = 1;
  for (int i = 0; i < ndims; ++i) {
    v.ext.push_back(extents[i]);
    n *= (size_t)extents[i];
  }
  v.da.assign(val, val + n);
  put(s, section, name, std::move(v));
  return DBS_SUCCESS;
}

DATABLOCK_STATUS
c_datablock_put_int_array_1d(c_datablock* s, const char* section, const char* name,
                             const int* val, int size)
{
  Value v;
  v.kind = kIntArr;
  v.ia.assign(val, val + size);
  put(s, section, name, std::move(v));
  return DBS_SUCCESS;
}

DATABLOCK_STATUS
c_datablock_put_int(c_datablock* s, const char* section, const char* name, int val)
{
  Value v;
  v.kind = kInt;
  v.i = val;
  put(s, section, name, std::move(v));
  return DBS_SUCCESS;
}

DATABLOCK_STATUS
c_datablock_put_double(c_datablock* s, const char* section, const char* name, double val)
{
  Value v;
  v.kind = kDouble;
  v.d = val;
  put(s, section, name, std::move(v));
  return DBS_SUCCESS;
}

DATABLOCK_STATUS
c_datablock_put_string(c_datablock* s, const char* section, const char* name, const char* val)
{
  Value v;
  v.kind = kString;
  v.s = val ? val : "";
  put(s, section, name, std::move(v));
  return DBS_SUCCESS;
}

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
}
