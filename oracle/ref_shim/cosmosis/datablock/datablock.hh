// Build shim (test infrastructure): an in-memory cosmosis::DataBlock with the
// members the reference's fixed-GL module headers use -- view<T>, get_val<T>,
// has_val, get_type and put_val.  Section and key names are case-insensitive,
// as in CosmoSIS (the reference reads omega_M and omega_m from one entry).
#ifndef Y3_REF_SHIM_DATABLOCK_HH
#define Y3_REF_SHIM_DATABLOCK_HH

#include "cosmosis/datablock/datablock_status.h"
#include "cosmosis/datablock/ndarray.hh"

#include <algorithm>
#include <cctype>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <variant>
#include <vector>

namespace cosmosis {

  class DataBlock {
  public:
    using value_t = std::variant<int,
                                 double,
                                 bool,
                                 std::string,
                                 std::vector<int>,
                                 std::vector<double>,
                                 ndarray<double>>;

    template <typename T>
    DATABLOCK_STATUS
    put_val(std::string const& section, std::string const& name, T const& v)
    {
      vals_[key_(section, name)] = value_t{v};
      return DBS_SUCCESS;
    }

    template <typename T>
    DATABLOCK_STATUS
    get_val(std::string const& section, std::string const& name, T& out) const
    {
      auto it = vals_.find(key_(section, name));
      if (it == vals_.end()) return DBS_NAME_NOT_FOUND;
      if (auto p = std::get_if<T>(&it->second)) {
        out = *p;
        return DBS_SUCCESS;
      }
      return DBS_WRONG_VALUE_TYPE;
    }

    template <typename T>
    T
    view(std::string const& section, std::string const& name) const
    {
      T out{};
      DATABLOCK_STATUS const s = get_val<T>(section, name, out);
      if (s != DBS_SUCCESS)
        throw std::runtime_error("DataBlock: cannot view " + section + "/" +
                                 name + " (" + datablock_status_str(s) + ")");
      return out;
    }

    bool
    has_val(std::string const& section, std::string const& name) const
    {
      return vals_.count(key_(section, name)) != 0;
    }

    DATABLOCK_STATUS
    get_type(std::string const& section,
             std::string const& name,
             datablock_type_t& t) const
    {
      auto it = vals_.find(key_(section, name));
      if (it == vals_.end()) return DBS_NAME_NOT_FOUND;
      static constexpr datablock_type_t kinds[] = {
        DBT_INT, DBT_DOUBLE, DBT_BOOL, DBT_STRING,
        DBT_INT1D, DBT_DOUBLE1D, DBT_DOUBLEND};
      t = kinds[it->second.index()];
      return DBS_SUCCESS;
    }

  private:
    static std::string
    lower_(std::string s)
    {
      std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) {
        return static_cast<char>(std::tolower(c));
      });
      return s;
    }
    static std::pair<std::string, std::string>
    key_(std::string const& section, std::string const& name)
    {
      return {lower_(section), lower_(name)};
    }

    std::map<std::pair<std::string, std::string>, value_t> vals_;
  };

} // namespace cosmosis

#endif
