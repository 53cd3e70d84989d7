// Build shim (test infrastructure): fmt::format for the "{}" placeholders the
// reference's table-file name helpers use (string and arithmetic arguments).
#ifndef Y3_REF_SHIM_FMT_CORE_H
#define Y3_REF_SHIM_FMT_CORE_H

#include <sstream>
#include <string>

namespace fmt {

  namespace shim_detail {
    inline void
    fill(std::ostringstream& os, std::string const& f, std::size_t pos)
    {
      os << f.substr(pos);
    }

    template <typename A, typename... R>
    void
    fill(std::ostringstream& os,
         std::string const& f,
         std::size_t pos,
         A const& a,
         R const&... rest)
    {
      std::size_t const at = f.find("{}", pos);
      if (at == std::string::npos) {
        os << f.substr(pos);
        return;
      }
      os << f.substr(pos, at - pos) << a;
      fill(os, f, at + 2, rest...);
    }
  }

  template <typename... A>
  std::string
  format(std::string const& f, A const&... args)
  {
    std::ostringstream os;
    shim_detail::fill(os, f, 0, args...);
    return os.str();
  }

} // namespace fmt

#endif
