// Build shim (test infrastructure): the reference's fixed-GL path includes the
// cubacpp headers only for type names of the retired adaptive integrators; a
// fixed-size array with element access is all those declarations need.
#ifndef Y3_REF_SHIM_CUBACPP_ARRAY_HH
#define Y3_REF_SHIM_CUBACPP_ARRAY_HH

#include <array>
#include <cstddef>

namespace cubacpp {
  template <std::size_t N>
  struct array {
    std::array<double, N> v{};
    double& operator[](std::size_t i) { return v[i]; }
    double const& operator[](std::size_t i) const { return v[i]; }
    static constexpr std::size_t size() { return N; }
  };
}

#endif
