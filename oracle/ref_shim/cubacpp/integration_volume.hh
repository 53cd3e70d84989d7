// Build shim (test infrastructure): the IntegrationVolume type name, which the
// reference's headers name in declarations of the retired adaptive modules.
// The fixed-GL path never constructs one.
#ifndef Y3_REF_SHIM_CUBACPP_INTEGRATION_VOLUME_HH
#define Y3_REF_SHIM_CUBACPP_INTEGRATION_VOLUME_HH

#include "cubacpp/array.hh"

#include <cstddef>

namespace cubacpp {
  template <std::size_t N>
  struct IntegrationVolume {
    IntegrationVolume() = default;
    IntegrationVolume(array<N> const& lo, array<N> const& hi)
      : lows(lo), highs(hi)
    {}
    array<N> lows{};
    array<N> highs{};
  };
}

#endif
