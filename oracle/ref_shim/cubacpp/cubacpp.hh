// Build shim (test infrastructure): the adaptive integrators of cubacpp
// (Cuhre, Vegas) by name only.  The reference headers compiled here declare
// adaptive modules next to the fixed-grid classes this build drives; those
// modules are never constructed, and integrate() refuses to run.
#ifndef Y3_REF_SHIM_CUBACPP_HH
#define Y3_REF_SHIM_CUBACPP_HH

#include "cubacpp/integration_volume.hh"

#include <stdexcept>
#include <vector>

namespace cubacpp {
  struct integration_result {
    std::vector<double> value, error, prob;
    long long neval = 0;
    int nregions = 0, status = -1;
  };

  struct shim_algorithm {
    long long maxeval = 0;
    template <typename F, typename V>
    integration_result
    integrate(F const&, double, double, V const&) const
    {
      throw std::logic_error("cubacpp adaptive integration is not part of this build");
    }
  };
  struct Cuhre : shim_algorithm {};
  struct Vegas : shim_algorithm {};
}

#endif
