// Build shim (test infrastructure): an n-dimensional row-major array with the
// members the reference's fixed-GL headers call on cosmosis::ndarray<T>
// (extents(), begin()/end(), size()).
#ifndef Y3_REF_SHIM_NDARRAY_HH
#define Y3_REF_SHIM_NDARRAY_HH

#include <cstddef>
#include <stdexcept>
#include <vector>

namespace cosmosis {

  template <typename T>
  class ndarray {
  public:
    ndarray() = default;
    ndarray(std::vector<T> vals, std::vector<std::size_t> extents)
      : vals_(std::move(vals)), extents_(std::move(extents))
    {
      std::size_t n = 1;
      for (auto e : extents_) n *= e;
      if (n != vals_.size())
        throw std::logic_error("ndarray: extents do not match the value count");
    }
    ndarray(T const* data, int ndims, int const* extents)
    {
      std::size_t n = 1;
      for (int d = 0; d != ndims; ++d) {
        extents_.push_back(static_cast<std::size_t>(extents[d]));
        n *= static_cast<std::size_t>(extents[d]);
      }
      vals_.assign(data, data + n);
    }

    std::vector<std::size_t> const& extents() const { return extents_; }
    std::size_t ndims() const { return extents_.size(); }
    std::size_t size() const { return vals_.size(); }
    T const* data() const { return vals_.data(); }
    auto begin() const { return vals_.cbegin(); }
    auto end() const { return vals_.cend(); }

  private:
    std::vector<T> vals_;
    std::vector<std::size_t> extents_;
  };

} // namespace cosmosis

#endif
