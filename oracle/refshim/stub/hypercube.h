// Minimal stand-in for SEP's hypercube.h, enough for the reference's
// operator/src/complex_vector.h to compile (it only names the type in the
// make_complex_vector declaration, which the shim does not call).
// Test infrastructure for the oracle's reference-kernel shim only.
#pragma once
#include <memory>
#include <vector>

namespace SEP {
struct axis {
  int n = 1;
  float o = 0.f, d = 1.f;
};
class hypercube {
 public:
  hypercube() = default;
  explicit hypercube(const std::vector<axis>& ax) : axes_(ax) {}
  axis getAxis(int i) const { return axes_[i - 1]; }
  std::vector<axis> getAxes() const { return axes_; }
  int getNdim() const { return (int)axes_.size(); }
  long long getN123() const {
    long long n = 1;
    for (const auto& a : axes_) n *= a.n;
    return n;
  }

 private:
  std::vector<axis> axes_;
};
}  // namespace SEP
