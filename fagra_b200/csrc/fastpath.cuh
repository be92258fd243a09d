// Specialized reduced operator for BAL-shaped Schur systems (retained width 9,
// eliminated width 3). Placeholder until the single-pass kernel lands: the
// generic two-kernel operator is used while enabled() is false.
#pragma once
#include "kernels.cuh"

namespace fg {

template <class TS>
struct FastPath {
  bool on = false;
  bool enabled() const { return on; }
  void invalidate() { on = false; }
  template <class Impl>
  fg_status prepare(Impl&) {
    return FG_OK;
  }
  template <class Impl, class TV>
  fg_status apply(Impl&, PView<TV>, double, TV*, double*, PcgState*) {
    return FG_OK;
  }
};

}  // namespace fg
