// Stand-in for the reference's xtensor-backed core/mat3.h, so that the
// reference's header-only PME math (pme_spline.h, pme_influence.h) compiles
// here without xtensor.  Only the element accessor those headers use.
// Test infrastructure: used by oracle/ref_build.sh only.
#pragma once
#include "atomiverse/core/precision.h"

namespace ATV {
class Mat3 {
  public:
    Mat3() {
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                m_[i][j] = 0.0;
    }
    AccReal& operator()(int i, int j) { return m_[i][j]; }
    const AccReal& operator()(int i, int j) const { return m_[i][j]; }

  private:
    AccReal m_[3][3];
};
} // namespace ATV
