// Source time functions evaluated on the host in double precision with the
// expressions of SourceTimeFunction::operator() (cpp/src/sim/description.cpp:88-113),
// so that the per-step amplitudes (real_t)stf(step * dt) equal the reference's.
#pragma once

#include <cmath>
#include <cstddef>

#include "../../include/insem_cuda.h"

namespace insem_b200 {

inline double stf_value(const insem_cuda_stf& s, double t) {
  constexpr double kPi = 3.14159265358979323846;
  switch (s.kind) {
    case INSEM_STF_RICKER: {
      const double x = kPi * s.f0 * (t - s.t0);
      const double a = x * x;
      return s.amplitude * (1.0 - 2.0 * a) * std::exp(-a);
    }
    case INSEM_STF_GAUSSIAN: {
      const double x = kPi * s.f0 * (t - s.t0);
      const double a = x * x;
      return s.amplitude * std::exp(-a);
    }
    case INSEM_STF_GAUSSIAN_DERIVATIVE: {
      const double tau = t - s.t0;
      const double y = kPi * s.f0;
      const double c = y * y;
      return s.amplitude * (-2.0 * c * tau) * std::exp(-c * tau * tau);
    }
    case INSEM_STF_SAMPLES: {
      if (s.n_samples <= 0 || s.samples == nullptr) return 0.0;
      const double x = t / s.sample_dt;
      if (x < 0.0 || x > static_cast<double>(s.n_samples - 1)) return 0.0;
      const auto i = static_cast<std::size_t>(x);
      if (i + 1 >= static_cast<std::size_t>(s.n_samples)) return s.amplitude * s.samples[s.n_samples - 1];
      const double w = x - static_cast<double>(i);
      return s.amplitude * ((1.0 - w) * s.samples[i] + w * s.samples[i + 1]);
    }
    default:
      return 0.0;
  }
}

}  // namespace insem_b200
