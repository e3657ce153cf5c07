// Time window of the misfit, shared by the misfit kernels.
#pragma once
#include "efwi_kernels.h"

namespace efwi {

// Time taper of cuda_window (utilities.cu:524-614) with the reference's mix
// of float variables and double arithmetic; returns the factor the data is
// multiplied by.
__device__ __forceinline__ float window_mult(const MisfitArgs &m, int it, int r) {
  const double kPi = 3.141592653589793238462643383279502884197169;
  const float ratio = 0.005f;
  const float t = it * m.dt;
  float t0, t3, off;
  if (!m.if_win) {
    t0 = 0.0f;
    t3 = m.nt * m.dt;
    off = m.nt * m.dt * ratio;
    if (2.0 * off >= t3 - t0) return 1.0f;
  } else {
    if (ratio > 0.5f) return 1.0f;
    t0 = m.win_start[r];
    t3 = m.win_end[r];
    const float tmax = m.nt * m.dt;
    if (t0 < 0.0f) t0 = 0.0f;
    if (t0 > tmax) t0 = tmax;
    if (t3 < 0.0f) t3 = 0.0f;
    if (t3 > tmax) t3 = tmax;
    off = (t3 - t0) * ratio;
    if (off <= 0.0f) return 1.0f;
  }
  const float t1 = t0 + off, t2 = t3 - off;
  float w;
  if (t >= t0 && t < t1) w = (float)sin(kPi / 2.0 * (t - t0) / (t1 - t0));
  else if (t >= t1 && t < t2) w = 1.0f;
  else if (t >= t2 && t < t3) w = (float)cos(kPi / 2.0 * (t - t2) / (t3 - t2));
  else w = 0.0f;
  if (!m.if_win) return w * w;
  return w * w * m.weights[r] * m.src_weight;
}

}  // namespace efwi
