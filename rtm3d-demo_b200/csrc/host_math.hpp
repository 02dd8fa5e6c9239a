// host_math.hpp -- host-side helpers shared inside the library.
#pragma once
#include <cstdint>

namespace rtmb {
// Sample it of the Ricker wavelet, t = it*dt - 1/fpeak (RTMSeismicSource::loadSamples / ricker,
// include/RTMSeismic.hpp:135-144, 191-198); rtmb_ricker fills a whole series with it.
float ricker_sample(uint32_t it, float dt, float fpeak);
}  // namespace rtmb
