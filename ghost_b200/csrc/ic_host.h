// ic_host.h -- host-side seeded initial conditions (ic_host.cpp)
#pragma once
#include <stdint.h>

namespace gb {

struct Grid {
  int nx, ny, nz, nxh, anis, arbsize;
  double Dkx, Dky, Dkz;
};

template <typename R> R randu(int32_t &idum);

template <typename R>
int32_t random_vpot(const Grid &g, int32_t seed, double kdn, double kup, int shape, R *C1, R *C2, R *C3);

}  // namespace gb
