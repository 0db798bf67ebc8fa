// Drop-in replacement of the reference's const.h (mrnorman/awflCloud const.h) for builds
// that run the operators on the B200 library (libawfl.so, include/awfl.h) instead of YAKL.
//
// Provides what driver.cpp and the operator headers use from the reference's const.h:
// the `real` type (double, const.h:29), the compile-time order ORD/NGLL (const.h:21-27),
// endrun (const.h:76-79), and the three yakl:: calls driver.cpp makes (init, fence,
// finalize), plus the YAML reader.
#pragma once

#include <chrono>
#include <cmath>
#include <cstdio>
#include <iostream>
#include <string>

#include "awfl.h"
#include "awfl_yaml.h"

#ifndef ORD
#define ORD 5
#endif

#ifndef NGLL
#define NGLL 3
#endif

typedef double real;

int constexpr ord = ORD;
int constexpr ngll = NGLL;

static_assert(ngll <= ord, "ERROR: ngll must be <= ord");
static_assert((ord == 5 && ngll == 3) || (ord == 9 && ngll == 5),
              "the B200 library is built for (ORD, NGLL) = (5, 3) and (9, 5)");

template <class T> void endrun(T err) {
  std::cerr << err << std::endl;
  throw err;
}

namespace yakl {
// The driver brackets its timed region with fence(): wait for all device work.
inline void init() {}
inline void fence() { awfl_device_synchronize(); }
inline void finalize() {}
}  // namespace yakl
