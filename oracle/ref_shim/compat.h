/* Host-compilation shim for the reference's constexpr headers (TEST
 * INFRASTRUCTURE, used only to build oracle/_ref/libibref.so).  The
 * reference marks its delta functions __host__ __device__; on the host those
 * attributes are empty. */
#pragma once
#define __host__
#define __device__
#define __forceinline__ inline
#include <cmath>
#include <cstdlib>
using std::abs;
using std::sqrt;
using std::cos;
