/* Host shim (TEST INFRASTRUCTURE): cuda::dtoh as a host copy. */
#pragma once
#include <cstring>
namespace cuda {
template <typename T> void dtoh(T* dst, const T* src, int n) { std::memcpy(dst, src, sizeof(T) * (std::size_t) n); }
}
