/* Host shim (TEST INFRASTRUCTURE): util::memory as a host buffer. */
#pragma once
#include <cstddef>
#include <vector>
namespace util {
template <typename T> struct memory {
	std::vector<T> v;
	explicit memory(std::size_t n) : v(n) {}
	T* data() { return v.data(); }
};
}
