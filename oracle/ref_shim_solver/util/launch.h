/* Host shim (TEST INFRASTRUCTURE): util::transform as a host loop. */
#pragma once
namespace util {
template <int nt = 128, int vt = 1, typename F, typename... A>
void transform(F&& f, int n, A&&... a) { for (int i = 0; i < n; ++i) f(i, a...); }
}
