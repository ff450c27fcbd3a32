/* Host shim (TEST INFRASTRUCTURE): what algo/gershgorin.h names from thrust;
 * the bridge never calls that function. */
#pragma once
namespace thrust {
template <typename P, typename It> It max_element(P, It b, It e) { It m = b; for (; b != e; ++b) if (*m < *b) m = b; return m; }
template <typename P, typename It> It min_element(P, It b, It e) { It m = b; for (; b != e; ++b) if (*b < *m) m = b; return m; }
}
