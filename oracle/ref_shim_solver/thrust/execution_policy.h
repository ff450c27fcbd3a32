/* Host shim (TEST INFRASTRUCTURE): see extrema.h in this directory. */
#pragma once
namespace thrust {
template <typename T> struct execution_policy {};
namespace system { namespace cuda { struct tag {}; } }
}
