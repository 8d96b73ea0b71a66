// Stand-in for the one Thrust name CODAG's encoder header uses (thrust::device), so that the
// header compiles with the host compiler for oracle/ref_rlev2_host.cpp.  The host functions
// that would use it are never called there.
#pragma once
namespace thrust {
struct shim_device_policy {};
inline constexpr shim_device_policy device{};
}  // namespace thrust
