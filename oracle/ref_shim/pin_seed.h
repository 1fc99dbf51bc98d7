// Force-included (g++ -include) when building the seed-pinned copy of the
// reference CPU factor.  The reference seeds each thread's std::mt19937 from
// std::random_device (cpu_implementation/driver_local.cpp:323-325), which makes
// every run different.  This header makes that seed come from the environment
// variable RCHOL_REF_SEED (default 1) so that a 1-thread run is reproducible and
// can be replayed exactly by the oracle.  The reference's sources are not
// modified: <random> is included first (its include guard makes the
// reference's own #include <random> a no-op) and the class name is then
// redirected to the stand-in below.  Test infrastructure only.
#pragma once
#include <random>
#include <cstdlib>

namespace std {
struct rchol_pinned_random_device {
    typedef unsigned int result_type;
    unsigned int operator()() {
        const char* s = std::getenv("RCHOL_REF_SEED");
        return s ? (unsigned int)std::strtoul(s, nullptr, 10) : 1u;
    }
    double entropy() const noexcept { return 0.0; }
};
}  // namespace std

#define random_device rchol_pinned_random_device
