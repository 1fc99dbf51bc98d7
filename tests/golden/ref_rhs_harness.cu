// Prints the reference's right-hand-side generators (gpu_implementation/
// solver.hpp:29-61) for the golden fixtures.  Built and run only by
// tests/golden/make_golden.py, inside the container that holds the reference.
#include "gpu_implementation/solver.hpp"
#include <cstdlib>

int main(int argc, char** argv) {
    size_t n = (size_t)std::atoll(argv[1]);
    unsigned long seed = std::strtoul(argv[2], nullptr, 10);
    int kind = std::atoi(argv[3]);  // 0 zero-sum, 1 uniform(-1,1)
    std::vector<double> v(n);
    if (kind == 0) generate_zero_sum_vector<double>(v.data(), n, seed);
    else generate_random_vector<double>(v.data(), n, seed);
    for (size_t i = 0; i < n; ++i) printf("%.17g\n", v[i]);
    return 0;
}
