// Reads whitespace-separated samples from stdin and prints blockAverage's mean,
// standard error and block count (include/moldyn/analyze/block_average.hpp), each
// to 17 significant digits.  CPU only: blockAverage does no device work.
#include <cstdio>
#include <iostream>
#include <vector>

#include "moldyn/analyze/block_average.hpp"

int main() {
    std::vector<double> samples;
    double x;
    while (std::cin >> x) samples.push_back(x);
    const moldyn::BlockResult r = moldyn::blockAverage(samples);
    std::printf("%.17g %.17g %zu\n", r.mean, r.standardError, r.blocks);
    return 0;
}
