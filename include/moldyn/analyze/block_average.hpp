// moldyn/analyze/block_average.hpp -- BlockResult and blockAverage (analyze/block_average.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
