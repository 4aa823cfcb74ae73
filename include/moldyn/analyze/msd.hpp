// moldyn/analyze/msd.hpp -- Msd (analyze/msd.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
