// moldyn/util/random.hpp -- Rng (util/random.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
