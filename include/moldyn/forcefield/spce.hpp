// moldyn/forcefield/spce.hpp -- SpceParameters, SpceSystem, buildSpceSystem (forcefield/spce.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
