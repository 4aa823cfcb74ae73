// moldyn/integrate/langevin.hpp -- LangevinBAOAB (integrate/langevin.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
