// moldyn/forcefield/spce_forcefield.hpp -- SpceForceField (forcefield/spce_forcefield.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
