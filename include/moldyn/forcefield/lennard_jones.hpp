// moldyn/forcefield/lennard_jones.hpp -- LennardJones and Truncation (forcefield/lennard_jones.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
