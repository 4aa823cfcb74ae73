// moldyn/forcefield/forcefield.hpp -- EnergyVirial and ForceField (forcefield/forcefield.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
