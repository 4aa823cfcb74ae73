// moldyn/util/lattice.hpp -- fccLattice (util/lattice.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
