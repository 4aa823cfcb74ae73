// moldyn/forcefield/ewald.hpp -- Ewald and EwaldTerms (forcefield/ewald.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
