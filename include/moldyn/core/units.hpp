// moldyn/core/units.hpp -- units (core/units.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
