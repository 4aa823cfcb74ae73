// moldyn/core/system.hpp -- System (core/system.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
