// moldyn/integrate/nose_hoover.hpp -- NoseHooverChain (integrate/nose_hoover.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
