// moldyn/core/box.hpp -- Box (core/box.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
