// moldyn/core/vec3.hpp -- Vec3 and its arithmetic (core/vec3.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
