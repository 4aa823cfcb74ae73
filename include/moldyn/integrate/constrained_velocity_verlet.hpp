// moldyn/integrate/constrained_velocity_verlet.hpp -- ConstrainedVelocityVerlet (integrate/constrained_velocity_verlet.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
