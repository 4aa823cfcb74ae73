// moldyn/integrate/velocity_verlet.hpp -- VelocityVerlet (integrate/velocity_verlet.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
