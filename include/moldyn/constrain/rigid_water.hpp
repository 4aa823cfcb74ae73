// moldyn/constrain/rigid_water.hpp -- RigidWater (constrain/rigid_water.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
