// moldyn/neighbor/verlet_list.hpp -- VerletList (neighbor/verlet_list.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
