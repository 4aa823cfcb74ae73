// moldyn/neighbor/cell_list.hpp -- CellList (neighbor/cell_list.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
