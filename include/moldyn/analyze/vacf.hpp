// moldyn/analyze/vacf.hpp -- Vacf (analyze/vacf.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
