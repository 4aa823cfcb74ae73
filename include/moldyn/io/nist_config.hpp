// moldyn/io/nist_config.hpp -- NistConfig and readNistConfig (io/nist_config.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
