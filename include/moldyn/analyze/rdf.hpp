// moldyn/analyze/rdf.hpp -- Rdf (analyze/rdf.hpp) on the GPU library, in namespace moldyn.
#pragma once

#include "../b200.hpp"
