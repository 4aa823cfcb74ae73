// moldyn/b200.hpp -- namespace moldyn over the GPU library's C++ API.
//
// The headers under include/moldyn/ sit at the reference's own include paths
// (moldyn/core/system.hpp, moldyn/neighbor/verlet_list.hpp, ...), so code written
// against the reference -- its apps/moldyn_run.cpp and apps/water_rdf.cpp
// included -- builds unchanged against this library when include/ comes first
// on the include path.  Every one of them brings in the whole C++ API
// (moldyn_b200.hpp) and makes its names visible as moldyn::Name.
#pragma once

#include "../moldyn_b200.hpp"

namespace moldyn {
using namespace ::moldyn_b200;
}  // namespace moldyn
