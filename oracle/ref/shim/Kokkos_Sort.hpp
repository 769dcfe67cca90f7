// Serial stand-in (test scaffolding): the reference's narrowphase header includes Kokkos_Sort.hpp but sorts with
// its own radix_sorter (src/bvh/util/sort.hpp), so nothing of it is needed here.
#pragma once
#include "Kokkos_Core.hpp"
