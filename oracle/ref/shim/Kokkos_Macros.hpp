// Serial stand-in (see Kokkos_Core.hpp in this folder).
#pragma once
#include "Kokkos_Core.hpp"
