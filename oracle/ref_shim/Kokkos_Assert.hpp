// Oracle-only stand-in: device assertions become no-ops on the host build.
#pragma once
#include "Kokkos_Macros.hpp"
#define KOKKOS_ASSERT(...)
