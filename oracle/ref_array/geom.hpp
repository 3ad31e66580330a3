// Oracle-only stand-in for the CMake-generated geom.hpp (src/utils/geom.hpp.in):
// the geometry comes from -DHCL_REF_SPHERICAL=0|1 instead of Heraclespp_GEOM.
#pragma once

#include <string_view>

namespace hclpp {

inline constexpr std::string_view geom_choice = HCL_REF_SPHERICAL ? "Spherical" : "Cartesian";

enum class Geometry : char { Geom_cartesian, Geom_spherical };

constexpr Geometry geom = HCL_REF_SPHERICAL ? Geometry::Geom_spherical : Geometry::Geom_cartesian;

} // namespace hclpp
