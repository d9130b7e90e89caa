// voronoi-cpp's geometry derivative (voronoi::GeometryDerivative<Mesh>), named by luna-cpp's src/hydro/mesh_derivative.hpp:
// TEST INFRASTRUCTURE ONLY. voronoi-cpp is not installed here; the reference's moving-step derivatives take their
// geometry derivative through hydro::GeometryDerivative, which the oracle driver implements itself, so the library
// class is only declared (using it is a compile error).
#pragma once

namespace voronoi {
template <class Mesh>
struct GeometryDerivative;
}  // namespace voronoi
