// Size-field producers (fields.cu).
#pragma once

#include "mesh.hpp"

namespace osh {

// element field "grad_<name>" (3 components per component of the vertex
// field `name`), mesh_element_gradients (element_gradients.cpp:72-91)
void element_gradients(Mesh& m, char const* name);
// vertex field `name` from the element field `name`, averaged with element
// volumes as weights, mesh_recover_by_volume (recover_by_volume.cpp:55-68)
void recover_by_volume(Mesh& m, char const* name);
// vertex field "adapt_size" = max(max_h - sum_j w_j |H_j|, min_h) from the
// 9k-component vertex field hess_name, mesh_size_from_hessian
// (size_from_hessian.cpp:44-72); weights may be null (all 1)
void size_from_hessian(Mesh& m, char const* hess_name, double const* weights, double min_h,
    double max_h);
// coordinates += factor * warp with factor halved until the minimum element
// quality reaches qual_floor; warp keeps the part not applied. Returns 1 if
// the whole warp was applied (mesh_warp_to_limit, warp_to_limit.cpp:31-81).
u32 warp_to_limit(Mesh& m, double qual_floor);

}  // namespace osh
