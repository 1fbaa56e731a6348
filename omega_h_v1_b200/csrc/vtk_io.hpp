// VTU mesh files compatible with the reference's vtk_io.cpp.
#pragma once

#include "mesh.hpp"

namespace osh {

// read_mesh_vtk: "x.vtu" (serial) or "x.pvtu" (its one piece "x.vtu", as a
// parallel mesh); throws Failure(E_IO) on a missing or malformed file
Mesh* read_vtk(char const* path);

// write_mesh_vtk_opts: binary (base64, optionally zlib) or ASCII arrays
void write_vtk(Mesh& m, char const* path, bool ascii, bool compress);

}  // namespace osh
