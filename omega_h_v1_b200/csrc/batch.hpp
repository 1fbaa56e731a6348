// Many meshes adapted together: the meshes are concatenated by CSR offsets
// into one disjoint union (a "batch"), every stage of a pass runs as one
// launch over the whole union, and each mesh keeps the pass sequence that
// mesh_adapt (adapt.cpp:47-94) would give it alone. The union preserves the
// relative order of each mesh's entities, every pass treats disconnected
// meshes independently, and per-segment controls (SegCtl) give each mesh its
// own quality floor and its own place in the refine / coarsen / shape loop,
// so each mesh comes out exactly as mesh_adapt would leave it.
#pragma once

#include <vector>

#include "passes.hpp"

namespace osh {

// one disjoint union of the meshes, on a stream of its own; every mesh must
// have the same dimension, representation and tag list
Mesh* concat_meshes(std::vector<Mesh*> const& ms);
Mesh* concat_meshes(std::vector<Mesh*> const& ms, cudaStream_t stream);

// order-sensitive 64-bit hash of a mesh's connectivity, tags (names, kinds
// and data) and global numbers, computed on the device
u64 mesh_digest(Mesh& m);

// the meshes of a union, in segment order (new Mesh objects on `stream`,
// or on streams of their own when stream is null)
std::vector<Mesh*> split_union(Mesh& u, cudaStream_t stream);

struct BatchMeshResult {
  std::vector<u32> ops;  // the passes that changed this mesh, in order
  u32 changed = 0;       // what mesh_adapt would return
  u32 passes = 0;        // passes that changed this mesh
  double elems_in = 0;   // elements entering those passes, summed
  int status = 0;        // 0, or E_MAXOPS when the pass cap was exceeded
};

struct BatchStats {
  u32 unions = 0;        // unions adapted
  u32 steps = 0;         // scheduling steps over all unions
  u32 union_passes = 0;  // passes run over whole unions
  u32 mesh_passes = 0;   // passes that changed a mesh, summed over meshes
  double elems_in = 0;   // elements entering those passes, summed
};
BatchStats& last_batch_stats();

// mesh_adapt of every segment of the union (in place)
void adapt_union(Mesh& u, double size_floor, double good_qual, u32 nlayers, u32 max_ops,
    std::vector<BatchMeshResult>& res);

// mesh_adapt of every mesh in `ms`, adapted in unions of at most
// `max_union_elems` input elements (0 = one union); each mesh that changed
// is overwritten with its result
void adapt_batch(std::vector<Mesh*> const& ms, double size_floor, double good_qual,
    u32 nlayers, u32 max_ops, unsigned long long max_union_elems,
    std::vector<BatchMeshResult>& res);

}  // namespace osh
