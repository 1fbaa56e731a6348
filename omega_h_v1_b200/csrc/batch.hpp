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
// forget the segment numbers of a mesh that leaves batched adaptation
void drop_segments(Mesh& m);

// throws E_ARG unless the meshes can share a union
void check_batchable(std::vector<Mesh*> const& ms);
Mesh* concat_meshes(std::vector<Mesh*> const& ms);
Mesh* concat_meshes(std::vector<Mesh*> const& ms, cudaStream_t stream);

// order-sensitive 64-bit hash of a mesh's connectivity, tags (names, kinds
// and data) and global numbers, computed on the device
u64 mesh_digest(Mesh& m);

// the meshes of a union, in segment order (new Mesh objects on `stream`,
// or on streams of their own when stream is null)
std::vector<Mesh*> split_union(Mesh& u, cudaStream_t stream);
// only the segments k with (*want)[k] (the others come back as null)
std::vector<Mesh*> split_union(Mesh& u, cudaStream_t stream, std::vector<char> const* want);

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
  // host seconds in forming unions, in passes, and in splitting meshes out
  double secs_concat = 0, secs_passes = 0, secs_split = 0;
};
BatchStats& last_batch_stats();

// mesh_adapt's pass loop (adapt.cpp:47-94) for every segment of a union,
// one scheduling step at a time: each step runs at most one refine pass, one
// coarsen pass and one shape step (swap, else collapse slivers) over the whole
// union, each acting on the segments that are at that point of their loop.
enum : u32 { ST_INIT, ST_REFINE, ST_COARSEN, ST_SHAPE, ST_DONE, ST_FAILED };
enum : u32 { OP_REFINE, OP_COARSEN, OP_SWAP, OP_CSLIVERS };

struct AdaptParams {
  double size_floor;
  double good_qual;
  u32 nlayers;
  u32 max_ops;
};

struct SegState {
  u32 state = ST_INIT;
  u32 ops = 0;
  double qf = 0;          // satisfy_size's quality floor
  BatchMeshResult res;
};

// per-segment control arrays of a union and the host copies of their results
struct UnionCtl {
  Mesh& u;
  u32 nm;
  u32* active = nullptr;                 // device
  double* floor = nullptr;               // device
  u32* selected = nullptr;               // device
  u32* elems = nullptr;                  // device
  unsigned long long* minkey = nullptr;  // device
  u32* h_u32 = nullptr;                  // pinned: selected[nm], elems[nm]
  unsigned long long* h_key = nullptr;   // pinned: minkey[nm]
  SegCtl ctl;

  explicit UnionCtl(Mesh& m);
  ~UnionCtl();
  UnionCtl(UnionCtl const&) = delete;
  UnionCtl& operator=(UnionCtl const&) = delete;
  // mesh_min_quality of every segment
  std::vector<double> min_quality();
  // one pass over the union acting on `group`: per-segment selected counts
  // land in h_u32[0..nm), elements entering the pass in h_u32[nm..2nm)
  void run(u32 op, std::vector<u32> const& group, std::vector<double> const& floors,
      double size_floor, double good_qual, u32 nlayers);
};

// Runs mesh_adapt's loop for many meshes held apart between passes: every
// step gathers the meshes that are at the same point of their loop into
// unions of at most max_union_elems current elements (0 = no limit), runs
// that pass over each union (one launch per stage), and splits out the
// meshes it changed. A union thus only holds meshes its pass acts on.
struct GroupRunner {
  AdaptParams ap{1.0 / 3.0, 0.3, 4, 50};
  unsigned long long max_union_elems = 0;
  cudaStream_t s = nullptr;  // unions and the meshes split out of them
  // one step for every live mesh; ms[k] is replaced (and owned[k] set) when
  // a pass changes it, the previous ms[k] deleted if it was owned. Returns
  // whether any mesh is still live.
  bool step(std::vector<Mesh*>& ms, std::vector<SegState>& st, std::vector<char>& owned);
};

// the tag list a mesh has after the passes `ops` (refine_build, coarsen_build
// and swap_build keep, drop and order tags by fixed rules), applied to a mesh
// split out of a union
struct Layout {
  std::vector<Tag> tags[4];  // name, type, ncomps, transfer (data unused)
};
Layout layout_of(Mesh& m);
Layout layout_after(u32 op, Layout const& in, u32 dim);
void apply_layout(Mesh& m, Layout const& want);

// mesh_adapt of every mesh in `ms` through a GroupRunner with unions of at
// most max_union_elems current elements (0 = no limit); each mesh that
// changed is overwritten with its result
void adapt_batch(std::vector<Mesh*> const& ms, double size_floor, double good_qual,
    u32 nlayers, u32 max_ops, unsigned long long max_union_elems,
    std::vector<BatchMeshResult>& res);

// mesh_adapt of every mesh, unchanged, by `nthreads` host threads (0 = 4)
// each issuing on a stream of its own; meshes start largest first while the
// device-memory estimates of those in flight fit `budget` bytes (0 = 70% of
// the device's free memory); each mesh ends exactly as osh_adapt leaves it
void adapt_concurrent(std::vector<Mesh*> const& ms, AdaptParams const& ap, u32 nthreads,
    unsigned long long budget, std::vector<BatchMeshResult>& res);

}  // namespace osh
