// The adaptation passes (refine / coarsen / swap / adapt driver) and the
// pieces they share: independent sets, class inheritance, expansion.
#pragma once

#include <vector>

#include "mesh.hpp"

namespace osh {

// segment controls of a disjoint union of meshes (SegCtl): whether the pass
// acts on the segment of vertex `vert`, and that segment's quality floor
__device__ inline bool seg_acts(SegView const& v, u32 vert)
{
  return !v.active || v.active[v.seg[vert]] != 0;
}
__device__ inline double seg_floor(SegView const& v, u32 vert, double f)
{
  return v.floor ? v.floor[v.seg[vert]] : f;
}

// add, per segment, the number of flagged entities of dimension ent_dim to
// m.ctl->selected (no-op for a single mesh)
void seg_tally(Mesh& m, u32 ent_dim, u32 const* flags);

// Luby independent set over the star graph of `ent_dim` entities
// (mesh_find_indset, indset.cpp:119-139). filter and goodness are device
// arrays; returns a device state array (1 = in set) or throws E_NOCONVERGE.
// With check = false the outcome is not read back here: the caller fetches
// at least INDSET_FETCH_SLOTS mailbox slots later (with its own read-back)
// and calls indset_check, which throws as find_indset would have.
constexpr u32 INDSET_FETCH_SLOTS = 51;
u32* find_indset(Mesh& m, u32 ent_dim, u32 const* filter, double const* goodness,
    bool check = true);
void indset_check(Mesh& m);

// copy rows of `width` elements: out[j] = in[i] for j in
// [offs[i]*k, offs[i+1]*k), for T of 1, 4 or 8 bytes
void expand_scaled(void const* in, u32 const* offs, u32 k, u32 n, u32 width,
    u32 esz, void* out, cudaStream_t s);

// one row expansion (as expand_scaled); expand_many runs up to eight per
// launch. list (optional): the rows that produce anything, n of them (the
// others are skipped without reading their offsets); in2 / out2 (optional):
// a second array copied with the same offsets
struct ExpandJob {
  void const* in = nullptr;
  u32 const* offs = nullptr;
  void* out = nullptr;
  u32 k = 1, n = 0, width = 0, esz = 4;
  u32 const* list = nullptr;
  void const* in2 = nullptr;
  void* out2 = nullptr;
};
void expand_many(std::vector<ExpandJob> const& jobs, cudaStream_t s);

// Per-dimension domains that produce entities of one dimension during a
// pass: ndoms[d] entities of dimension d, each producing
// (offs[d][i+1]-offs[d][i]) * scale[d] products. Slot 0 is the "same"
// entities carried over from the old mesh. (inherit.cpp:8-138)
struct Doms {
  u32 ndoms[4] = {0, 0, 0, 0};
  u32 const* offs[4] = {nullptr, nullptr, nullptr, nullptr};
  // (optional) the domains that produce anything, in order, and their count
  u32 const* list[4] = {nullptr, nullptr, nullptr, nullptr};
  u32 nlist[4] = {0, 0, 0, 0};
  u32 scale[4] = {1, 1, 1, 1};
  u32 ngen[4] = {0, 0, 0, 0};  // host copy of each domain's product count
  u32 ngo[5] = {0, 0, 0, 0, 0};
  void finish()
  {
    ngo[0] = 0;
    for (u32 i = 0; i < 4; ++i) ngo[i + 1] = ngo[i] + ngen[i];
  }
};

// class_dim / class_id of the products of `prod_dim` (inherit_class,
// inherit.cpp:217-232)
// `also` (optional): further row expansions launched with the labels' copies
// `defer` (optional): the copies are appended there for the caller to
// launch (expand_many) instead of launched here; what they read must stay
// allocated until then
void inherit_class(Mesh& m, Mesh& out, u32 prod_dim, Doms const& d,
    std::vector<ExpandJob> const* also = nullptr, std::vector<ExpandJob>* defer = nullptr);

// u64 global numbering of a single-rank parallel mesh after a pass
// (inherit_globals, parallel_modify.cpp:79-111): survivors keep their order,
// new entities follow.
void inherit_globals(Mesh& out, u32 d);

// element coordinates (interp_to_elems of "coordinates", element_field.cpp)
void interp_coords_to_elems(Mesh& m);

u32 refine_by_size(Mesh& m, double qual_floor);
void uniformly_refine(Mesh& m);
u32 coarsen_by_size(Mesh& m, double qual_floor, double size_floor);
u32 coarsen_slivers(Mesh& m, double qual_floor, u32 nlayers);
u32 swap_slivers(Mesh& m, double good_qual, u32 nlayers);
u32 mesh_adapt(Mesh& m, double size_floor, double good_qual, u32 nlayers, u32 max_ops);

// per-stage sets of each pass, without modifying the mesh (device outputs)
u32 refine_sets(Mesh& m, double qual_floor, u32* cand, u32* good, double* quals,
    u32* indset);
u32 coarsen_sets(Mesh& m, double qual_floor, double size_floor, u32* codes_size,
    u32* codes_class, u32* codes_qual, double* quals2, u32* cand, double* col_qual,
    u32* indset, u32* gen_vert);
u32 swap_sets(Mesh& m, double good_qual, u32 nlayers, u32* slivers, u32* cand,
    u32* interior, u32* good, double* quals, u32* ring_sizes, u32* indset);

// mark helpers (mark.cpp)
u32* mark_down(Mesh& m, u32 high, u32 low, u32 const* marked_highs);
u32* mark_up(Mesh& m, u32 low, u32 high, u32 const* marked_lows);
u32* mark_slivers(Mesh& m, double good_qual, u32 nlayers);

// small device counter helpers
struct Counter {
  u32* d;
  cudaStream_t s;
  explicit Counter(cudaStream_t st) : s(st)
  {
    d = dalloc<u32>(1, s);
    CK(cudaMemsetAsync(d, 0, sizeof(u32), s));
  }
  ~Counter() { cudaFreeAsync(d, s); }
  void zero() { CK(cudaMemsetAsync(d, 0, sizeof(u32), s)); }
  u32 get() { return read_u32(d, s); }
};

// per-pass statistics, read by the C API for reporting
struct PassStats {
  u32 op = 0;            // 1 refine, 2 coarsen, 3 swap, 4 coarsen_slivers
  u32 elems_in = 0;
  u32 elems_out = 0;
  u32 nselected = 0;     // split edges / collapsed verts / swapped edges
  u32 indset_rounds = 0;
};
PassStats& last_pass_stats();

// statistics of the last mesh_adapt call on this thread
struct AdaptStats {
  u32 passes = 0;          // passes that changed the mesh
  double elems_in = 0;     // elements entering those passes, summed
};
AdaptStats& last_adapt_stats();

}  // namespace osh
