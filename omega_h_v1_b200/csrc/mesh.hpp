// Device-resident mesh store with the reference's lazy adjacency cache
// (mesh.cpp:27-334): per-dimension entity-to-vertex connectivity, tags,
// upward / downward / star / dual adjacency derived on first request and
// dropped when a pass replaces the mesh.
//
// Layout in HBM (all u32 local ids, f64 fields, u64 global numbers):
//   down[d][0]        verts_of_ents, deg(d,0) per entity, entity-major
//   down[h][l]        lows_of_highs (0 < l < h), deg(h,l) per high entity
//   up[l][h]          CSR: offs[n_l+1], adj[n_uses], dirs[n_uses]; each row
//                     sorted by use index (high * deg + dir), which is the
//                     order the reference's CPU invert_map produces
//   tags[d]           ordered list of named arrays, n_d * ncomps values each
//   globals[d]        u64 global numbers (parallel meshes only)
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "runtime.hpp"

namespace osh {

struct Tag {
  std::string name;
  u32 type = T_F64;
  u32 ncomps = 1;
  u32 transfer = X_NOT;
  void* data = nullptr;  // device
};

inline u32 tag_esz(u32 type)
{
  return type == T_U8 ? 1u : type == T_U32 ? 4u : 8u;
}

struct UpAdj {
  u32* offs = nullptr;
  u32* adj = nullptr;
  u32* dirs = nullptr;
  // rows carried through a pass: the first pre[l] uses of row l are already
  // in order and precede the rest (null when nothing is known)
  u32* pre = nullptr;
  u32 npre = 0;  // sum of pre
};

struct Graph {
  u32* offs = nullptr;
  u32* adj = nullptr;
  u32 nadj = 0;
};

// Several meshes adapted together as one disjoint union. Every vertex knows
// the mesh ("segment") it came from; a pass reads the per-segment controls
// below so that it acts only on some segments, with a quality floor of each
// segment's own, and reports how many entities it selected per segment.
struct SegCtl {
  u32 const* active = nullptr;    // device, per segment: the pass may act
  double const* floor = nullptr;  // device, per segment: quality floor
  u32* selected = nullptr;        // device, per segment: entities selected
};

// what a kernel sees of SegCtl (all null for a single mesh)
struct SegView {
  u32 const* seg = nullptr;
  u32 const* active = nullptr;
  double const* floor = nullptr;
};

struct Mesh {
  u32 dim = 3;
  bool full = false;
  bool parallel = false;
  u32 counts[4] = {0, 0, 0, 0};
  u32* down[4][4] = {};
  UpAdj up[4][4] = {};
  bool have_up[4][4] = {};
  bool up_sorted[4][4] = {};  // rows in use-index order (the reference's)
  Graph star[4][4] = {};
  bool have_star[4][4] = {};
  u32* dual = nullptr;
  // reflect_down's search rows: every edge (1) / triangle (2) listed once, in
  // one of its smallest vertex's sub-rows (4 / 8 per vertex, picked by a
  // hash of its other vertices), as (other vertices..., id) records:
  // uint2 {v1, id} for edges, uint4 {v1, v2, id, 0} for triangles
  u32* low_row_offs[3] = {nullptr, nullptr, nullptr};
  u32* low_rows[3] = {nullptr, nullptr, nullptr};
  // (during a pass's searches) vertices of the products whose lows are
  // searched, stamped search_gen in the stream's marks; the rows then list
  // only lows with a marked smallest vertex
  u32* search_marks = nullptr;
  u32 search_gen = 0;
  std::vector<Tag> tags[4];
  // Global numbers and owners. On one rank every pass renumbers them to the
  // trivial values (global number = owner id = local index, owner rank 0);
  // those are held as flags and written out only when read (ask_globals,
  // ask_own_ranks, ask_own_ids). An array, when present, wins over its flag.
  u64* globals[4] = {};
  u32* own_ranks[4] = {};
  u32* own_ids[4] = {};
  bool globals_iota[4] = {};
  bool ranks_zero[4] = {};
  bool ids_iota[4] = {};
  u32 ghost_layers = 0;
  double* qual_cache = nullptr;  // element qualities of this mesh state
  // disjoint union of nseg meshes: segment of every vertex (owned), and the
  // controls of the running pass (not owned; null = every segment acts)
  u32 nseg = 0;
  u32* seg = nullptr;
  SegCtl const* ctl = nullptr;
  // reject quality candidates on a single-precision estimate with an error
  // bound before computing them in double (decisions are unchanged)
  bool fp32_filter = false;
  cudaStream_t s = nullptr;
  bool own_stream = false;
  std::shared_ptr<Mailbox> mb;  // shared by a mesh and the meshes it spawns

  // stream == nullptr creates (and later destroys) a stream of its own,
  // unless exact_stream is set: then nullptr is the legacy default stream
  Mesh(u32 dim, bool full, bool parallel, cudaStream_t stream,
      std::shared_ptr<Mailbox> mailbox = nullptr, bool exact_stream = false);
  ~Mesh();
  Mesh(Mesh const&) = delete;
  Mesh& operator=(Mesh const&) = delete;

  // a new empty mesh on the same stream (m_out of a pass)
  Mesh* spawn() const;
  // a deep copy (connectivity, tags, globals; no derived adjacency) on a
  // stream of its own
  Mesh* clone();
  // run all further work of this mesh on `stream` (not owned)
  void use_stream(cudaStream_t stream);
  // a stream and a mailbox of its own (for a mesh handed out of a batch)
  void own_new_stream();
  // replace every array of this mesh with those of `with` (which is deleted);
  // overwrite_mesh (mesh.cpp:329-334)
  void overwrite(Mesh* with);
  void clear_contents();

  void set_ents(u32 d, u32 n, u32* verts);
  bool has_dim(u32 d) const { return d == 0 || down[d][0] != nullptr; }
  u32 count(u32 d);

  u32 const* ask_down(u32 high, u32 low);
  // reflect_down's rows for lows of dimension `low` (built once per state)
  void build_low_rows(u32 const* lows, u32 nlows);
  void reflect_many(u32 const* highs, u32 const* lows, u32 const* firsts, u32* const* outs,
      u32 npairs);
  void mark_search_verts(u32 const* first);
  void drop_search_rows();
  // down(high, low) of the high entities [first, n_high) by search, into out
  void reflect_range(u32 high, u32 low, u32 first, u32* out);
  // Upward adjacency. Rows are always the same sets; `sorted` asks for the
  // reference's row order (ascending use index), which only some consumers
  // depend on (edge rings, transfers, vertex_dest, the C API). Rows built
  // for order-free consumers are sorted in place on the first ordered ask.
  UpAdj const& ask_up(u32 low, u32 high, bool sorted = true);
  Graph const& ask_star(u32 low, u32 high);
  u32 const* ask_dual();

  Tag* find_tag(u32 d, char const* name);
  Tag& add_tag(u32 d, u32 type, char const* name, u32 ncomps, u32 transfer,
      void* data);
  void remove_tag(u32 d, char const* name);
  double const* coords();

  // element qualities (cached until the mesh changes) and their minimum
  double const* qualities();
  double min_quality();
  double* element_sizes();      // caller frees
  double* measure_edges();      // caller frees: |x1-x0| / mean size

  SegView segview() const
  {
    SegView v;
    if (seg && ctl) {
      v.seg = seg;
      v.active = ctl->active;
      v.floor = ctl->floor;
    }
    return v;
  }

  // replaces the global numbers of dimension d and forgets its owners
  // (mesh_set_globals, parallel_mesh.cpp:191-196)
  void set_globals(u32 d, u64* g);
  // the same with global number = local index, held as a flag
  void set_iota_globals(u32 d);
  bool has_globals(u32 d) const { return globals[d] || globals_iota[d]; }
  bool has_own_ranks(u32 d) const { return own_ranks[d] || ranks_zero[d]; }
  bool has_own_ids(u32 d) const { return own_ids[d] || ids_iota[d]; }
  // the arrays, written out (on the mesh's stream) if held as flags; null
  // when the mesh has none
  u64 const* ask_globals(u32 d);
  u32 const* ask_own_ranks(u32 d);
  u32 const* ask_own_ids(u32 d);

  // Ghosting bookkeeping of a single-rank parallel mesh. The reference ghosts
  // a parallel mesh at the start of every pass (mesh_ensure_ghosting,
  // ghost_mesh.cpp:283-291), which on one rank leaves the entities as they
  // are but records one ghost layer and the owner ranks of every dimension;
  // each exchange on a dimension (mesh_ask_exchanger, parallel_mesh.cpp:
  // 96-105) adds owner ranks and ids there. A pass that then finds nothing
  // to do leaves the mesh in that state, which shows in
  // osh_num_ghost_layers, osh_own_rank / osh_own_id and the own_rank /
  // own_id arrays of its files. On one rank the owner rank is 0 and the
  // owner id the entity's own index, so the owners are present (as flags)
  // exactly when the reference would hold them. No-ops unless the mesh is
  // parallel and not a union of segments.
  void ensure_ghosting(u32 nlayers);
  void note_exchange(u32 d);
  void derive_model(double crease_angle);  // host classification
  void make_parallel();
};

// down(high, low) of `out`, the mesh a pass built from `m`, for every pair
// m has (h = 2..dim, l = 1..h-1): surviving high entities (same_of[h]:
// survivor offsets of m's highs; the nsame_of[h] survivors are numbered
// first in out) take their old lows through same_of[l] (the lows' survivor
// offsets), all pairs in one launch; the entities the pass made are
// searched, all pairs in one launch, with search rows limited to the
// products' vertices when they are few
void carry_down_all(Mesh& m, Mesh& out, u32* const* same_of, u32 const* nsame_of);

// up(low, high) of `out` for every pair m has: surviving lows keep their
// old rows' uses by surviving highs (mapped, in order), then the uses of the
// entities the pass made are added; rows come out unsorted. Every pair's
// counts are scanned together in one launch.
// (same_of[d]: survivor offsets of m's entities of dimension d, nullptr
// for a dimension the pass does not keep; nsame_of[d] survivors, numbered
// first in out; newid_of[d] (optional): each old entity's new id, INV for
// the ones that do not survive)
void carry_up_all(Mesh& m, Mesh& out, u32* const* same_of, u32 const* nsame_of,
    u32* const* newid_of);
// new id of every old entity, or INV where it did not survive (caller frees)
u32* carry_new_ids(u32 const* same, u32 n, cudaStream_t s);
// whether a pass over m carries some upward adjacency of dimension `high`
// (and so wants the new ids of its kept entities)
inline bool carried_high(Mesh const& m, u32 high)
{
  if (high == 0 || high > 3) return false;
  for (u32 l = 0; l < high; ++l)
    if (m.have_up[l][high]) return true;
  return false;
}

// derivation helpers (mesh.cu)
void up_from_down(u32 high, u32 low, u32 nhighs, u32 nlows, u32 const* lows_of_highs,
    UpAdj& out, cudaStream_t s);
// the same rows in arbitrary order within each row
void up_from_down_unsorted(u32 high, u32 low, u32 nhighs, u32 nlows,
    u32 const* lows_of_highs, UpAdj& out, cudaStream_t s);
// put the rows of an upward adjacency into ascending use order, in place
void sort_up_rows(u32 high, u32 low, u32 nhighs, u32 nlows, UpAdj const& u,
    cudaStream_t s);

}  // namespace osh
