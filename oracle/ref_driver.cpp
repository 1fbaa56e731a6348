// Test infrastructure only (never shipped, never timed as the product).
//
// A thin extern "C" driver over the reference library built from the
// reference's own sources (oracle/Makefile). Python (oracle/ref.py) loads it
// with ctypes to run the reference's adaptation passes on the same seeded
// inputs as our CUDA path, and to read back connectivity, tags, adjacency
// and the per-pass candidate / independent sets.
//
// Mesh set-up follows the reference's own tests (test_warp_3d.cpp:115-119):
// new_mesh(dim, MESH_REDUCED, 0), mesh_set_ents, "coordinates" tag,
// mesh_derive_model(m, PI/4), mesh_set_rep(m, MESH_FULL).

#include <cstdlib>
#include <cstring>

#include "adapt.hpp"
#include "algebra.hpp"
#include "arrays.hpp"
#include "check_collapse_class.hpp"
#include "coarsen.hpp"
#include "coarsen_qualities.hpp"
#include "collapse_codes.hpp"
#include "collapses_to_verts.hpp"
#include "derive_model.hpp"
#include "element_gradients.hpp"
#include "doubles.hpp"
#include "indset.hpp"
#include "mark.hpp"
#include "mesh.hpp"
#include "parallel_mesh.hpp"
#include "quality.hpp"
#include "recover_by_volume.hpp"
#include "refine.hpp"
#include "refine_qualities.hpp"
#include "size.hpp"
#include "size_from_hessian.hpp"
#include "swap.hpp"
#include "swap_qualities.hpp"
#include "tables.hpp"
#include "tag.hpp"
#include "vtk_io.hpp"
#include "warp_to_limit.hpp"

using namespace omega_h;

#define M(p) reinterpret_cast<struct mesh*>(p)

extern "C" {

void* refd_new_reduced(unsigned dim, unsigned nverts, double const* coords,
    unsigned nelems, unsigned const* conn)
{
  struct mesh* m = new_mesh(dim, MESH_REDUCED, 0);
  mesh_set_ents(m, 0, nverts, 0);
  unsigned vpe = the_down_degrees[dim][0];
  unsigned* c = LOOP_MALLOC(unsigned, nelems * vpe);
  memcpy(c, conn, sizeof(unsigned) * nelems * vpe);
  mesh_set_ents(m, dim, nelems, c);
  double* x = LOOP_MALLOC(double, nverts * 3);
  memcpy(x, coords, sizeof(double) * nverts * 3);
  mesh_add_tag(m, 0, TAG_F64, "coordinates", 3, x);
  return m;
}

void refd_derive_model_full(void* p)
{
  mesh_derive_model(M(p), PI / 4);
  mesh_set_rep(M(p), MESH_FULL);
}

void refd_make_parallel(void* p) { mesh_make_parallel(M(p)); }

// read_mesh_vtk / write_mesh_vtk_opts (vtk_io.cpp:787-826); ascii selects
// VTK_ASCII, else VTK_BINARY (zlib-compressed in the USE_ZLIB=1 build)
void* refd_read_vtk(char const* path) { return read_mesh_vtk(path); }

void refd_write_vtk(void* p, char const* path, unsigned ascii)
{
  write_mesh_vtk_opts(M(p), path, ascii ? VTK_ASCII : VTK_BINARY);
}

unsigned refd_is_full(void* p) { return mesh_get_rep(M(p)) == MESH_FULL; }
unsigned refd_is_parallel(void* p) { return mesh_is_parallel(M(p)); }
unsigned refd_ghost_layers(void* p) { return mesh_ghost_layers(M(p)); }

void refd_free(void* p) { free_mesh(M(p)); }

unsigned refd_dim(void* p) { return mesh_dim(M(p)); }

unsigned refd_count(void* p, unsigned dim) { return mesh_count(M(p), dim); }

void refd_add_tag(void* p, unsigned dim, char const* name, unsigned type,
    unsigned ncomps, unsigned transfer, void const* data)
{
  unsigned n = mesh_count(M(p), dim) * ncomps;
  unsigned sz = tag_size(static_cast<enum tag_type>(type));
  void* d = loop_host_malloc(sz * n);
  memcpy(d, data, sz * n);
  add_tag2(mesh_tags(M(p), dim), static_cast<enum tag_type>(type), name,
      ncomps, static_cast<enum osh_transfer>(transfer), d);
}

void refd_free_tag(void* p, unsigned dim, char const* name)
{
  mesh_free_tag(M(p), dim, name);
}

unsigned refd_ntags(void* p, unsigned dim) { return mesh_count_tags(M(p), dim); }

char const* refd_tag_name(void* p, unsigned dim, unsigned i)
{
  return mesh_get_tag(M(p), dim, i)->name;
}
unsigned refd_tag_type(void* p, unsigned dim, unsigned i)
{
  return mesh_get_tag(M(p), dim, i)->type;
}
unsigned refd_tag_ncomps(void* p, unsigned dim, unsigned i)
{
  return mesh_get_tag(M(p), dim, i)->ncomps;
}
unsigned refd_tag_transfer(void* p, unsigned dim, unsigned i)
{
  return mesh_get_tag(M(p), dim, i)->transfer_type;
}
void refd_tag_data(void* p, unsigned dim, unsigned i, void* out)
{
  struct const_tag* t = mesh_get_tag(M(p), dim, i);
  unsigned n = mesh_count(M(p), dim) * t->ncomps;
  memcpy(out, t->d.raw, tag_size(t->type) * n);
}

void refd_down(void* p, unsigned high, unsigned low, unsigned* out)
{
  unsigned n = mesh_count(M(p), high) * the_down_degrees[high][low];
  memcpy(out, mesh_ask_down(M(p), high, low), sizeof(unsigned) * n);
}

unsigned refd_up_size(void* p, unsigned low, unsigned high)
{
  return mesh_ask_up(M(p), low, high)->offsets[mesh_count(M(p), low)];
}

void refd_up(void* p, unsigned low, unsigned high, unsigned* offs,
    unsigned* adj, unsigned* dirs)
{
  struct const_up* u = mesh_ask_up(M(p), low, high);
  unsigned n = mesh_count(M(p), low);
  unsigned nadj = u->offsets[n];
  memcpy(offs, u->offsets, sizeof(unsigned) * (n + 1));
  memcpy(adj, u->adj, sizeof(unsigned) * nadj);
  memcpy(dirs, u->directions, sizeof(unsigned) * nadj);
}

unsigned refd_star_size(void* p, unsigned low, unsigned high)
{
  return mesh_ask_star(M(p), low, high)->offsets[mesh_count(M(p), low)];
}

void refd_star(void* p, unsigned low, unsigned high, unsigned* offs,
    unsigned* adj)
{
  struct const_graph* g = mesh_ask_star(M(p), low, high);
  unsigned n = mesh_count(M(p), low);
  memcpy(offs, g->offsets, sizeof(unsigned) * (n + 1));
  memcpy(adj, g->adj, sizeof(unsigned) * g->offsets[n]);
}

void refd_dual(void* p, unsigned* out)
{
  unsigned d = mesh_dim(M(p));
  unsigned n = mesh_count(M(p), d) * the_down_degrees[d][d - 1];
  memcpy(out, mesh_ask_dual(M(p)), sizeof(unsigned) * n);
}

unsigned refd_has_globals(void* p, unsigned dim)
{
  if (!mesh_is_parallel(M(p)))
    return 0;
  return mesh_ask_globals(M(p), dim) != 0;
}

void refd_globals(void* p, unsigned dim, unsigned long* out)
{
  memcpy(out, mesh_ask_globals(M(p), dim),
      sizeof(unsigned long) * mesh_count(M(p), dim));
}

void refd_set_globals(void* p, unsigned dim, unsigned long const* in)
{
  unsigned n = mesh_count(M(p), dim);
  unsigned long* g = LOOP_MALLOC(unsigned long, n);
  memcpy(g, in, sizeof(unsigned long) * n);
  mesh_set_globals(M(p), dim, g);
}

double refd_min_quality(void* p) { return mesh_min_quality(M(p)); }

void refd_qualities(void* p, double* out)
{
  double* q = mesh_qualities(M(p));
  memcpy(out, q, sizeof(double) * mesh_count(M(p), mesh_dim(M(p))));
  loop_free(q);
}

void refd_edge_lengths(void* p, double* out)
{
  double* l = mesh_measure_edges_for_adapt(M(p));
  memcpy(out, l, sizeof(double) * mesh_count(M(p), 1));
  loop_free(l);
}

unsigned refd_refine_by_size(void* p, double qf) { return refine_by_size(M(p), qf); }
void refd_uniformly_refine(void* p) { uniformly_refine(M(p)); }
unsigned refd_coarsen_by_size(void* p, double qf, double sf)
{
  return coarsen_by_size(M(p), qf, sf);
}
unsigned refd_coarsen_slivers(void* p, double qf, unsigned nl)
{
  return coarsen_slivers(M(p), qf, nl);
}
unsigned refd_swap_slivers(void* p, double gq, unsigned nl)
{
  return swap_slivers(M(p), gq, nl);
}
unsigned refd_adapt(void* p, double sf, double gq, unsigned nl, unsigned mo)
{
  return mesh_adapt(M(p), sf, gq, nl, mo);
}

/* The pass sequence of mesh_adapt (adapt.cpp:47-94) calling the reference's
   own passes, counting the passes that change the mesh and the elements
   entering them (the throughput metric's numerator). Returns 1 on success,
   0 when max_ops is exceeded (the reference would abort). */
unsigned refd_adapt_counted(void* p, double sf, double gq, unsigned nl,
    unsigned max_ops, unsigned* passes, double* elems_in)
{
  struct mesh* m = M(p);
  unsigned ops = 0;
  double in = 0;
  unsigned dim = mesh_dim(m);
  double qf = mesh_min_quality(m);
  if (gq < qf) qf = gq;
  unsigned before = mesh_count(m, dim);
#define COUNTED(call)                 \
  (before = mesh_count(m, dim), (call))
#define INCR()                        \
  do {                                \
    in += before;                     \
    if (ops > max_ops) {              \
      *passes = ops;                  \
      *elems_in = in;                 \
      return 0;                       \
    }                                 \
    ++ops;                            \
  } while (0)
  while (COUNTED(refine_by_size(m, qf))) INCR();
  while (COUNTED(coarsen_by_size(m, qf, sf))) INCR();
  for (;;) {
    if (mesh_min_quality(m) >= gq) break;
    if (dim == 3 && COUNTED(swap_slivers(m, gq, nl))) {
      INCR();
      continue;
    }
    if (COUNTED(coarsen_slivers(m, gq, nl))) {
      INCR();
      continue;
    }
    break;
  }
#undef INCR
#undef COUNTED
  *passes = ops;
  *elems_in = in;
  return 1;
}

/* Refine selection on the current mesh, without modifying it: the steps of
   refine_by_size (refine.cpp:17-27) and choose_refinement_indset
   (refine_common.cpp:131-160). Outputs are per edge. Returns 1 when an
   independent set was computed. */
unsigned refd_refine_sets(void* p, double qual_floor, unsigned* cand,
    unsigned* good, double* quals, unsigned* indset)
{
  struct mesh* m = M(p);
  unsigned n = mesh_count(m, 1);
  double* len = mesh_measure_edges_for_adapt(m);
  unsigned* g = LOOP_MALLOC(unsigned, n);
  for (unsigned i = 0; i < n; ++i)
    cand[i] = g[i] = len[i] > 1.0;
  loop_free(len);
  double* q = mesh_refine_qualities(m, 1, &g, qual_floor, 0);
  unsigned any = 0;
  for (unsigned i = 0; i < n; ++i) {
    good[i] = g[i];
    quals[i] = g[i] ? q[i] : 0.0;
    indset[i] = 0;
    any |= g[i];
  }
  if (any) {
    unsigned* s = mesh_find_indset(m, 1, g, q);
    memcpy(indset, s, sizeof(unsigned) * n);
    loop_free(s);
  }
  loop_free(g);
  loop_free(q);
  return any;
}

/* Coarsen selection without modifying the mesh: the steps of coarsen_by_size
   (coarsen.cpp:23-36) and coarsen_common (coarsen_common.cpp:109-189).
   codes/quals2 are per edge (quals2 two per edge, 0 where unused);
   cand/col_qual/indset/gen_vert per vertex. Returns 1 if an indset exists. */
unsigned refd_coarsen_sets(void* p, double qual_floor, double size_floor,
    unsigned* codes_size, unsigned* codes_class, unsigned* codes_qual,
    double* quals2, unsigned* cand, double* col_qual, unsigned* indset,
    unsigned* gen_vert)
{
  struct mesh* m = M(p);
  unsigned dim = mesh_dim(m);
  unsigned ne = mesh_count(m, 1);
  unsigned nv = mesh_count(m, 0);
  double* len = mesh_measure_edges_for_adapt(m);
  unsigned* codes = LOOP_MALLOC(unsigned, ne);
  for (unsigned i = 0; i < ne; ++i)
    codes[i] = codes_size[i] =
      (len[i] < size_floor) ? COLLAPSE_BOTH : DONT_COLLAPSE;
  loop_free(len);
  for (unsigned i = 0; i < nv; ++i) {
    cand[i] = 0; col_qual[i] = 0; indset[i] = 0; gen_vert[i] = INVALID;
  }
  check_collapse_class(m, codes);
  memcpy(codes_class, codes, sizeof(unsigned) * ne);
  double const* coords = mesh_find_tag(m, 0, "coordinates")->d.f64;
  double* q2 = coarsen_qualities(dim, ne, codes,
      mesh_ask_down(m, dim, 0), mesh_ask_down(m, 1, 0),
      mesh_ask_up(m, 0, dim)->offsets, mesh_ask_up(m, 0, dim)->adj,
      mesh_ask_up(m, 0, dim)->directions, coords, qual_floor, 0);
  unsigned any = 0;
  for (unsigned i = 0; i < ne; ++i) {
    codes_qual[i] = codes[i];
    for (unsigned j = 0; j < 2; ++j)
      quals2[i * 2 + j] = collapses(codes[i], j) ? q2[i * 2 + j] : 0.0;
    any |= codes[i];
  }
  if (!any) {
    loop_free(codes);
    loop_free(q2);
    return 0;
  }
  mesh_add_tag(m, 1, TAG_U32, "col_codes", 1, codes);
  mesh_add_tag(m, 1, TAG_F64, "col_quals", 2, q2);
  valid_collapses_to_verts(m);
  unsigned const* c = mesh_find_tag(m, 0, "candidates")->d.u32;
  double const* cq = mesh_find_tag(m, 0, "col_qual")->d.f64;
  for (unsigned i = 0; i < nv; ++i) {
    cand[i] = c[i];
    col_qual[i] = c[i] ? cq[i] : 0.0;
  }
  unsigned* s = mesh_find_indset(m, 0, c, cq);
  mesh_add_tag(m, 0, TAG_U32, "indset", 1, s);
  unsigned* gv = collapsing_vertex_destinations(m);
  for (unsigned i = 0; i < nv; ++i) {
    indset[i] = s[i];
    gen_vert[i] = s[i] ? gv[i] : INVALID;
  }
  loop_free(gv);
  mesh_free_tag(m, 0, "indset");
  mesh_free_tag(m, 0, "candidates");
  mesh_free_tag(m, 0, "col_qual");
  mesh_free_tag(m, 1, "col_codes");
  mesh_free_tag(m, 1, "col_quals");
  return 1;
}

/* Swap selection without modifying the mesh: swap_slivers (swap.cpp:138-154)
   and swap_common (swap.cpp:99-136) up to the independent set.
   Per element: slivers (after layer growth). Per edge: cand (marked down),
   interior (after unmark_boundary), good (after swap quality), quals, ring
   sizes and indset. */
unsigned refd_swap_sets(void* p, double good_qual, unsigned nlayers,
    unsigned* slivers_out, unsigned* cand, unsigned* interior,
    unsigned* good, double* quals, unsigned* ring_sizes, unsigned* indset)
{
  struct mesh* m = M(p);
  unsigned dim = mesh_dim(m);
  unsigned ne = mesh_count(m, 1);
  unsigned nelems = mesh_count(m, dim);
  unsigned* slivers = mesh_mark_slivers(m, good_qual, nlayers);
  memcpy(slivers_out, slivers, sizeof(unsigned) * nelems);
  unsigned* c = mesh_mark_down(m, dim, 1, slivers);
  loop_free(slivers);
  memcpy(cand, c, sizeof(unsigned) * ne);
  mesh_unmark_boundary(m, 1, c);
  memcpy(interior, c, sizeof(unsigned) * ne);
  for (unsigned i = 0; i < ne; ++i) {
    good[i] = 0; quals[i] = 0; ring_sizes[i] = 0; indset[i] = 0;
  }
  unsigned any = 0;
  for (unsigned i = 0; i < ne; ++i)
    any |= c[i];
  if (!any) {
    loop_free(c);
    return 0;
  }
  double* q;
  unsigned* rs;
  mesh_swap_qualities(m, c, &q, &rs);
  any = 0;
  for (unsigned i = 0; i < ne; ++i) {
    good[i] = c[i];
    if (c[i]) {
      quals[i] = q[i];
      ring_sizes[i] = rs[i];
      any = 1;
    }
  }
  if (any) {
    unsigned* s = mesh_find_indset(m, 1, c, q);
    memcpy(indset, s, sizeof(unsigned) * ne);
    loop_free(s);
  }
  loop_free(c);
  loop_free(q);
  loop_free(rs);
  return any;
}


// size-field producers (element_gradients.cpp, recover_by_volume.cpp,
// size_from_hessian.cpp, warp_to_limit.cpp); callers only warp meshes whose
// unwarped quality meets the floor, so the halving loop ends
void refd_element_gradients(void* p, char const* name) { mesh_element_gradients(M(p), name); }
void refd_recover_by_volume(void* p, char const* name) { mesh_recover_by_volume(M(p), name); }
void refd_size_from_hessian(void* p, char const* hess_name, double const* weights,
    double min_h, double max_h)
{
  mesh_size_from_hessian(M(p), hess_name, weights, min_h, max_h);
}
unsigned refd_warp_to_limit(void* p, double qual_floor)
{
  return mesh_warp_to_limit(M(p), qual_floor);
}

}
